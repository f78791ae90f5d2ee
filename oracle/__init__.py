"""CPU oracle for the CKKS hot path — TEST INFRASTRUCTURE ONLY.

`ckks_oracle.cpp` restates the reference evaluator's algorithms (pdroalves/aoa,
aoa-ntt) on the CPU; this module builds it (g++, no GPU) and binds it with
ctypes.  Only tests/, the smoke check in __graft_entry__.py and the CPU
baseline / reference arm of bench.py may import this package.  The product
(aoa_b200) never does: its path fails loudly without its CUDA library.

Parity status: pinned on the reference's own outputs.  The reference's
aoa-ntt kernels, built from its sources (oracle/ref/Makefile) and run through
its API on a B200, produced tests/golden/reference_outputs.npz (forward and
inverse hierarchical transforms at 2^10 and 2^12, ModUp, ModDown and rescale
at two levels, on the reference's own primes and precompute); the oracle
equals them word for word (tests/test_oracle_reference_outputs.py).  Its
arithmetic is also checked against exact big-integer results and its
transforms and products against an independent Python model and the
schoolbook negacyclic product (the reference's own NTL-based tests,
aoa-ntt/tests/tests.cpp:300-694); see tests/test_oracle_*.py.
"""
import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_SRC = os.path.join(_HERE, "ckks_oracle.cpp")
_LIB = os.path.join(_HERE, "_build", "liboracle.so")

ST_COEF, ST_NTT = 1, 2


def build(force=False):
    """Compile the oracle shared library (plain g++, OpenMP, no FMA contraction)."""
    if not force and os.path.exists(_LIB) and os.path.getmtime(_LIB) >= os.path.getmtime(_SRC):
        return _LIB
    os.makedirs(os.path.dirname(_LIB), exist_ok=True)
    tmp = _LIB + ".tmp%d" % os.getpid()
    cmd = ["g++", "-O2", "-std=c++17", "-fopenmp", "-ffp-contract=off", "-fPIC", "-shared",
           "-o", tmp, _SRC]
    subprocess.check_call(cmd)
    os.replace(tmp, _LIB)
    return _LIB


_lib = None
u64p = ctypes.POINTER(ctypes.c_uint64)
i64p = ctypes.POINTER(ctypes.c_int64)
f64p = ctypes.POINTER(ctypes.c_double)


def lib():
    global _lib
    if _lib is None:
        _lib = ctypes.CDLL(build())
        L = _lib
        u64, c_int, c_long, vp = ctypes.c_uint64, ctypes.c_int, ctypes.c_long, ctypes.c_void_p
        sigs = {
            "oc_mulmod_exact": (u64, [u64, u64, u64]),
            "oc_powmod": (u64, [u64, u64, u64]),
            "oc_invmod": (u64, [u64, u64]),
            "oc_is_prime": (c_int, [u64]),
            "oc_smallest_primitive_root": (u64, [u64]),
            "oc_gen_ntt_primes": (c_int, [c_int, u64, c_int, u64p]),
            "oc_ref_barrett_mu": (u64, [u64]),
            "oc_ref_mulmod": (u64, [u64, u64, u64]),
            "oc_ref_mod128": (u64, [u64, u64, u64]),
            "oc_ref_mulmod_mismatches": (c_long, [u64, c_long, u64]),
            "oc_set_threads": (None, [c_int]),
            "oc_get_threads": (c_int, []),
            "oc_create": (vp, [c_int, c_int, c_int, u64p, u64p]),
            "oc_destroy": (None, [vp]),
            "oc_ntt_fwd": (None, [vp, u64p, c_int, c_int]),
            "oc_ntt_inv": (None, [vp, u64p, c_int, c_int]),
            "oc_ntt_fwd_batch": (None, [vp, u64p, c_int, c_int, c_int]),
            "oc_ntt_inv_batch": (None, [vp, u64p, c_int, c_int, c_int]),
            "oc_psi": (u64, [vp, c_int]),
            "oc_prime": (u64, [vp, c_int]),
            "oc_proot": (u64, [vp, c_int]),
            "oc_table": (c_int, [vp, c_int, u64p]),
            "oc_modup": (None, [vp, u64p, c_int, u64p]),
            "oc_moddown": (None, [vp, u64p, c_int, u64p]),
            "oc_rescale": (None, [vp, u64p, u64p, c_int]),
            "oc_automorph": (None, [vp, u64p, u64p, c_long, c_int]),
            "oc_swk_gen": (None, [vp, u64p, u64p, u64p, c_int, i64p, u64p, u64p]),
            "oc_square_secret": (None, [vp, u64p, u64p]),
            "oc_rotate_secret": (None, [vp, u64p, c_int, u64p]),
            "oc_conjugate_secret": (None, [vp, u64p, u64p]),
            "oc_hmult": (None, [vp, u64p, u64p, c_int, u64p, u64p, c_int, u64p, u64p, c_int,
                                u64, u64, c_int, u64p, u64p, u64p]),
            "oc_rotate_left": (None, [vp, u64p, u64p, c_int, c_int, u64p, u64p, c_int, u64p, u64p]),
            "oc_conjugate": (None, [vp, u64p, u64p, c_int, u64p, u64p, c_int, u64p, u64p]),
            "oc_add": (c_int, [vp, u64p, u64p, c_int, u64p, u64p, c_int, c_int, u64p, u64p]),
            "oc_encrypt": (None, [vp, u64p, u64p, i64p, i64p, u64p, u64p, c_int, u64p, u64p]),
            "oc_decrypt": (None, [vp, u64p, u64p, c_int, u64p, u64p]),
            "oc_ksi_pows": (None, [c_int, f64p, f64p]),
            "oc_encode": (None, [vp, f64p, f64p, c_int, c_int, u64, c_int, u64p]),
            "oc_decode": (None, [vp, u64p, c_int, u64, f64p, f64p]),
            "oc_fft_special_inv": (None, [c_int, f64p, f64p, c_int]),
            "oc_fft_special": (None, [c_int, f64p, f64p, c_int]),
            "oc_dgt_create": (vp, [c_int, c_int, u64p, u64p, u64p]),
            "oc_dgt_destroy": (None, [vp]),
            "oc_dgt_fwd": (None, [vp, u64p, c_int, c_int]),
            "oc_dgt_inv": (None, [vp, u64p, c_int, c_int]),
            "oc_gi_mul": (None, [vp, u64p, u64p, u64p, c_int, c_int]),
            "oc_dgt_twist": (None, [vp, c_int, u64p, u64p]),
        }
        for name, (res, args) in sigs.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
    return _lib


def P(a):
    """ctypes pointer to a C-contiguous numpy array (u64 / i64 / f64)."""
    if a.dtype == np.uint64:
        return a.ctypes.data_as(u64p)
    if a.dtype == np.int64:
        return a.ctypes.data_as(i64p)
    if a.dtype == np.float64:
        return a.ctypes.data_as(f64p)
    raise TypeError(a.dtype)


def u64(x):
    return np.ascontiguousarray(x, dtype=np.uint64)


def gen_ntt_primes(bits, modulus, count):
    out = np.zeros(count, dtype=np.uint64)
    n = lib().oc_gen_ntt_primes(bits, modulus, count, P(out))
    return [int(v) for v in out[:n]]


class Oracle:
    """One parameter set: ring degree N, k Q primes, kl B primes."""

    def __init__(self, N, q_primes, b_primes, proots=None):
        self.N, self.k, self.kl = N, len(q_primes), len(b_primes)
        self.primes = [int(q) for q in q_primes] + [int(q) for q in b_primes]
        pr = u64(self.primes)
        gp = P(u64(proots)) if proots is not None else None
        self._h = lib().oc_create(N, self.k, self.kl, P(pr), gp)
        if not self._h:
            raise ValueError("oracle: unsupported parameters (2N must divide q-1)")

    def __del__(self):
        if getattr(self, "_h", None):
            lib().oc_destroy(self._h)
            self._h = None

    # -- transforms -------------------------------------------------------
    def ntt_fwd(self, x, first=0):
        x = u64(x).copy()
        lib().oc_ntt_fwd(self._h, P(x), first, x.size // self.N)
        return x

    def ntt_inv(self, x, first=0):
        x = u64(x).copy()
        lib().oc_ntt_inv(self._h, P(x), first, x.size // self.N)
        return x

    def psi(self, rid):
        return int(lib().oc_psi(self._h, rid))

    def proot(self, rid):
        return int(lib().oc_proot(self._h, rid))

    def table(self, which):
        n = lib().oc_table(self._h, which, None)
        out = np.zeros(n, dtype=np.uint64)
        lib().oc_table(self._h, which, P(out))
        return out

    # -- RNS --------------------------------------------------------------
    def modup(self, x_q, level):
        x_q = u64(x_q)
        out = np.zeros((self.kl, self.N), dtype=np.uint64)
        lib().oc_modup(self._h, P(x_q), level, P(out))
        return out

    def moddown(self, x_qb, level):
        x_qb = u64(x_qb)
        out = np.zeros((self.k, self.N), dtype=np.uint64)
        lib().oc_moddown(self._h, P(x_qb), level, P(out))
        return out

    def rescale(self, c0, c1, level):
        c0, c1 = u64(c0).copy(), u64(c1).copy()
        lib().oc_rescale(self._h, P(c0), P(c1), level)
        return c0, c1

    def automorph(self, x, power, nres):
        x = u64(x)
        out = np.zeros_like(x)
        lib().oc_automorph(self._h, P(x), P(out), power, nres)
        return out

    # -- keys -------------------------------------------------------------
    def secret_residues(self, coeffs, nres=None):
        """Signed small coefficients -> [nres][N] residues (sample_hw cast, sampler.cu:157-192)."""
        nres = self.k + self.kl if nres is None else nres
        c = np.asarray(coeffs, dtype=np.int64)
        out = np.zeros((nres, self.N), dtype=np.uint64)
        for r in range(nres):
            q = self.primes[r]
            out[r] = np.where(c >= 0, c, c + q).astype(np.uint64)
        return out

    def swk_gen(self, s1, s2, a, e, a_state=ST_COEF):
        s1, s2, a, e = u64(s1), u64(s2), u64(a), np.ascontiguousarray(e, dtype=np.int64)
        nqb = self.k + self.kl
        ob = np.zeros((nqb, self.N), dtype=np.uint64)
        oa = np.zeros((nqb, self.N), dtype=np.uint64)
        lib().oc_swk_gen(self._h, P(s1), P(s2), P(a), a_state, P(e), P(ob), P(oa))
        return ob, oa

    def square_secret(self, s):
        s = u64(s)
        out = np.zeros_like(s)
        lib().oc_square_secret(self._h, P(s), P(out))
        return out

    def rotate_secret(self, s, r):
        s = u64(s)
        out = np.zeros_like(s)
        lib().oc_rotate_secret(self._h, P(s), r, P(out))
        return out

    def conjugate_secret(self, s):
        s = u64(s)
        out = np.zeros_like(s)
        lib().oc_conjugate_secret(self._h, P(s), P(out))
        return out

    # -- CKKS ops ---------------------------------------------------------
    def hmult(self, a, b, evk, level, scale_a, scale_b, rescale=True, a_state=ST_COEF, b_state=ST_COEF):
        a0, a1 = u64(a[0]), u64(a[1])
        b0, b1 = u64(b[0]), u64(b[1])
        eb, ea = u64(evk[0]), u64(evk[1])
        o0 = np.zeros((self.k, self.N), dtype=np.uint64)
        o1 = np.zeros_like(o0)
        sc = np.zeros(1, dtype=np.uint64)
        lib().oc_hmult(self._h, P(a0), P(a1), a_state, P(b0), P(b1), b_state, P(eb), P(ea),
                       level, int(scale_a), int(scale_b), 1 if rescale else 0, P(o0), P(o1), P(sc))
        return o0, o1, int(sc[0])

    def rotate_left(self, c, r, rtk, level, state=ST_COEF):
        c0, c1 = u64(c[0]), u64(c[1])
        kb, ka = u64(rtk[0]), u64(rtk[1])
        o0 = np.zeros((self.k, self.N), dtype=np.uint64)
        o1 = np.zeros_like(o0)
        lib().oc_rotate_left(self._h, P(c0), P(c1), state, r, P(kb), P(ka), level, P(o0), P(o1))
        return o0, o1

    def conjugate(self, c, cjk, level, state=ST_COEF):
        c0, c1 = u64(c[0]), u64(c[1])
        kb, ka = u64(cjk[0]), u64(cjk[1])
        o0 = np.zeros((self.k, self.N), dtype=np.uint64)
        o1 = np.zeros_like(o0)
        lib().oc_conjugate(self._h, P(c0), P(c1), state, P(kb), P(ka), level, P(o0), P(o1))
        return o0, o1

    def add(self, a, b, subtract=False, a_state=ST_COEF, b_state=ST_COEF):
        a0, a1, b0, b1 = u64(a[0]), u64(a[1]), u64(b[0]), u64(b[1])
        o0 = np.zeros((self.k, self.N), dtype=np.uint64)
        o1 = np.zeros_like(o0)
        st = lib().oc_add(self._h, P(a0), P(a1), a_state, P(b0), P(b1), b_state,
                          1 if subtract else 0, P(o0), P(o1))
        return o0, o1, st

    def encrypt(self, m, u, e1, e2, pk, pk_state=ST_NTT):
        m, u = u64(m), u64(u)
        e1 = np.ascontiguousarray(e1, dtype=np.int64)
        e2 = np.ascontiguousarray(e2, dtype=np.int64)
        pb, pa = u64(pk[0]), u64(pk[1])
        o0 = np.zeros((self.k, self.N), dtype=np.uint64)
        o1 = np.zeros_like(o0)
        lib().oc_encrypt(self._h, P(m), P(u), P(e1), P(e2), P(pb), P(pa), pk_state, P(o0), P(o1))
        return o0, o1

    def decrypt(self, c, s, state=ST_NTT):
        c0, c1, s = u64(c[0]), u64(c[1]), u64(s)
        out = np.zeros((self.k, self.N), dtype=np.uint64)
        lib().oc_decrypt(self._h, P(c0), P(c1), state, P(s), P(out))
        return out

    def encode(self, values, scale, empty=0, nres=None):
        v = np.asarray(values, dtype=np.complex128)
        re = np.ascontiguousarray(v.real)
        im = np.ascontiguousarray(v.imag)
        nres = self.k if nres is None else nres
        out = np.zeros((nres, self.N), dtype=np.uint64)
        lib().oc_encode(self._h, P(re), P(im), len(v), empty, int(scale), nres, P(out))
        return out

    def decode(self, m0, slots, scale):
        m0 = u64(m0)
        re = np.zeros(slots)
        im = np.zeros(slots)
        lib().oc_decode(self._h, P(m0), slots, int(scale), P(re), P(im))
        return re + 1j * im


def reference_prime_set(table, k, kl, prec):
    """Q and B primes as fill_ckks_coprimes_bucket picks them (aoa-ntt
    src/cuda/manager.cu:426-464) from the fixture `table` (reference_primes.json)."""
    b = table["buckets"]
    q0 = b["63"][0]
    if prec in (45, 55):
        bucket = b[str(prec)]
        return [q0] + bucket[:k - 1], bucket[k - 1:k - 1 + kl]
    if prec in (48, 52):
        return [q0] + b[str(prec)][:k - 1], b["55"][:kl]
    raise ValueError("the reference supports prec 45/48/52/55 only")


def reference_proots(table, primes):
    return [int(table["proots"][str(q)]) for q in primes]


class DgtOracle:
    """The reference's DGT (aoa-dgt src/cuda/dgt.cu) for folded length N = n/2
    over `primes`, with generators `proots` and roots r (r^N = i) given as
    (re, im) pairs.  Arrays are [nres][N][2] uint64 (re, im interleaved, the
    reference's GaussianInteger layout)."""

    def __init__(self, N, primes, proots, roots):
        self.N = N
        self.primes = [int(q) for q in primes]
        pa = np.array(self.primes, dtype=np.uint64)
        ga = np.array([int(g) for g in proots], dtype=np.uint64)
        ra = np.array([int(v) for r in roots for v in r], dtype=np.uint64)
        self._h = lib().oc_dgt_create(N, len(self.primes), P(pa), P(ga), P(ra))

    def __del__(self):
        if getattr(self, "_h", None):
            lib().oc_dgt_destroy(self._h)
            self._h = None

    def fwd(self, x, first=0):
        y = u64(x).copy()
        lib().oc_dgt_fwd(self._h, P(y), first, y.shape[0])
        return y

    def inv(self, x, first=0):
        y = u64(x).copy()
        lib().oc_dgt_inv(self._h, P(y), first, y.shape[0])
        return y

    def gi_mul(self, a, b, first=0):
        a, b = u64(a), u64(b)
        c = np.zeros_like(a)
        lib().oc_gi_mul(self._h, P(a), P(b), P(c), first, a.shape[0])
        return c

    def twist(self, rid):
        nth = np.zeros((self.N, 2), dtype=np.uint64)
        inv = np.zeros_like(nth)
        lib().oc_dgt_twist(self._h, rid, P(nth), P(inv))
        return nth, inv


def fold(coeffs):
    """[nres][2N] coefficients -> [nres][N][2] Gaussian integers a_j + i a_{j+N}
    (poly_copy_to_device, aoa-dgt src/arithmetic/polynomial.cu:92-116)."""
    c = u64(coeffs)
    n2 = c.shape[-1] // 2
    return np.ascontiguousarray(np.stack([c[..., :n2], c[..., n2:]], axis=-1))


def unfold(gi):
    """Inverse of fold (poly_copy_to_host, polynomial.cu:118-154)."""
    g = u64(gi)
    return np.ascontiguousarray(np.concatenate([g[..., 0], g[..., 1]], axis=-1))


def dgt_prime_set(table, k, kl, prec):
    """Q and B primes as the DGT variant's fill_ckks_coprimes_bucket picks them
    (aoa-dgt src/cuda/cudaengine.cu:545-583): B continues the 55-bit bucket at
    index k-1 for every precision but 45."""
    b = table["buckets"]
    q0 = b["63"][0]
    if prec == 45:
        return [q0] + b["45"][:k - 1], b["45"][k - 1:k - 1 + kl]
    if prec in (48, 52, 55):
        return [q0] + b[str(prec)][:k - 1], b["55"][k - 1:k - 1 + kl]
    raise ValueError("the DGT variant supports prec 45/48/52/55 only")


def dgt_roots(table, primes, N):
    """(generators, roots r with r^N = i) of `primes` from the fixture
    (tests/golden/dgt_roots.json)."""
    g = [int(table["proots"][str(q)]) for q in primes]
    r = [tuple(int(v) for v in table["nthroot"][str(q)][str(N)]) for q in primes]
    return g, r
