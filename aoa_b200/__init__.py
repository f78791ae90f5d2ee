"""aoa_b200 — B200-native CKKS evaluation engine (host-side Python mirror).

The compute path is libaoa_b200.so (hand-written sm_100a CUDA behind the C ABI
in include/aoa_ckks.h).  This package wraps that ABI with the objects of the
reference's API (pdroalves/aoa aoa-ntt: CUDAManager/Context/poly_t/cipher_t
and the ckks_* free functions) for Python callers, tests and the benchmark.
"""
import ctypes

import numpy as np

from . import capi
from .capi import AoaError, AOA_COEF, AOA_NTT, AOA_DGT

__all__ = ["Engine", "Context", "DeviceArray", "AoaError", "AOA_COEF", "AOA_NTT", "AOA_DGT"]


class Engine:
    """One parameter set (ring degree, Q primes, special primes).

    Replaces CUDAManager::init(k, kl, N, scalingfactor) (aoa-ntt
    src/cuda/manager.cu:762-800) with explicit prime lists.
    """

    def __init__(self, log_n, q_primes, b_primes, scale_bits=0, generators=None, dgt_roots=None):
        lib = capi.load()
        self.log_n, self.N = log_n, 1 << log_n
        self.q_primes = [int(q) for q in q_primes]
        self.b_primes = [int(q) for q in b_primes]
        self.k, self.kl = len(self.q_primes), len(self.b_primes)
        self.primes = self.q_primes + self.b_primes
        self._primes_arr = np.array(self.primes, dtype=np.uint64)
        self._gens_arr = None if generators is None else np.array(generators, dtype=np.uint64)
        p = capi.Params()
        p.log_n, p.k, p.kl = log_n, self.k, self.kl
        p.primes = self._primes_arr.ctypes.data_as(capi.u64p)
        p.generators = None if self._gens_arr is None else self._gens_arr.ctypes.data_as(capi.u64p)
        p.scale_bits, p.dnum = scale_bits, 1
        self._roots_arr = None if dgt_roots is None else np.array([int(v) for r in dgt_roots for v in r],
                                                                   dtype=np.uint64)
        p.dgt_roots = None if self._roots_arr is None else self._roots_arr.ctypes.data_as(capi.u64p)
        self.scale_bits = scale_bits
        h = ctypes.c_void_p()
        capi.check(lib.aoa_engine_create(ctypes.byref(p), ctypes.byref(h)))
        self.handle = h

    def tune(self, knob, value):
        """Set a launch-shape knob ("ntt_split", "dgt_split", "ntt_cols_div", "ntt_cols_kind",
        "ntt_rows_div", "ntt_waves", "ntt_waves_large", "ntt_chunk_bytes",
        "ntt_cols_tma", "conv_tensor_cores", "fuse", "batch_streams", "spin_limit")."""
        capi.check(capi.load().aoa_engine_tune(self.handle, knob.encode(), float(value)))

    TRANSFORM_KNOBS = ("ntt_split", "ntt_cols_div", "ntt_cols_kind", "ntt_rows_div", "ntt_waves",
                       "ntt_waves_large", "ntt_chunk_bytes")

    def tune_get(self, knob):
        """Current value of a launch-shape knob."""
        v = ctypes.c_double()
        capi.check(capi.load().aoa_engine_tune_get(self.handle, knob.encode(), ctypes.byref(v)))
        return v.value

    def transform_shapes(self):
        """The transform knobs as a dict (ints where the knob is integral)."""
        out = {}
        for k in self.TRANSFORM_KNOBS:
            v = self.tune_get(k)
            out[k] = int(v) if v == int(v) else v
        return out

    def autotune(self, limbs=0):
        """Time candidate transform shapes on this engine's ring and keep the
        fastest; returns the tuner's report (choice, timings in ms)."""
        import json
        buf = ctypes.create_string_buffer(1 << 16)
        capi.check(capi.load().aoa_engine_autotune(self.handle, int(limbs), buf, len(buf)))
        return json.loads(buf.value.decode())

    def close(self):
        if getattr(self, "handle", None):
            capi.load().aoa_engine_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Context:
    """A CUDA stream bound to an engine (reference Context, tool/context.h:16-49)."""

    def __init__(self, engine, stream=None):
        self.engine = engine
        h = ctypes.c_void_p()
        capi.check(capi.load().aoa_ctx_create(engine.handle, stream, ctypes.byref(h)))
        self.handle = h

    @property
    def stream(self):
        s = ctypes.c_void_p()
        capi.check(capi.load().aoa_ctx_stream(self.handle, ctypes.byref(s)))
        return s.value

    def sync(self):
        capi.check(capi.load().aoa_ctx_sync(self.handle))

    def close(self):
        if getattr(self, "handle", None):
            capi.load().aoa_ctx_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- memory ------------------------------------------------------------
    def alloc(self, shape, dtype=np.uint64):
        return DeviceArray(self, shape, dtype)

    def upload(self, host):
        host = np.ascontiguousarray(host)
        d = DeviceArray(self, host.shape, host.dtype)
        d.copy_from(host)
        return d

    # -- transforms ------------------------------------------------------------
    def ntt_fwd(self, d, npolys, first_prime, nlimbs, poly_stride=None):
        capi.check(capi.load().aoa_ntt_fwd(self.handle, d.ptr, npolys, first_prime, nlimbs,
                                           poly_stride or nlimbs))

    def ntt_inv(self, d, npolys, first_prime, nlimbs, poly_stride=None):
        capi.check(capi.load().aoa_ntt_inv(self.handle, d.ptr, npolys, first_prime, nlimbs,
                                           poly_stride or nlimbs))

    def dgt_fwd(self, d, npolys, first_prime, nlimbs, poly_stride=None):
        """DGT of planar GI limbs (DGTEngine::execute_dgt FORWARD)."""
        capi.check(capi.load().aoa_dgt_fwd(self.handle, d.ptr, npolys, first_prime, nlimbs,
                                           poly_stride or nlimbs))

    def dgt_inv(self, d, npolys, first_prime, nlimbs, poly_stride=None):
        capi.check(capi.load().aoa_dgt_inv(self.handle, d.ptr, npolys, first_prime, nlimbs,
                                           poly_stride or nlimbs))

    def set_transform(self, domain):
        """AOA_NTT (aoa-ntt) or AOA_DGT (aoa-dgt) for this context's evaluations."""
        capi.check(capi.load().aoa_ctx_set_transform(self.handle, domain))


class DeviceArray:
    """Device allocation on a context's stream (stream-ordered malloc/free)."""

    def __init__(self, ctx, shape, dtype=np.uint64):
        self.ctx, self.shape, self.dtype = ctx, tuple(np.atleast_1d(shape)), np.dtype(dtype)
        self.nbytes = int(np.prod(self.shape)) * self.dtype.itemsize
        h = ctypes.c_void_p()
        capi.check(capi.load().aoa_device_alloc(ctx.handle, max(self.nbytes, 8), ctypes.byref(h)))
        self.ptr = h

    def copy_from(self, host):
        host = np.ascontiguousarray(host, dtype=self.dtype)
        assert host.nbytes == self.nbytes
        capi.check(capi.load().aoa_memcpy_h2d(self.ctx.handle, self.ptr, capi.ptr(host), self.nbytes))
        self.ctx.sync()

    def numpy(self):
        out = np.empty(self.shape, dtype=self.dtype)
        capi.check(capi.load().aoa_memcpy_d2h(self.ctx.handle, capi.ptr(out), self.ptr, self.nbytes))
        self.ctx.sync()
        return out

    def offset(self, elements):
        return ctypes.c_void_p(self.ptr.value + elements * self.dtype.itemsize)

    def free(self):
        if getattr(self, "ptr", None) is not None and self.ctx.handle:
            capi.load().aoa_device_free(self.ctx.handle, self.ptr)
            self.ptr = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


class Ciphertext:
    """cipher_t on the device: two polys of k limbs, level, slots, scale, domain."""

    def __init__(self, ctx):
        self.ctx = ctx
        h = ctypes.c_void_p()
        capi.check(capi.load().aoa_ct_create(ctx.handle, ctypes.byref(h)))
        self.handle = h

    @classmethod
    def from_residues(cls, ctx, c0, c1, level=None, slots=0, scale=None, domain=AOA_COEF):
        ct = cls(ctx)
        ct.upload(c0, c1, domain)
        E = ctx.engine
        nl = np.asarray(c0).shape[0]
        ct.set(level if level is not None else nl - 1, slots,
               scale if scale is not None else (1 << E.scale_bits if E.scale_bits else 1), domain)
        return ct

    def copy(self):
        """A new ciphertext with a device copy of this one's data and metadata."""
        out = Ciphertext(self.ctx)
        E = self.ctx.engine
        lib = capi.load()
        src, dst = ctypes.c_void_p(), ctypes.c_void_p()
        capi.check(lib.aoa_ct_data(self.handle, ctypes.byref(src)))
        capi.check(lib.aoa_ct_data(out.handle, ctypes.byref(dst)))
        capi.check(lib.aoa_memcpy_d2d(self.ctx.handle, dst, src, 2 * E.k * E.N * 8))
        level, slots, scale, domain = self._get()
        out.set(level, slots, scale, domain)
        return out

    def upload(self, c0, c1, domain=AOA_COEF):
        host = np.ascontiguousarray(np.stack([np.asarray(c0, dtype=np.uint64), np.asarray(c1, dtype=np.uint64)]))
        capi.check(capi.load().aoa_ct_upload(self.ctx.handle, self.handle, capi.ptr(host), host.shape[1], domain))
        self.ctx.sync()

    def download(self, nlimbs=None, domain=AOA_COEF):
        nlimbs = nlimbs or (self.level + 1)
        out = np.empty((2, nlimbs, self.ctx.engine.N), dtype=np.uint64)
        capi.check(capi.load().aoa_ct_download(self.ctx.handle, self.handle, capi.ptr(out), nlimbs, domain))
        return out[0], out[1]

    def set(self, level, slots, scale, domain):
        capi.check(capi.load().aoa_ct_set(self.handle, level, slots, int(scale), domain))

    def _get(self):
        lv, sl, dm = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        sc = ctypes.c_uint64()
        capi.check(capi.load().aoa_ct_get(self.handle, ctypes.byref(lv), ctypes.byref(sl), ctypes.byref(sc),
                                          ctypes.byref(dm)))
        return lv.value, sl.value, sc.value, dm.value

    level = property(lambda self: self._get()[0])
    slots = property(lambda self: self._get()[1])
    scale = property(lambda self: self._get()[2])
    domain = property(lambda self: self._get()[3])

    @property
    def device_ptr(self):
        p = ctypes.c_void_p()
        capi.check(capi.load().aoa_ct_data(self.handle, ctypes.byref(p)))
        return p

    def close(self):
        if getattr(self, "handle", None) and self.ctx.handle:
            capi.load().aoa_ct_destroy(self.ctx.handle, self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class SwitchKey:
    """SwitchKey {b, a} over the QB basis (relinearisation, rotation or conjugation key)."""

    def __init__(self, ctx, b, a, domain=AOA_NTT, handle=None):
        self.ctx = ctx
        if handle is not None:
            self.handle = handle
            return
        b = np.ascontiguousarray(b, dtype=np.uint64)
        a = np.ascontiguousarray(a, dtype=np.uint64)
        h = ctypes.c_void_p()
        capi.check(capi.load().aoa_swk_create(ctx.handle, capi.ptr(b), capi.ptr(a), domain, ctypes.byref(h)))
        self.handle = h

    @classmethod
    def generate(cls, ctx, s1, s2, a, e, a_domain=AOA_COEF):
        """Switching key for s1 under s2 (b = rho(s1) + e - a s2, a) from given
        draws; s1 / s2 / a are [k+kl][N] device arrays (s1 may be None), e a
        device array of N int64 (ckks_new_evk & co., ckkskeys.cpp:101-191)."""
        h = ctypes.c_void_p()
        capi.check(capi.load().aoa_swk_generate(ctx.handle, None if s1 is None else s1.ptr, s2.ptr, a.ptr, a_domain,
                                                e.ptr, ctypes.byref(h)))
        return cls(ctx, None, None, handle=h)

    def numpy(self):
        """(b, a, domain) copied to the host."""
        d = ctypes.c_void_p()
        dom = ctypes.c_int()
        capi.check(capi.load().aoa_swk_data(self.handle, ctypes.byref(d), ctypes.byref(dom)))
        E = self.ctx.engine
        out = np.empty((2, len(E.primes), E.N), dtype=np.uint64)
        capi.check(capi.load().aoa_memcpy_d2h(self.ctx.handle, capi.ptr(out), d, out.nbytes))
        self.ctx.sync()
        return out[0], out[1], dom.value

    def close(self):
        if getattr(self, "handle", None) and self.ctx.handle:
            capi.load().aoa_swk_destroy(self.ctx.handle, self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _h(x):
    return None if x is None else x.handle


# ---- reference-named evaluation API (aoa-ntt include/newckks/ckks/ckks.h) -------

def ckks_mul(ctx, c3, c1, c2, evk):
    """HMult + relinearise + rescale into c3 (ckks_mul, ckks.cpp:334-347)."""
    capi.check(capi.load().aoa_hmult_relin_rescale(ctx.handle, c3.handle, c1.handle, c2.handle, _h(evk)))


def ckks_mul_without_rescale(ctx, c3, c1, c2, evk):
    capi.check(capi.load().aoa_hmult(ctx.handle, c3.handle, c1.handle, c2.handle, _h(evk)))


def ckks_rescale(ctx, c):
    capi.check(capi.load().aoa_rescale(ctx.handle, c.handle))


def ckks_add(ctx, c3, c1, c2):
    capi.check(capi.load().aoa_add(ctx.handle, c3.handle, c1.handle, c2.handle))


def ckks_sub(ctx, c3, c1, c2):
    capi.check(capi.load().aoa_sub(ctx.handle, c3.handle, c1.handle, c2.handle))


def ckks_rotate_left(ctx, c2, c1, steps, rtk):
    capi.check(capi.load().aoa_rotate(ctx.handle, c2.handle, c1.handle, steps, _h(rtk)))


def ckks_rotate_right(ctx, c2, c1, steps, rtk):
    capi.check(capi.load().aoa_rotate(ctx.handle, c2.handle, c1.handle, -steps, _h(rtk)))


def ckks_conjugate(ctx, c2, c1, cjk):
    capi.check(capi.load().aoa_conjugate(ctx.handle, c2.handle, c1.handle, _h(cjk)))


class PinnedArray:
    """Page-locked host array (aoa_host_alloc) viewed as numpy."""

    def __init__(self, shape, dtype=np.uint64):
        self.shape, self.dtype = tuple(shape), np.dtype(dtype)
        nbytes = int(np.prod(self.shape)) * self.dtype.itemsize
        h = ctypes.c_void_p()
        capi.check(capi.load().aoa_host_alloc(max(nbytes, 8), ctypes.byref(h)))
        self.ptr = h
        buf = (ctypes.c_char * max(nbytes, 8)).from_address(h.value)
        self.array = np.frombuffer(buf, dtype=self.dtype, count=int(np.prod(self.shape))).reshape(self.shape)

    def free(self):
        if getattr(self, "ptr", None) is not None:
            self.array = None
            capi.load().aoa_host_free(self.ptr)
            self.ptr = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


def kernel_launches():
    """Kernels launched by libaoa_b200.so so far in this process."""
    return int(capi.load().aoa_kernel_launches())


def ckks_mul_plain(ctx, c3, c1, c2, evk):
    """The reference's per-call ckks_mul sequence on this engine (comparison path)."""
    capi.check(capi.load().aoa_hmult_plain(ctx.handle, c3.handle, c1.handle, c2.handle, _h(evk)))


def ckks_rotate_plain(ctx, c2, c1, steps, rtk):
    """The reference's per-call ckks_rotate_left sequence on this engine
    (comparison path; output in coefficients)."""
    capi.check(capi.load().aoa_rotate_plain(ctx.handle, c2.handle, c1.handle, steps, _h(rtk)))


def ckks_conjugate_plain(ctx, c2, c1, cjk):
    """The reference's per-call ckks_conjugate sequence on this engine (comparison path)."""
    capi.check(capi.load().aoa_conjugate_plain(ctx.handle, c2.handle, c1.handle, _h(cjk)))


def ckks_mul_batch(ctx, outs, c1s, c2s, evk, rescale=True):
    """outs[i] = c1s[i] * c2s[i] (+ relinearise, + rescale) in grouped batched launches."""
    n = len(outs)
    if not (len(c1s) == len(c2s) == n):
        raise ValueError("batch lists differ in length")
    arr = ctypes.c_void_p * max(n, 1)
    o = arr(*[x.handle.value for x in outs])
    a = arr(*[x.handle.value for x in c1s])
    b = arr(*[x.handle.value for x in c2s])
    capi.check(capi.load().aoa_hmult_batch(ctx.handle, n, o, a, b, _h(evk), 1 if rescale else 0))


def ckks_rotate_batch(ctx, outs, cts, steps, rtk):
    """outs[i] = cts[i] rotated left by `steps` slots, one key for the batch,
    in grouped batched launches."""
    n = len(outs)
    if len(cts) != n:
        raise ValueError("batch lists differ in length")
    arr = ctypes.c_void_p * max(n, 1)
    capi.check(capi.load().aoa_rotate_batch(ctx.handle, n, arr(*[x.handle.value for x in outs]),
                                            arr(*[x.handle.value for x in cts]), steps, _h(rtk)))


def ckks_rotate_batch_steps(ctx, outs, cts, steps, rtks):
    """outs[i] = cts[i] rotated left by steps[i] slots with rtks[i], grouped by
    level only (ops of different steps share the launches)."""
    n = len(outs)
    if not (len(cts) == len(steps) == len(rtks) == n):
        raise ValueError("batch lists differ in length")
    arr = ctypes.c_void_p * max(n, 1)
    st = (ctypes.c_int * max(n, 1))(*[int(s) for s in steps])
    capi.check(capi.load().aoa_rotate_batch_steps(ctx.handle, n, arr(*[x.handle.value for x in outs]),
                                                  arr(*[x.handle.value for x in cts]), st,
                                                  arr(*[None if k is None else k.handle.value for k in rtks])))


def ckks_conjugate_batch(ctx, outs, cts, cjk):
    n = len(outs)
    if len(cts) != n:
        raise ValueError("batch lists differ in length")
    arr = ctypes.c_void_p * max(n, 1)
    capi.check(capi.load().aoa_conjugate_batch(ctx.handle, n, arr(*[x.handle.value for x in outs]),
                                               arr(*[x.handle.value for x in cts]), _h(cjk)))


# ---- encoder and encryption (aoa-ntt src/ckks/encoder.cu, ckks.cpp:87-192) --------

def ckks_encode(ctx, values, empty_slots=0, scale=None, nlimbs=None, domain=AOA_COEF, out=None):
    """Encode complex `values` (+ `empty_slots` zeros) into a [nlimbs][N] device
    polynomial (CKKSContext::encode, ckkscontext.cpp:5-19).  Returns (poly, scale)."""
    eng = ctx.engine
    if scale is None:
        scale = 1 << eng.scale_bits
    nlimbs = nlimbs or eng.k
    v = np.ascontiguousarray(np.asarray(values, dtype=np.complex128))
    out = out if out is not None else ctx.alloc((nlimbs, eng.N))
    capi.check(capi.load().aoa_encode(ctx.handle, capi.ptr(v) if v.size else None, v.size, empty_slots,
                                      int(scale), nlimbs, domain, out.ptr))
    return out, int(scale)


def ckks_decode(ctx, poly, slots, scale, domain=AOA_COEF):
    """Decode `slots` complex values from limb 0 of a device polynomial
    (CKKSContext::decode, ckkscontext.cpp:21-38)."""
    out = np.empty(slots, dtype=np.complex128)
    capi.check(capi.load().aoa_decode(ctx.handle, poly.ptr, domain, slots, int(scale), capi.ptr(out)))
    return out


def ckks_encrypt(ctx, values, pk, u, e1, e2, empty_slots=0, scale=None, out=None):
    """Encode and encrypt (ckks_encrypt, ckks.cpp:109-128) with the sampler's
    draws given: u (ternary), e1, e2 (Gaussian) as N signed integers each."""
    m, scale = ckks_encode(ctx, values, empty_slots, scale)
    dv = [ctx.upload(np.ascontiguousarray(x, dtype=np.int64)) for x in (u, e1, e2)]
    out = out if out is not None else Ciphertext(ctx)
    slots = len(values) + empty_slots
    capi.check(capi.load().aoa_encrypt(ctx.handle, out.handle, m.ptr, AOA_COEF, pk.handle, dv[0].ptr, dv[1].ptr,
                                       dv[2].ptr, slots, int(scale)))
    ctx.sync()
    return out


def ckks_decrypt_poly(ctx, ct, sk, sk_domain=AOA_COEF):
    """m = c1 s + c0 (ckks_decrypt_poly, ckks.cpp:179-192) as a device array
    [level+1][N] in coefficients; sk is a [k][N] device array."""
    m = ctx.alloc((ct.level + 1, ctx.engine.N))
    capi.check(capi.load().aoa_decrypt(ctx.handle, ct.handle, sk.ptr, sk_domain, m.ptr))
    return m


def ckks_decrypt(ctx, ct, sk, sk_domain=AOA_COEF):
    """Decrypt and decode (ckks_decrypt, ckks.cpp:195-215)."""
    m = ckks_decrypt_poly(ctx, ct, sk, sk_domain)
    return ckks_decode(ctx, m, ct.slots, ct.scale)


# ---- key generation (CKKSKeychain, aoa-ntt src/ckks/ckkskeys.cpp:20-191) ----------

def galois_left(N, r):
    """Galois element of a left rotation by r slots: 5^r mod 2N."""
    return pow(5, r % (N // 2), 2 * N)


def galois_conjugate(N):
    return 2 * N - 1


def ckks_pk_generate(ctx, s, a, e, a_domain=AOA_COEF, out=None):
    """Public key (e - a s, a) over Q as a ciphertext (ckks_new_pk); s, a: [k][N]
    device arrays, e: device array of N int64."""
    out = out if out is not None else Ciphertext(ctx)
    capi.check(capi.load().aoa_pk_generate(ctx.handle, out.handle, s.ptr, a.ptr, a_domain, e.ptr))
    return out


def ckks_secret_square(ctx, s, nlimbs):
    out = ctx.alloc((nlimbs, ctx.engine.N))
    capi.check(capi.load().aoa_secret_square(ctx.handle, s.ptr, out.ptr, nlimbs))
    return out


def ckks_secret_galois(ctx, s, galois, nlimbs):
    out = ctx.alloc((nlimbs, ctx.engine.N))
    capi.check(capi.load().aoa_secret_galois(ctx.handle, s.ptr, out.ptr, int(galois), nlimbs))
    return out


def ckks_keygen(ctx, s, draws, rotations=(), conjugation=False):
    """All keys of a secret s ([k+kl][N] device residues, coefficients) from the
    sampler draws `draws` (a dict of device arrays: "pk": (a, e), "evk": (a, e),
    ("rtk", r): (a, e), "cjk": (a, e); a uniform [k+kl][N], e N int64), on the
    device (ckks_new_keys, ckkskeys.cpp:20-73).  Returns a dict of keys."""
    E = ctx.engine
    nqb = len(E.primes)
    keys = {}
    a, e = draws["pk"]
    keys["pk"] = ckks_pk_generate(ctx, s, a, e)
    s2 = ckks_secret_square(ctx, s, nqb)
    a, e = draws["evk"]
    keys["evk"] = SwitchKey.generate(ctx, s2, s, a, e)
    keys["rtk"] = {}
    for r in rotations:
        sr = ckks_secret_galois(ctx, s, galois_left(E.N, r), nqb)
        a, e = draws[("rtk", r)]
        keys["rtk"][r] = SwitchKey.generate(ctx, sr, s, a, e)
    if conjugation:
        sc = ckks_secret_galois(ctx, s, galois_conjugate(E.N), nqb)
        a, e = draws["cjk"]
        keys["cjk"] = SwitchKey.generate(ctx, sc, s, a, e)
    return keys


# ---- plaintext / constant operations (aoa-ntt src/ckks/ckks.cpp:423-690) ----------

def ckks_mul_pt(ctx, out, ct, pt, pt_scale, pt_domain=AOA_COEF, rescale=True):
    """out = ct * pt for an encoded plaintext device array pt ([k][N])."""
    capi.check(capi.load().aoa_mul_plaintext(ctx.handle, out.handle, ct.handle, pt.ptr, pt_domain, int(pt_scale),
                                             1 if rescale else 0))


def ckks_mul_values(ctx, out, ct, values, rescale=True):
    """ckks_mul(ctx, c2, c1, complex*) (ckks.cpp:610-632): encode at the
    ciphertext's scale and slot count, multiply, rescale."""
    v = np.asarray(values, dtype=np.complex128)
    pt, scale = ckks_encode(ctx, v, empty_slots=ct.slots - v.size, scale=ct.scale)
    ckks_mul_pt(ctx, out, ct, pt, scale, rescale=rescale)


def ckks_mul_const(ctx, out, ct, val, rescale=True):
    capi.check(capi.load().aoa_mul_const(ctx.handle, out.handle, ct.handle, float(val), 1 if rescale else 0))


def ckks_add_const(ctx, out, ct, val):
    capi.check(capi.load().aoa_add_const(ctx.handle, out.handle, ct.handle, float(val)))


def ckks_sumslots(ctx, out, ct, rtks):
    """Rotate-and-sum over the slots (ckks_sumslots); rtks maps each power-of-two
    step 2^j to its left-rotation SwitchKey."""
    n = max((s.bit_length() for s in rtks), default=0)
    arr = (ctypes.c_void_p * max(n, 1))()
    for step, key in rtks.items():
        arr[step.bit_length() - 1] = key.handle.value
    capi.check(capi.load().aoa_sumslots(ctx.handle, out.handle, ct.handle, arr, n))


def ckks_batch_inner_prod(ctx, out, ct, other, rtks):
    """ckks_batch_inner_prod (ckks.cpp:470-482): multiply (by a ciphertext, a
    SwitchKey-relinearised product needs evk in `rtks["evk"]`, or by complex
    values) then sum the slots."""
    if isinstance(other, Ciphertext):
        ckks_mul(ctx, out, ct, other, rtks["evk"])
    else:
        ckks_mul_values(ctx, out, ct, other)
    ckks_sumslots(ctx, out, out, {k: v for k, v in rtks.items() if isinstance(k, int)})


# ---- device samplers (Philox4x32-10; Sampler, aoa-ntt src/cuda/sampler.cu) ----------

def sample_uniform(ctx, first_prime, nlimbs, seed, stream=0):
    """[nlimbs][N] uniform residues under primes first_prime.. on the device."""
    out = ctx.alloc((nlimbs, ctx.engine.N))
    capi.check(capi.load().aoa_sample_uniform(ctx.handle, out.ptr, first_prime, nlimbs, seed, stream))
    return out


def sample_gaussian(ctx, n, seed, stream=0, sigma=3.2):
    """n rounded Gaussian integers (int64) on the device (sample_DG)."""
    out = ctx.alloc((n,), np.int64)
    capi.check(capi.load().aoa_sample_gaussian(ctx.handle, out.ptr, n, float(sigma), seed, stream))
    return out


def sample_ternary(ctx, n, hw, seed, stream=0):
    """n int64 in {-1, 0, 1} with exactly hw non-zeros (sample_hw / sample_Z0)."""
    out = ctx.alloc((n,), np.int64)
    capi.check(capi.load().aoa_sample_ternary(ctx.handle, out.ptr, n, hw, seed, stream))
    return out


def ckks_keygen_sampled(ctx, seed, rotations=(), conjugation=False, hw=64):
    """Secret (ternary, Hamming weight hw) and all keys from the device
    samplers (streams 0..: secret, pk a / e, evk a / e, then per rotation key
    and the conjugation key).  Returns (secret as [k+kl][N] residues on the
    device, keys)."""
    E = ctx.engine
    nqb = len(E.primes)
    s_int = sample_ternary(ctx, E.N, hw, seed, 0)
    s = ctx.alloc((nqb, E.N))
    capi.check(capi.load().aoa_signed_to_residues(ctx.handle, s_int.ptr, s.ptr, 0, nqb))
    stream = [1]

    def draw():
        a = sample_uniform(ctx, 0, nqb, seed, stream[0])
        e = sample_gaussian(ctx, E.N, seed, stream[0] + 1)
        stream[0] += 2
        return a, e
    draws = {"pk": draw(), "evk": draw()}
    for r in rotations:
        draws[("rtk", r)] = draw()
    if conjugation:
        draws["cjk"] = draw()
    return s, ckks_keygen(ctx, s, draws, rotations, conjugation)


def ckks_encrypt_sampled(ctx, values, pk, seed, stream=0, empty_slots=0, scale=None, out=None):
    """ckks_encrypt with its draws from the device samplers: u ternary with N/2
    non-zeros (sample_Z0), e1 and e2 rounded Gaussian (streams stream ..
    stream + 2)."""
    m, scale = ckks_encode(ctx, values, empty_slots, scale)
    N = ctx.engine.N
    u = sample_ternary(ctx, N, N // 2, seed, stream)
    e1 = sample_gaussian(ctx, N, seed, stream + 1)
    e2 = sample_gaussian(ctx, N, seed, stream + 2)
    out = out if out is not None else Ciphertext(ctx)
    capi.check(capi.load().aoa_encrypt(ctx.handle, out.handle, m.ptr, AOA_COEF, pk.handle, u.ptr, e1.ptr, e2.ptr,
                                       len(values) + empty_slots, int(scale)))
    return out


# ---- compositions (aoa-ntt src/ckks/ckks.cpp:423-455, 732-906) ---------------------

# Maclaurin coefficients of the reference's function approximations
# (CKKSContext, aoa-ntt include/newckks/ckks/ckkscontext.h:101-120), with the
# number of terms each of its functions evaluates (ckks.cpp:813-906).  The
# values are the reference's, quirks included (its cosine table), so that the
# results match it.
MACLAURIN = {
    "exp": ([1.0, 1.0, 1.0 / 2, 1.0 / 6, 1.0 / 24, 1.0 / 120, 1.0 / 720, 1.0 / 5040, 1.0 / 40320, 1.0 / 362880,
             1.0 / 3628800], 11),
    "sin": ([0.0, 1.0, 0.0, -1.0 / 6, 0.0, 1.0 / 120, 0.0, -1.0 / 5040, 0.0, 1.0 / 362880, 0.0, -1.0 / 39916800], 12),
    "cos": ([1.0, 0.0, -0.5, 1.0 / 24, 0.0, -1.0 / 720, 0.0, 1.0 / 40320, 0.0, -1.0 / 362880, 0.0, 1.0 / 362880], 12),
    "sigmoid": ([1.0 / 2, 1.0 / 4, 0.0, -1.0 / 48, 0.0, 1.0 / 480, 0.0, -17.0 / 80640, 0.0, 31.0 / 1451520], 8),
}


def ckks_power(ctx, out, ct, x, evk):
    """ct^x by square-and-multiply (ckks_power)."""
    capi.check(capi.load().aoa_power(ctx.handle, out.handle, ct.handle, int(x), evk.handle if evk else None))


def ckks_eval_polynomial(ctx, out, ct, coeffs, evk):
    """sum_i coeffs[i] ct^i by Horner's rule (ckks_eval_polynomial)."""
    c = np.ascontiguousarray(coeffs, dtype=np.float64)
    capi.check(capi.load().aoa_eval_polynomial(ctx.handle, out.handle, ct.handle,
                                               c.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), c.size,
                                               evk.handle))


def _maclaurin(name):
    def f(ctx, out, ct, evk):
        coeffs, n = MACLAURIN[name]
        ckks_eval_polynomial(ctx, out, ct, coeffs[:n], evk)
    f.__name__ = "ckks_" + name
    f.__doc__ = "ckks_%s: the reference's %d-term Maclaurin polynomial." % (name, MACLAURIN[name][1])
    return f


ckks_exp = _maclaurin("exp")
ckks_sin = _maclaurin("sin")
ckks_cos = _maclaurin("cos")
ckks_sigmoid = _maclaurin("sigmoid")


def ckks_inner_prod(ctx, out, a, b, evk=None):
    """sum_i a[i] * b[i] with one rescale (ckks_inner_prod); b is a list of
    ciphertexts (needs evk) or of real weights."""
    n = len(a)
    pa = (ctypes.c_void_p * n)(*[x.handle.value for x in a])
    if b and isinstance(b[0], Ciphertext):
        pb = (ctypes.c_void_p * n)(*[x.handle.value for x in b])
        capi.check(capi.load().aoa_inner_prod(ctx.handle, out.handle, pa, pb, n, evk.handle))
    else:
        w = np.ascontiguousarray(b, dtype=np.float64)
        capi.check(capi.load().aoa_inner_prod_const(ctx.handle, out.handle, pa,
                                                    w.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), n))


# ---- CUDA graphs ------------------------------------------------------------------

class Graph:
    """A captured sequence of a context's asynchronous work, replayed with one launch."""

    def __init__(self, ctx, handle):
        self.ctx, self.handle = ctx, handle

    @classmethod
    def capture(cls, ctx, fn):
        """Run fn() under stream capture on ctx and instantiate the result."""
        lib = capi.load()
        capi.check(lib.aoa_ctx_capture_begin(ctx.handle))
        try:
            fn()
        finally:
            h = ctypes.c_void_p()
            st = lib.aoa_ctx_capture_end(ctx.handle, ctypes.byref(h))
        capi.check(st)
        return cls(ctx, h)

    @property
    def nodes(self):
        n = ctypes.c_long()
        capi.check(capi.load().aoa_graph_nodes(self.handle, ctypes.byref(n)))
        return n.value

    def launch(self):
        capi.check(capi.load().aoa_graph_launch(self.ctx.handle, self.handle))

    def close(self):
        if getattr(self, "handle", None):
            capi.load().aoa_graph_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
