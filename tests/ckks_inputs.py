"""Seeded synthetic CKKS inputs shared by the oracle and GPU parity tests.

Distributions follow the reference sampler (aoa-ntt src/cuda/sampler.cu):
ternary secret of Hamming weight 64 (sample_hw, HAMMINGWEIGHT 64), ternary u
with N/2 non-zeros (sample_Z0), rounded Gaussian noise sigma = 3.2 (sample_DG),
uniform residues (sample_uniform).  numpy PCG64 streams replace cuRAND; the
values enter every implementation as explicit inputs.
"""
import numpy as np

from oracle import ST_COEF, ST_NTT

SIGMA = 3.2
HW = 64


def ternary_hw(rng, n, hw=HW):
    c = np.zeros(n, dtype=np.int64)
    pos = rng.choice(n, size=min(hw, n), replace=False)
    c[pos] = rng.choice([-1, 1], size=len(pos))
    return c


def gaussian(rng, n, sigma=SIGMA):
    return np.rint(rng.normal(0.0, sigma, n)).astype(np.int64)


def uniform_residues(rng, primes, n):
    return np.array([rng.integers(0, q, n, dtype=np.uint64) for q in primes], dtype=np.uint64)


def signed_to_residues(coeffs, primes):
    """Small signed integers -> [len(primes)][N] canonical residues."""
    c = np.asarray(coeffs, dtype=np.int64)
    base = c.astype(np.uint64)          # negatives wrap to 2^64 + c
    neg = c < 0
    out = np.empty((len(primes), c.size), dtype=np.uint64)
    for r, q in enumerate(primes):
        row = base.copy()
        row[neg] += np.uint64(q)        # 2^64 + c + q wraps to q + c
        out[r] = row
    return out


def make_keys(o, seed=2, rotations=(), conjugation=False, hw=HW):
    """Secret, public, relinearisation, rotation and conjugation keys from one seed."""
    rng = np.random.default_rng(seed)
    N, primes = o.N, o.primes
    s_coef = ternary_hw(rng, N, hw)
    s = signed_to_residues(s_coef, primes)
    keys = {"s_coef": s_coef, "s": s}
    zero = np.zeros_like(s)
    a = uniform_residues(rng, primes, N)
    e = gaussian(rng, N)
    pb, pa = o.swk_gen(zero, s, a, e, a_state=ST_COEF)
    keys["pk"] = (pb[: o.k], pa[: o.k])
    keys["pk_raw"] = (a, e)
    s2 = o.square_secret(s)
    a = uniform_residues(rng, primes, N)
    e = gaussian(rng, N)
    keys["evk"] = o.swk_gen(s2, s, a, e, a_state=ST_COEF)
    keys["evk_raw"] = (s2, a, e)
    keys["rtk"] = {}
    keys["rtk_raw"] = {}
    for r in rotations:
        sr = o.rotate_secret(s, r)
        a = uniform_residues(rng, primes, N)
        e = gaussian(rng, N)
        keys["rtk"][r] = o.swk_gen(sr, s, a, e, a_state=ST_COEF)
        keys["rtk_raw"][r] = (sr, a, e)
    if conjugation:
        sc = o.conjugate_secret(s)
        a = uniform_residues(rng, primes, N)
        e = gaussian(rng, N)
        keys["cjk"] = o.swk_gen(sc, s, a, e, a_state=ST_COEF)
        keys["cjk_raw"] = (sc, a, e)
    return keys


def encryption_noise(o, seed):
    rng = np.random.default_rng(seed)
    N = o.N
    u = np.zeros(N, dtype=np.int64)
    pos = rng.choice(N, size=N // 2, replace=False)
    u[pos] = rng.choice([-1, 1], size=len(pos))
    return u, gaussian(rng, N), gaussian(rng, N)


def encrypt_values(o, keys, values, scale, seed=3):
    m = o.encode(values, scale)
    u, e1, e2 = encryption_noise(o, seed)
    ur = signed_to_residues(u, o.primes[: o.k])
    return o.encrypt(m, ur, e1, e2, keys["pk"], pk_state=ST_NTT)


def decrypt_values(o, keys, c, slots, scale, state=ST_NTT):
    m = o.decrypt(c, keys["s"][: o.k], state=state)
    return o.decode(m[0], slots, scale)
