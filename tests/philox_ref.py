"""Host restatement of Philox4x32-10 (Salmon, Moraes, Dror, Shaw, SC 2011) and
of the device samplers' output rules: the tests compare
aoa_sample_uniform / aoa_sample_gaussian / aoa_sample_ternary against it."""
import numpy as np

M0, M1 = np.uint64(0xD2511F53), np.uint64(0xCD9E8D57)
W0, W1 = 0x9E3779B9, 0xBB67AE85
MASK = np.uint64(0xFFFFFFFF)


def philox(index, stream, seed):
    """Vectorised over `index` (uint64 array): four uint64 arrays of 32-bit words."""
    idx = np.asarray(index, dtype=np.uint64)
    c0 = idx & MASK
    c1 = idx >> np.uint64(32)
    c2 = np.full_like(idx, stream & 0xFFFFFFFF)
    c3 = np.full_like(idx, (stream >> 32) & 0xFFFFFFFF)
    k0, k1 = seed & 0xFFFFFFFF, (seed >> 32) & 0xFFFFFFFF
    for _ in range(10):
        p0 = M0 * c0
        p1 = M1 * c2
        hi0, lo0 = p0 >> np.uint64(32), p0 & MASK
        hi1, lo1 = p1 >> np.uint64(32), p1 & MASK
        c0, c1, c2, c3 = hi1 ^ c1 ^ np.uint64(k0), lo1, hi0 ^ c3 ^ np.uint64(k1), lo0
        k0 = (k0 + W0) & 0xFFFFFFFF
        k1 = (k1 + W1) & 0xFFFFFFFF
    return c0, c1, c2, c3


def uniform(primes, n, seed, stream):
    out = np.zeros((len(primes), n), dtype=np.uint64)
    for l, q in enumerate(primes):
        x0, x1, x2, x3 = philox(np.arange(l * n, (l + 1) * n, dtype=np.uint64), stream, seed)
        for i in range(n):
            v = (int(x3[i]) << 96) | (int(x2[i]) << 64) | (int(x1[i]) << 32) | int(x0[i])
            out[l, i] = v % q
    return out


def gaussian(n, seed, stream, sigma=3.2):
    x0, x1, x2, x3 = philox(np.arange(n, dtype=np.uint64), stream, seed)
    a = (x1 << np.uint64(32)) | x0
    b = (x3 << np.uint64(32)) | x2
    u1 = ((a >> np.uint64(11)).astype(np.float64) + 1.0) * 2.0 ** -53
    u2 = (b >> np.uint64(11)).astype(np.float64) * 2.0 ** -53
    z = np.sqrt(-2.0 * np.log(u1)) * np.cos(2.0 * np.pi * u2)
    return np.rint(z * sigma).astype(np.int64)


def ternary(n, hw, seed, stream):
    x0, x1, _, _ = philox(np.arange(n, dtype=np.uint64), stream, seed)
    keys = (x0 << np.uint64(32)) | np.arange(n, dtype=np.uint64)
    out = np.zeros(n, dtype=np.int64)
    pos = np.argsort(keys, kind="stable")[:hw]
    out[pos] = np.where((x1[pos] & np.uint64(1)) == 1, -1, 1)
    return out
