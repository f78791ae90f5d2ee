"""GPU transform parity against the oracle (bit-exact), through the C ABI."""
import os

import numpy as np
import pytest

import oracle
from oracle import Oracle, reference_prime_set
from tests.gpu_util import require_gpu

pytestmark = pytest.mark.gpu


def _engine_and_oracle(log_n, q, b):
    import aoa_b200
    E = aoa_b200.Engine(log_n, q, b)
    return E, aoa_b200.Context(E), Oracle(1 << log_n, q, b)


def _rand(rng, primes, n, npolys=1):
    return np.array([[rng.integers(0, p, n, dtype=np.uint64) for p in primes] for _ in range(npolys)],
                    dtype=np.uint64)


@pytest.mark.parametrize("log_n", [10, 11, 12, 13, 14, 15, 16, 17])
def test_ntt_reference_primes(ref_table, log_n):
    require_gpu()
    Q, B = reference_prime_set(ref_table, 3, 2, 55)
    if log_n == 17:   # 2N = 2^18 must divide q - 1: keep the table primes that allow it
        ok = [q for q in [ref_table["buckets"]["63"][0]] + ref_table["buckets"]["55"] if (q - 1) % (1 << 18) == 0]
        Q, B = ok[:3], ok[3:5]
    E, ctx, o = _engine_and_oracle(log_n, Q, B)
    rng = np.random.default_rng(log_n)
    x = _rand(rng, Q + B, 1 << log_n, npolys=2)
    d = ctx.upload(x)
    ctx.ntt_fwd(d, 2, 0, len(Q + B))
    X = d.numpy()
    for p in range(2):
        assert np.array_equal(X[p], o.ntt_fwd(x[p])), "forward mismatch"
    ctx.ntt_inv(d, 2, 0, len(Q + B))
    assert np.array_equal(d.numpy(), x), "inverse(forward(x)) != x"
    y = _rand(rng, Q + B, 1 << log_n)
    dy = ctx.upload(y)
    ctx.ntt_inv(dy, 1, 0, len(Q + B))
    assert np.array_equal(dy.numpy()[0], o.ntt_inv(y[0]))


@pytest.mark.parametrize("log_n", [12, 16])
def test_ntt_60bit_primes_strided(log_n):
    require_gpu()
    ps = oracle.gen_ntt_primes(60, 1 << 17, 6)
    E, ctx, o = _engine_and_oracle(log_n, ps[:4], ps[4:])
    rng = np.random.default_rng(5)
    n = 1 << log_n
    # 3 polys of stride 6 limbs; transform limbs 0..2 with primes 2..4
    x = np.array([[rng.integers(0, ps[min(l + 2, 5)], n, dtype=np.uint64) for l in range(6)] for _ in range(3)])
    d = ctx.upload(x)
    ctx.ntt_fwd(d, 3, 2, 3, poly_stride=6)
    X = d.numpy()
    for p in range(3):
        assert np.array_equal(X[p, :3], o.ntt_fwd(x[p, :3], first=2))
        assert np.array_equal(X[p, 3:], x[p, 3:])          # untouched limbs
    ctx.ntt_inv(d, 3, 2, 3, poly_stride=6)
    assert np.array_equal(d.numpy(), x)


def test_ntt_golden_vectors():
    require_gpu()
    import aoa_b200
    g = np.load(os.path.join(os.path.dirname(__file__), "golden", "ntt_n1024.npz"))
    primes = [int(v) for v in g["primes"]]
    E = aoa_b200.Engine(10, primes[:-1], primes[-1:])
    ctx = aoa_b200.Context(E)
    d = ctx.upload(g["x"])
    ctx.ntt_fwd(d, 1, 0, len(primes))
    assert np.array_equal(d.numpy(), g["X"])


def test_ntt_edge_values(ref_table):
    """All-zero, all (q-1) and single-impulse limbs."""
    require_gpu()
    Q, B = reference_prime_set(ref_table, 2, 1, 55)
    E, ctx, o = _engine_and_oracle(13, Q, B)
    n = 1 << 13
    x = np.zeros((3, n), dtype=np.uint64)
    x[1] = np.uint64(Q[1] - 1)
    x[2, 17] = 1
    d = ctx.upload(x)
    ctx.ntt_fwd(d, 1, 0, 3)
    assert np.array_equal(d.numpy(), o.ntt_fwd(x))
