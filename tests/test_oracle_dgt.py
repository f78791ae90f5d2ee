"""Pins of the oracle's DGT restatement (aoa-dgt src/cuda/dgt.cu).

* the fixture roots are roots of i of the right order (what the reference's
  compute_nthroot asserts);
* the restated transform, non-hierarchical (N <= 512) and hierarchical
  (N >= 1024), equals an independent closed form: position bitrev(k) holds
  sum_n x_n r^n w^(n k), w = g^((p-1)/N);
* inverse(forward(x)) = x, and the DGT product of two folded polynomials is
  their negacyclic product (the reference's TestDGT.Transform and
  TestArithmetic.Mul, aoa-dgt tests/unit_tests/test_arithmetic.cu:359-389,
  563-603);
* GIMul is the Gaussian-integer product (TestDGT.GIMul, test_arithmetic.cu:444-478).
"""
import json
import os

import numpy as np
import pytest

import oracle
from oracle import DgtOracle, dgt_prime_set, dgt_roots, fold, unfold

HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.fixture(scope="module")
def dgt_table():
    with open(os.path.join(HERE, "golden", "dgt_roots.json")) as f:
        return json.load(f)


def _gimul(x, y, p):
    return ((x[0] * y[0] - x[1] * y[1]) % p, (x[0] * y[1] + x[1] * y[0]) % p)


def _gipow(x, e, p):
    r = (1, 0)
    while e:
        if e & 1:
            r = _gimul(r, x, p)
        x = _gimul(x, x, p)
        e >>= 1
    return r


def _brv(x, bits):
    return int(format(x, "0%db" % bits)[::-1], 2) if bits else 0


def _dft(v, w, p):
    """Cyclic DFT X_k = sum v_n w^(n k) (recursive radix 2, Python ints)."""
    n = len(v)
    if n == 1:
        return list(v)
    ev, od = _dft(v[0::2], w * w % p, p), _dft(v[1::2], w * w % p, p)
    out = [0] * n
    t = 1
    for k in range(n // 2):
        a, b = ev[k], od[k] * t % p
        out[k], out[k + n // 2] = (a + b) % p, (a - b) % p
        t = t * w % p
    return out


def _rand_gi(rng, primes, N):
    return np.stack([np.stack([rng.integers(0, q, N, dtype=np.uint64), rng.integers(0, q, N, dtype=np.uint64)],
                              axis=-1) for q in primes])


def test_fixture_roots_are_roots_of_i(dgt_table):
    for q, rs in list(dgt_table["nthroot"].items())[::10]:
        for n, r in rs.items():
            assert _gipow(tuple(r), int(n), int(q)) == (0, 1)


@pytest.mark.parametrize("N", [16, 64, 512, 1024, 2048])
def test_dgt_matches_closed_form(dgt_table, N):
    Q, B = dgt_prime_set(dgt_table, 2, 1, 55)
    primes = Q + B
    g, r = dgt_roots(dgt_table, primes, N)
    D = DgtOracle(N, primes, g, r)
    rng = np.random.default_rng(N)
    x = _rand_gi(rng, primes, N)
    y = D.fwd(x)
    bits = N.bit_length() - 1
    for rid, p in enumerate(primes):
        w = pow(g[rid], (p - 1) // N, p)
        tw = [(int(a), int(b)) for a, b in x[rid]]
        rn = (1, 0)
        for n in range(N):
            tw[n] = _gimul(tw[n], rn, p)
            rn = _gimul(rn, r[rid], p)
        re = _dft([t[0] for t in tw], w, p)
        im = _dft([t[1] for t in tw], w, p)
        want = np.zeros((N, 2), dtype=np.uint64)
        for k in range(N):
            want[_brv(k, bits)] = (re[k], im[k])
        assert np.array_equal(y[rid], want), "N=%d rid=%d" % (N, rid)


@pytest.mark.parametrize("N,prec", [(16, 45), (64, 48), (1024, 52), (4096, 55)])
def test_dgt_product_is_negacyclic(dgt_table, N, prec):
    Q, B = dgt_prime_set(dgt_table, 3, 2, prec)
    primes = Q + B
    g, r = dgt_roots(dgt_table, primes, N)
    D = DgtOracle(N, primes, g, r)
    rng = np.random.default_rng(N + prec)
    n = 2 * N
    a = np.array([rng.integers(0, q, n, dtype=np.uint64) for q in primes])
    b = np.array([rng.integers(0, q, n, dtype=np.uint64) for q in primes])
    A, Bf = D.fwd(fold(a)), D.fwd(fold(b))
    assert np.array_equal(D.inv(A), fold(a))
    c = unfold(D.inv(D.gi_mul(A, Bf)))
    o = oracle.Oracle(n, Q, B, proots=g)      # the pinned NTT oracle gives the negacyclic product
    fa, fb = o.ntt_fwd(a), o.ntt_fwd(b)
    prod = np.array([[int(u) * int(v) % q for u, v in zip(fa[i], fb[i])] for i, q in enumerate(primes)],
                    dtype=np.uint64)
    assert np.array_equal(c, o.ntt_inv(prod))


def test_gi_mul_is_gaussian_product(dgt_table):
    Q, B = dgt_prime_set(dgt_table, 2, 2, 55)
    primes = Q + B
    g, r = dgt_roots(dgt_table, primes, 16)
    D = DgtOracle(16, primes, g, r)
    rng = np.random.default_rng(5)
    a, b = _rand_gi(rng, primes, 16), _rand_gi(rng, primes, 16)
    c = D.gi_mul(a, b)
    for rid, p in enumerate(primes):
        for t in range(16):
            x = (int(a[rid, t, 0]), int(a[rid, t, 1]))
            y = (int(b[rid, t, 0]), int(b[rid, t, 1]))
            assert tuple(int(v) for v in c[rid, t]) == _gimul(x, y, p)


def test_dgt_twist_tables(dgt_table):
    Q, B = dgt_prime_set(dgt_table, 2, 1, 55)
    primes = Q + B
    for N in (16, 1024):
        g, r = dgt_roots(dgt_table, primes, N)
        D = DgtOracle(N, primes, g, r)
        for rid, p in enumerate(primes):
            nth, inv = D.twist(rid)
            assert tuple(int(v) for v in nth[1]) == r[rid]
            scale = 1 if N >= 1024 else pow(N, -1, p)
            for t in (0, 1, 7, N - 1):
                prod = _gimul(tuple(int(v) for v in nth[t]), tuple(int(v) for v in inv[t]), p)
                assert prod == (scale % p, 0)
