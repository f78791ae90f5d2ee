"""Pins of the oracle's transform (CPU only).

The reference's only exact pin of NTT-based arithmetic is the negacyclic
product against NTL (TestNTTArithmetic.Mul/MulAdd/MulInt, aoa-ntt
tests/tests.cpp:564-694); its Transform test is vacuous.  Here the restated
hierarchical transform is pinned to the closed form a(psi^(2*bitrev(p)+1)) and
its products to the schoolbook product from tests/pymodel.py.
"""
import numpy as np
import pytest

import oracle
from oracle import Oracle, reference_prime_set
from tests import pymodel


def _rand_poly(rng, primes, n):
    return np.array([rng.integers(0, q, n, dtype=np.uint64) for q in primes], dtype=np.uint64)


@pytest.mark.parametrize("N", [8, 64, 128, 512, 2048])
def test_ntt_closed_form(ref_table, rng, N):
    Q, B = reference_prime_set(ref_table, 2, 1, 55)
    o = Oracle(N, Q, B)
    x = _rand_poly(rng, Q + B, N)
    X = o.ntt_fwd(x)
    for r, q in enumerate(Q + B):
        want = pymodel.ntt_closed_form([int(v) for v in x[r]], q, o.psi(r)) if N <= 512 else None
        if want is not None:
            assert [int(v) for v in X[r]] == want
        else:  # spot positions at larger N
            lg = N.bit_length() - 1
            for p in (0, 1, N // 2 + 3, N - 1):
                ev = pow(o.psi(r), 2 * pymodel.bitrev(p, lg) + 1, q)
                acc = sum(int(c) * pow(ev, i, q) for i, c in enumerate(x[r])) % q
                assert acc == int(X[r, p])
    assert np.array_equal(o.ntt_inv(X), x)


@pytest.mark.parametrize("prec", [55, 48, 45])
def test_ntt_product_is_negacyclic(ref_table, rng, prec):
    N = 256
    Q, B = reference_prime_set(ref_table, 3, 2, prec)
    o = Oracle(N, Q, B)
    a, b, c = (_rand_poly(rng, Q, N) for _ in range(3))
    A, Bt, Cc = o.ntt_fwd(a), o.ntt_fwd(b), o.ntt_fwd(c)
    for r, q in enumerate(Q):
        prod = o.ntt_inv(np.array([(int(x) * int(y)) % q for x, y in zip(A[r], Bt[r])], dtype=np.uint64),
                         first=r)
        want = pymodel.negacyclic_mul([int(v) for v in a[r]], [int(v) for v in b[r]], q)
        assert [int(v) for v in prod] == want
        # MulAdd: a*b + c
        s = o.ntt_inv(np.array([(int(x) * int(y) + int(z)) % q for x, y, z in zip(A[r], Bt[r], Cc[r])],
                               dtype=np.uint64), first=r)
        assert [int(v) for v in s] == [(w + int(cc)) % q for w, cc in zip(want, c[r])]


def test_ntt_roundtrip_large(rng):
    qs = oracle.gen_ntt_primes(60, 1 << 17, 3)
    o = Oracle(1 << 16, qs[:2], qs[2:])
    x = _rand_poly(rng, qs, 1 << 16)
    X = o.ntt_fwd(x)
    assert np.array_equal(o.ntt_inv(X), x)
    lg = 16
    for p in (0, 12345):
        ev = pow(o.psi(0), 2 * pymodel.bitrev(p, lg) + 1, qs[0])
        acc = 0
        pw = 1
        for v in x[0]:
            acc = (acc + int(v) * pw) % qs[0]
            pw = pw * ev % qs[0]
        assert acc == int(X[0, p])


def test_golden_ntt_vectors(ref_table):
    """Committed N=2^10 vectors (tests/golden/make_golden.py, Python model)."""
    g = np.load(__import__("os").path.join(__import__("os").path.dirname(__file__), "golden", "ntt_n1024.npz"))
    Q = [int(v) for v in g["primes"]]
    o = Oracle(1024, Q[:-1], Q[-1:])
    assert np.array_equal(o.ntt_fwd(g["x"]), g["X"])
