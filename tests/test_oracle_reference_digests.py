"""The oracle at the headline shape against the reference itself.

tests/golden/reference_digests.json holds digests of what pdroalves/aoa's
aoa-ntt and aoa-dgt computed on a B200 at N = 2^16 with 30 Q and 31 special
primes (their own 55-bit prime set, 63-bit q0; oracle/ref/ref_ckks_harness.cu
and ref_dgt_ckks_harness.cu --digest):
ckks_mul (HMult, relinearise, rescale; src/ckks/ckks.cpp:273-347) and
ckks_rotate_left by one slot (ckks.cpp:982-1009) of the seeded operands and
keys of the CKKS records (tests/test_oracle_reference_ckks.py) at level 29.
Each output limb is reduced to sum_j c_j (2j + 1) G mod 2^64 (G =
0x9E3779B97F4A7C15), a digest that any change of a residue changes; the
oracle's outputs must give the same digests and scales."""
import json
import os

import numpy as np
import pytest

from oracle import Oracle
from tests.test_oracle_reference_ckks import SCALE_A, SCALE_B, seeded_ct, seeded_key

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "reference_digests.json")
G = np.uint64(0x9E3779B97F4A7C15)


def load(variant="aoa-ntt"):
    with open(GOLDEN) as f:
        return [d for d in json.load(f) if d["variant"] == variant][0]


def digests(c0, c1, n):
    """Digest of limbs 0..n-1 of c0, then of c1."""
    N = c0.shape[1]
    with np.errstate(over="ignore"):
        w = (2 * np.arange(N, dtype=np.uint64) + np.uint64(1)) * G
        return [int(np.sum(x[i] * w, dtype=np.uint64)) for x in (c0, c1) for i in range(n)]


def test_both_reference_variants_agree():
    """aoa-ntt and aoa-dgt give the same residues at the headline shape (the
    transform only changes the domain of exact products)."""
    a, b = load("aoa-ntt"), load("aoa-dgt")
    assert a["primes"] == b["primes"]
    assert a["hmult"] == b["hmult"] and a["rotate1"] == b["rotate1"]


def test_fixture_is_the_headline_shape():
    d = load()
    assert (d["N"], d["k"], d["kl"]) == (1 << 16, 30, 31) and len(d["primes"]) == 61
    assert d["primes"][0] >= 1 << 62 and all(p < 1 << 56 for p in d["primes"][1:])
    assert len(d["hmult"]["digests"]) == 2 * 29 and len(d["rotate1"]["digests"]) == 2 * 30


@pytest.fixture(scope="module")
def full():
    d = load()
    N, k = d["N"], d["k"]
    primes = d["primes"]
    return d, N, k, primes, Oracle(N, primes[:k], primes[k:])


def test_oracle_hmult_digests_equal_reference(full):
    d, N, k, primes, o = full
    a = seeded_ct(101, 102, primes[:k], N)
    b = seeded_ct(103, 104, primes[:k], N)
    evk = tuple(o.ntt_fwd(x) for x in seeded_key(111, 112, primes, N))
    o0, o1, scale = o.hmult(a, b, evk, k - 1, SCALE_A, SCALE_B, rescale=True)
    assert d["hmult"]["level"] == k - 2 and scale == d["hmult"]["scale"]
    assert digests(o0, o1, k - 1) == d["hmult"]["digests"]


def test_oracle_rotation_digests_equal_reference(full):
    d, N, k, primes, o = full
    c = seeded_ct(105, 106, primes[:k], N)
    rtk = tuple(o.ntt_fwd(x) for x in seeded_key(123, 124, primes, N))
    o0, o1 = o.rotate_left(c, 1, rtk, k - 1)
    assert d["rotate1"]["level"] == k - 1 and d["rotate1"]["scale"] == SCALE_A
    assert digests(o0, o1, k) == d["rotate1"]["digests"]
