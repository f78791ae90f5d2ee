"""Pins of the oracle's number theory against exact arithmetic and the
reference's prime tables (CPU only)."""
import numpy as np
import oracle


def test_smallest_primitive_root_matches_reference_table(ref_table):
    L = oracle.lib()
    for q, g in ref_table["proots"].items():
        assert L.oc_smallest_primitive_root(int(q)) == g, q


def test_reference_buckets_are_ntt_primes(ref_table):
    L = oracle.lib()
    for bits, vals in ref_table["buckets"].items():
        assert vals == sorted(vals, reverse=True)
        for q in vals:
            assert L.oc_is_prime(q)
            assert q.bit_length() == int(bits)


def test_reference_barrett_is_exact_on_canonical_products(ref_table):
    """The reference's mod() (common.cu:257-291) returns the canonical residue for
    products of canonical operands on every table prime (its TestPrimitives.mulmod
    checks the same against NTL, tests.cpp:368-396)."""
    L = oracle.lib()
    for vals in ref_table["buckets"].values():
        for q in vals[:16]:
            assert L.oc_ref_mulmod_mismatches(q, 200000, q & 0xFFFF) == 0, q


def test_reference_barrett_spot_values(ref_table):
    L = oracle.lib()
    rng = np.random.default_rng(7)
    for q in ref_table["buckets"]["55"][:4] + ref_table["buckets"]["63"][:1]:
        for _ in range(200):
            a, b = int(rng.integers(0, q)), int(rng.integers(0, q))
            assert L.oc_ref_mulmod(a, b, q) == a * b % q
        # 128-bit inputs below 2^(2*bits) as in TestPrimitives.mod
        for _ in range(100):
            x = int(rng.integers(0, q)) * int(rng.integers(0, q))
            assert L.oc_ref_mod128(x >> 64, x & (2**64 - 1), q) == x % q


def test_powmod_invmod_exact():
    L = oracle.lib()
    q = 1152921504606584833  # 60-bit prime, q = 1 mod 2^17
    assert L.oc_is_prime(q)
    for a in (2, 3, 12345678901234567, q - 1):
        assert L.oc_powmod(a, q - 2, q) == pow(a, q - 2, q)
        assert L.oc_invmod(a, q) * a % q == 1


def test_prime_search_rule():
    ps = oracle.gen_ntt_primes(60, 1 << 17, 61)
    assert len(ps) == 61
    assert ps == sorted(ps, reverse=True)
    L = oracle.lib()
    for q in ps:
        assert q.bit_length() == 60 and q % (1 << 17) == 1 and L.oc_is_prime(q)
    # exhaustive: no prime of the form was skipped between consecutive picks
    for hi, lo in zip(ps[:5], ps[1:6]):
        for c in range(lo + (1 << 17), hi, 1 << 17):
            assert not L.oc_is_prime(c)


def test_prime_search_rule_one_mod_2_32():
    """The benchmark's prime set: the 61 largest 60-bit primes q = 1 mod 2^32,
    the same from the library's search and the oracle's, none skipped."""
    from aoa_b200 import params
    ps = oracle.gen_ntt_primes(60, 1 << 32, 61)
    assert ps == params.ntt_primes(60, 1 << 32, 61)
    assert len(ps) == 61 and ps == sorted(ps, reverse=True)
    L = oracle.lib()
    for q in ps:
        assert q.bit_length() == 60 and q % (1 << 32) == 1 and L.oc_is_prime(q)
    for hi, lo in zip(ps[:5], ps[1:6]):
        for c in range(lo + (1 << 32), hi, 1 << 32):
            assert not L.oc_is_prime(c)
