"""Pins of the oracle's RNS conversions and CKKS operations (CPU only)."""
import os

import numpy as np
import pytest

from oracle import Oracle, reference_prime_set, ST_COEF, ST_NTT
import oracle
from tests import pymodel
from tests.ckks_inputs import make_keys, encrypt_values, decrypt_values


def test_golden_rns_vectors():
    g = np.load(os.path.join(os.path.dirname(__file__), "golden", "rns_n64.npz"))
    Q, B = [int(v) for v in g["q"]], [int(v) for v in g["b"]]
    lvl = int(g["level"])
    o = Oracle(64, Q, B)
    assert np.array_equal(o.modup(g["xq"], lvl), g["modup"])
    qb = np.concatenate([g["xq"], g["xb"]])
    assert np.array_equal(o.moddown(qb, lvl)[: lvl + 1], g["moddown"])
    r0, _ = o.rescale(g["xq"], g["xq"], lvl)
    assert np.array_equal(r0[:lvl], g["rescale"])


@pytest.mark.parametrize("level", [0, 2, 4])
def test_rns_against_model_60bit(rng, level):
    qs = oracle.gen_ntt_primes(60, 1 << 7, 9)
    Q, B = qs[:5], qs[5:]
    N = 32
    o = Oracle(N, Q, B)
    xq = np.array([rng.integers(0, q, N, dtype=np.uint64) for q in Q])
    xb = np.array([rng.integers(0, b, N, dtype=np.uint64) for b in B])
    lq = [[int(v) for v in r] for r in xq]
    lb = [[int(v) for v in r] for r in xb]
    assert [[int(v) for v in r] for r in o.modup(xq, level)] == pymodel.modup(lq, Q, B, level)
    got = o.moddown(np.concatenate([xq, xb]), level)[: level + 1]
    assert [[int(v) for v in r] for r in got] == pymodel.moddown(lq, lb, Q, B, level)
    if level > 0:
        r0, _ = o.rescale(xq, xq, level)
        assert [[int(v) for v in r] for r in r0[:level]] == pymodel.rescale(lq, Q, level)


def test_automorphism_against_model(ref_table, rng):
    Q, B = reference_prime_set(ref_table, 2, 1, 55)
    N = 64
    o = Oracle(N, Q, B)
    x = np.array([rng.integers(0, q, N, dtype=np.uint64) for q in Q])
    for power in (5, 25, 2 * N - 1):
        got = o.automorph(x, power, len(Q))
        for r, q in enumerate(Q):
            assert [int(v) for v in got[r]] == pymodel.automorph([int(v) for v in x[r]], power, q)


def _params(ref_table, N, k, kl, prec):
    Q, B = reference_prime_set(ref_table, k, kl, prec)
    return Oracle(N, Q, B)


def test_encode_decode_roundtrip(ref_table, rng):
    o = _params(ref_table, 1024, 3, 3, 55)
    slots = 512
    v = rng.uniform(-1, 1, slots) + 1j * rng.uniform(-1, 1, slots)
    m = o.encode(v, 1 << 55)
    back = o.decode(m[0], slots, 1 << 55)
    assert np.max(np.abs(back - v)) < 1e-9


@pytest.mark.parametrize("N,k,kl,prec", [(1024, 3, 3, 55), (2048, 4, 4, 48)])
def test_hmult_rescale_decrypts(ref_table, N, k, kl, prec):
    o = _params(ref_table, N, k, kl, prec)
    keys = make_keys(o, seed=5)
    rng = np.random.default_rng(9)
    slots = N // 2
    scale = 1 << prec
    v1 = rng.uniform(-2, 2, slots) + 1j * rng.uniform(-2, 2, slots)
    v2 = rng.uniform(-2, 2, slots) + 1j * rng.uniform(-2, 2, slots)
    c1 = encrypt_values(o, keys, v1, scale, seed=11)
    c2 = encrypt_values(o, keys, v2, scale, seed=12)
    level = k - 1
    o0, o1, sc = o.hmult(c1, c2, keys["evk"], level, scale, scale, rescale=True, a_state=ST_NTT, b_state=ST_NTT)
    assert sc == (scale * scale) // o.primes[level]
    got = decrypt_values(o, keys, (o0, o1), slots, sc, state=ST_COEF)
    assert np.max(np.abs(got - v1 * v2)) < 0.005          # ERRBOUND, tests.cpp:34


def test_rotate_and_conjugate_decrypt(ref_table):
    o = _params(ref_table, 1024, 3, 3, 55)
    keys = make_keys(o, seed=6, rotations=(1, 4), conjugation=True)
    rng = np.random.default_rng(3)
    slots = 512
    scale = 1 << 55
    v = rng.uniform(-1, 1, slots) + 1j * rng.uniform(-1, 1, slots)
    c = encrypt_values(o, keys, v, scale, seed=13)
    for r in (1, 4):
        r0, r1 = o.rotate_left(c, r, keys["rtk"][r], o.k - 1, state=ST_NTT)
        got = decrypt_values(o, keys, (r0, r1), slots, scale, state=ST_COEF)
        assert np.max(np.abs(got - np.roll(v, -r))) < 0.01     # rotation bound, tests.cpp:1570-1579
    j0, j1 = o.conjugate(c, keys["cjk"], o.k - 1, state=ST_NTT)
    got = decrypt_values(o, keys, (j0, j1), slots, scale, state=ST_COEF)
    assert np.max(np.abs(got - np.conj(v))) < 0.01
