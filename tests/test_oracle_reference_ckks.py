"""The oracle's CKKS layer against outputs of the reference evaluators themselves.

tests/golden/reference_ckks_outputs.npz holds what pdroalves/aoa's aoa-ntt
CKKS layer computed on a B200 through its API (oracle/ref/ref_ckks_harness.cu,
built from the reference's sources by oracle/ref/Makefile; fixture written by
tests/golden/make_reference_outputs.py), and
tests/golden/reference_dgt_ckks_outputs.npz the same records from aoa-dgt's
CKKS layer (oracle/ref/ref_dgt_ckks_harness.cu; src/ckks.cpp, src/keys.cpp,
src/ckkscontext.cpp, src/tool/encoder.cu of aoa-dgt):
- on seeded operands: ckks_mul and ckks_mul_without_rescale (src/ckks/ckks.cpp:
  273-347), ckks_rotate_left (ckks.cpp:982-1009), ckks_conjugate
  (ckks.cpp:1011-1040), ckks_add / ckks_sub (ckks.cpp:240-271) at two levels,
  and CKKSContext::encode (src/ckks/ckkscontext.cpp:5-19, encoder.cu:139-216);
- with the reference's own keys (ckks_new_sk, ckks_keygen; cuRAND draws):
  ckks_encrypt of two value vectors, their ckks_mul, a left rotation by one
  slot, and ckks_decrypt of each.
Seeded operands are regenerated here from the seeds the harness documents;
every residue the oracle computes must equal the reference's, and its decoded
values the reference's decryptions."""
import json
import os

import numpy as np
import pytest

from oracle import ST_COEF, Oracle, dgt_roots
from tests.test_oracle_reference_outputs import splitmix_residues

HERE = os.path.dirname(os.path.abspath(__file__))
FIXTURES = ("reference_ckks_outputs.npz", "reference_dgt_ckks_outputs.npz")   # aoa-ntt, aoa-dgt
SCALE_A, SCALE_B = (1 << 40) + 3, (1 << 40) + 5
LEVELS = (3, 1)          # input levels of the seeded cases (k = 4)
ROTATIONS = (1, 4)


def load(name=FIXTURES[0]):
    path = os.path.join(HERE, "golden", name)
    assert os.path.exists(path), "missing fixture " + path
    g = np.load(path)
    N, k, kl, prec = (int(v) for v in g["n1024_params"])
    primes = [int(p) for p in g["n1024_primes"]]
    return g, N, k, kl, prec, primes


def dgt_generators(primes, N):
    """aoa-dgt's generators for `primes` (tests/golden/dgt_roots.json)."""
    with open(os.path.join(HERE, "golden", "dgt_roots.json")) as f:
        return dgt_roots(json.load(f), primes, N // 2)[0]


def splitmix_values(seed, slots):
    """Complex values of the harness: re, im = 2 u - 1, u the top 53 bits of
    consecutive splitmix64 outputs times 2^-53 (re first)."""
    w = _splitmix_words(seed, 2 * slots)
    u = (w >> np.uint64(11)).astype(np.float64) * 2.0 ** -53
    u = 2.0 * u - 1.0
    return u[0::2] + 1j * u[1::2]


def _splitmix_words(seed, n):
    with np.errstate(over="ignore"):
        idx = np.arange(1, n + 1, dtype=np.uint64)
        z = np.uint64(seed) + idx * np.uint64(0x9E3779B97F4A7C15)
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        return z ^ (z >> np.uint64(31))


def ct_record(words, N):
    """[aux, scale, slots, c0 limbs, c1 limbs] -> (aux, scale, slots, c0, c1)."""
    aux, scale, slots = (int(v) for v in words[:3])
    body = words[3:]
    n = body.size // (2 * N)
    c0 = body[: n * N].reshape(n, N)
    c1 = body[n * N:].reshape(n, N)
    return aux, scale, slots, c0, c1


def seeded_ct(seed0, seed1, q_primes, N):
    return splitmix_residues(seed0, q_primes, N), splitmix_residues(seed1, q_primes, N)


def seeded_key(seed_b, seed_a, primes, N):
    """A switching key of the harness (coefficient domain) over the QB basis."""
    return splitmix_residues(seed_b, primes, N), splitmix_residues(seed_a, primes, N)


def decoded(words):
    v = words.view(np.float64)
    return v[0::2] + 1j * v[1::2]


@pytest.fixture(scope="module", params=FIXTURES)
def ref(request):
    g, N, k, kl, prec, primes = load(request.param)
    proots = dgt_generators(primes, N) if "dgt" in request.param else None
    o = Oracle(N, primes[:k], primes[k:], proots=proots)
    return g, N, k, kl, prec, primes, o


def test_fixture_holds_every_record(ref):
    g = ref[0]
    names = set(g.files)
    for must in ["hmult_l2", "hmult_l0", "hmult_norescale_l3", "hmult_norescale_l1", "rotate1_l3", "rotate4_l1",
                 "conjugate_l3", "add_l1", "sub_l3", "encode_s512", "encode_s8", "sk", "evk", "enc300", "enc301",
                 "mul_keys", "dec300", "dec_mul", "rot1_keys", "dec_rot1"]:
        assert "n1024_" + must in names, must


@pytest.mark.parametrize("level", LEVELS)
@pytest.mark.parametrize("rescale", [True, False])
def test_hmult_equals_reference(ref, level, rescale):
    g, N, k, kl, prec, primes, o = ref
    a = seeded_ct(101, 102, primes[:k], N)
    b = seeded_ct(103, 104, primes[:k], N)
    evk = tuple(o.ntt_fwd(x) for x in seeded_key(111, 112, primes, N))
    o0, o1, scale = o.hmult(a, b, evk, level, SCALE_A, SCALE_B, rescale=rescale)
    name = ("hmult_l%d" % (level - 1)) if rescale else ("hmult_norescale_l%d" % level)
    _, rscale, rslots, r0, r1 = ct_record(g["n1024_" + name], N)
    n = r0.shape[0]
    assert n == (level if rescale else level + 1)
    assert scale == rscale == SCALE_A * SCALE_B // primes[level]
    assert rslots == N // 2
    assert np.array_equal(o0[:n], r0) and np.array_equal(o1[:n], r1)


@pytest.mark.parametrize("level", LEVELS)
@pytest.mark.parametrize("r", ROTATIONS)
def test_rotate_left_equals_reference(ref, level, r):
    g, N, k, kl, prec, primes, o = ref
    c = seeded_ct(105, 106, primes[:k], N)
    rtk = tuple(o.ntt_fwd(x) for x in seeded_key(113 + 10 * r, 114 + 10 * r, primes, N))
    o0, o1 = o.rotate_left(c, r, rtk, level)
    aux, scale, slots, r0, r1 = ct_record(g["n1024_rotate%d_l%d" % (r, level)], N)
    assert aux == r and scale == SCALE_A and r0.shape[0] == level + 1
    assert np.array_equal(o0[: level + 1], r0) and np.array_equal(o1[: level + 1], r1)


@pytest.mark.parametrize("level", LEVELS)
def test_conjugate_equals_reference(ref, level):
    g, N, k, kl, prec, primes, o = ref
    c = seeded_ct(105, 106, primes[:k], N)
    cjk = tuple(o.ntt_fwd(x) for x in seeded_key(115, 116, primes, N))
    o0, o1 = o.conjugate(c, cjk, level)
    _, scale, slots, r0, r1 = ct_record(g["n1024_conjugate_l%d" % level], N)
    assert np.array_equal(o0[: level + 1], r0) and np.array_equal(o1[: level + 1], r1)


@pytest.mark.parametrize("level", LEVELS)
@pytest.mark.parametrize("subtract", [False, True])
def test_add_sub_equal_reference(ref, level, subtract):
    g, N, k, kl, prec, primes, o = ref
    a = seeded_ct(101, 102, primes[:k], N)
    c = seeded_ct(105, 106, primes[:k], N)
    o0, o1, _ = o.add(a, c, subtract=subtract)
    _, scale, slots, r0, r1 = ct_record(g["n1024_%s_l%d" % ("sub" if subtract else "add", level)], N)
    assert np.array_equal(o0[: level + 1], r0) and np.array_equal(o1[: level + 1], r1)


@pytest.mark.parametrize("slots", [512, 8])
def test_encode_equals_reference(ref, slots):
    g, N, k, kl, prec, primes, o = ref
    w = g["n1024_encode_s%d" % slots]
    assert int(w[0]) == SCALE_A
    got = o.encode(splitmix_values(200 + slots, slots), SCALE_A)
    assert np.array_equal(got, w[1:].reshape(k, N))


def test_reference_keys_hmult_and_decryptions(ref):
    """The reference's own keys and ciphertexts: the oracle's HMult of its two
    encryptions equals its ckks_mul output word for word, and the oracle's
    decryption of each ciphertext it wrote equals its ckks_decrypt."""
    g, N, k, kl, prec, primes, o = ref
    slots = N // 2
    s = g["n1024_sk"].view(np.int64)
    assert set(np.unique(s)) <= {-1, 0, 1}
    s_res = o.secret_residues(s, nres=k)
    evk_w = g["n1024_evk"].reshape(2, k + kl, N)
    evk = (o.ntt_fwd(evk_w[0]), o.ntt_fwd(evk_w[1]))
    _, sc1, sl1, a0, a1 = ct_record(g["n1024_enc300"], N)
    _, sc2, sl2, b0, b1 = ct_record(g["n1024_enc301"], N)
    assert sc1 == sc2 == 1 << prec and sl1 == sl2 == slots
    o0, o1, scale = o.hmult((a0, a1), (b0, b1), evk, k - 1, sc1, sc2)
    _, rscale, _, r0, r1 = ct_record(g["n1024_mul_keys"], N)
    assert scale == rscale
    assert np.array_equal(o0[: k - 1], r0) and np.array_equal(o1[: k - 1], r1)
    v1, v2 = splitmix_values(300, slots), splitmix_values(301, slots)
    for name, dec, expect, tol in (("enc300", "dec300", v1, 1e-9), ("mul_keys", "dec_mul", v1 * v2, 1e-6),
                                   ("rot1_keys", "dec_rot1", np.roll(v1, -1), 1e-6)):
        _, sc, sl, c0, c1 = ct_record(g["n1024_" + name], N)
        m = o.decrypt((np.vstack([c0, np.zeros((k - c0.shape[0], N), np.uint64)]),
                       np.vstack([c1, np.zeros((k - c1.shape[0], N), np.uint64)])), s_res, state=ST_COEF)
        got = o.decode(m[0], sl, sc)
        want = decoded(g["n1024_" + dec])
        assert np.array_equal(got, want), name           # the same FP64 decode, bit for bit
        assert np.max(np.abs(got - expect)) < tol, name   # and the values that went in
