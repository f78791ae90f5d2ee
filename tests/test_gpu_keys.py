"""GPU key generation from given draws against the oracle (CKKSKeychain,
aoa-ntt src/ckks/ckkskeys.cpp:20-191): public, relinearisation, rotation and
conjugation keys must equal the oracle's residue for residue, and keys made
in a DGT context must relinearise exactly like the oracle's."""
import numpy as np
import pytest

import oracle
from oracle import Oracle
from tests.ckks_inputs import make_keys, uniform_residues
from tests.gpu_util import require_gpu

pytestmark = pytest.mark.gpu


def _engine(log_n=12, k=4, kl=3):
    import aoa_b200
    ps = oracle.gen_ntt_primes(60, 2 << log_n, k + kl)
    E = aoa_b200.Engine(log_n, ps[:k], ps[k:])
    return aoa_b200, E, aoa_b200.Context(E), Oracle(1 << log_n, ps[:k], ps[k:])


def _draws(ctx, keys, rotations, conjugation):
    d = {"pk": (ctx.upload(keys["pk_raw"][0]), ctx.upload(keys["pk_raw"][1]))}
    d["evk"] = tuple(ctx.upload(x) for x in keys["evk_raw"][1:])
    for r in rotations:
        d[("rtk", r)] = tuple(ctx.upload(x) for x in keys["rtk_raw"][r][1:])
    if conjugation:
        d["cjk"] = tuple(ctx.upload(x) for x in keys["cjk_raw"][1:])
    return d


def _canonical(x, primes):
    """The reference's coefficient automorphism writes q (not 0) for a negated
    zero; reduce such entries so residues compare as numbers mod q."""
    x = np.array(x, dtype=np.uint64)
    for i, q in enumerate(primes):
        x[i][x[i] == np.uint64(q)] = 0
    return x


def test_keygen_matches_oracle():
    require_gpu()
    aoa, E, ctx, o = _engine()
    rot = (1, 3, -2)
    keys = make_keys(o, seed=17, rotations=rot, conjugation=True)
    s = ctx.upload(keys["s"])
    nqb = len(E.primes)
    # secrets of the keys
    assert np.array_equal(aoa.ckks_secret_square(ctx, s, nqb).numpy(), keys["evk_raw"][0])
    for r in rot:
        g = aoa.galois_left(E.N, r)
        assert np.array_equal(aoa.ckks_secret_galois(ctx, s, g, nqb).numpy(),
                              _canonical(keys["rtk_raw"][r][0], E.primes)), r
    sc = aoa.ckks_secret_galois(ctx, s, aoa.galois_conjugate(E.N), nqb).numpy()
    assert np.array_equal(sc, _canonical(keys["cjk_raw"][0], E.primes))
    # the keys
    got = aoa.ckks_keygen(ctx, s, _draws(ctx, keys, rot, True), rotations=rot, conjugation=True)
    pb, pa = got["pk"].download(domain=aoa.AOA_NTT)
    assert np.array_equal(pb, keys["pk"][0]) and np.array_equal(pa, keys["pk"][1])
    b, a, dom = got["evk"].numpy()
    assert dom == aoa.AOA_NTT
    assert np.array_equal(b, keys["evk"][0]) and np.array_equal(a, keys["evk"][1])
    for r in rot:
        b, a, _ = got["rtk"][r].numpy()
        assert np.array_equal(b, keys["rtk"][r][0]) and np.array_equal(a, keys["rtk"][r][1]), r
    b, a, _ = got["cjk"].numpy()
    assert np.array_equal(b, keys["cjk"][0]) and np.array_equal(a, keys["cjk"][1])


def test_keygen_in_dgt_context_relinearises_like_oracle():
    require_gpu()
    aoa, E, ctx, o = _engine(log_n=12, k=4, kl=4)
    ctx.set_transform(aoa.AOA_DGT)
    keys = make_keys(o, seed=23)
    s = ctx.upload(keys["s"])
    got = aoa.ckks_keygen(ctx, s, _draws(ctx, keys, (), False))
    _, _, dom = got["evk"].numpy()
    assert dom == aoa.AOA_DGT
    rng = np.random.default_rng(2)
    N = E.N
    a0, a1 = uniform_residues(rng, E.q_primes, N), uniform_residues(rng, E.q_primes, N)
    ca = aoa.Ciphertext.from_residues(ctx, a0, a1, slots=N // 2, scale=1 << 40)
    cb = aoa.Ciphertext.from_residues(ctx, a1, a0, slots=N // 2, scale=1 << 40)
    out = aoa.Ciphertext(ctx)
    aoa.ckks_mul(ctx, out, ca, cb, got["evk"])
    w0, w1, _ = o.hmult((a0, a1), (a1, a0), keys["evk"], E.k - 1, 1 << 40, 1 << 40)
    g0, g1 = out.download(nlimbs=E.k - 1, domain=aoa.AOA_COEF)
    assert np.array_equal(g0, w0[:E.k - 1]) and np.array_equal(g1, w1[:E.k - 1])
    # the public key made in the DGT domain equals the oracle's after a domain change
    pb, pa = got["pk"].download(domain=aoa.AOA_NTT)
    assert np.array_equal(pb, keys["pk"][0]) and np.array_equal(pa, keys["pk"][1])
