"""Plaintext multiply, constant multiply / add and slot sums on the GPU against
the oracle's exact arithmetic (aoa-ntt src/ckks/ckks.cpp:484-690)."""
import numpy as np
import pytest

import oracle
from oracle import Oracle
from tests.ckks_inputs import make_keys, uniform_residues
from tests.gpu_util import require_gpu

pytestmark = pytest.mark.gpu


def _setup(transform=None, log_n=12, k=4, kl=3):
    import aoa_b200
    ps = oracle.gen_ntt_primes(60, 2 << log_n, k + kl)
    E = aoa_b200.Engine(log_n, ps[:k], ps[k:], scale_bits=40)
    ctx = aoa_b200.Context(E)
    if transform:
        ctx.set_transform(transform)
    return aoa_b200, E, ctx, Oracle(1 << log_n, ps[:k], ps[k:])


def _mulmod_rows(a, b, primes):
    return np.array([[int(x) * int(y) % q for x, y in zip(a[i], b[i])] for i, q in enumerate(primes)],
                    dtype=np.uint64)


@pytest.mark.parametrize("transform", [None, 3])
def test_mul_plaintext_and_rescale(transform):
    require_gpu()
    aoa, E, ctx, o = _setup(transform)
    rng = np.random.default_rng(1)
    N, k = E.N, E.k
    c0, c1 = uniform_residues(rng, E.q_primes, N), uniform_residues(rng, E.q_primes, N)
    vals = rng.uniform(-1, 1, 64) + 1j * rng.uniform(-1, 1, 64)
    scale = 1 << 40
    pt = o.encode(vals, scale)
    ct = aoa.Ciphertext.from_residues(ctx, c0, c1, slots=64, scale=scale)
    out = aoa.Ciphertext(ctx)
    aoa.ckks_mul_pt(ctx, out, ct, ctx.upload(pt), scale)
    fp = o.ntt_fwd(pt)
    w0 = o.ntt_inv(_mulmod_rows(o.ntt_fwd(c0), fp, E.q_primes))
    w1 = o.ntt_inv(_mulmod_rows(o.ntt_fwd(c1), fp, E.q_primes))
    w0, w1 = o.rescale(w0, w1, k - 1)
    assert out.level == k - 2 and out.scale == scale * scale // E.q_primes[k - 1]
    g0, g1 = out.download(nlimbs=k - 1, domain=aoa.AOA_COEF)
    assert np.array_equal(g0, w0[:k - 1]) and np.array_equal(g1, w1[:k - 1])


@pytest.mark.parametrize("val", [0.75, -1.25])
def test_mul_and_add_const(val):
    require_gpu()
    aoa, E, ctx, o = _setup()
    rng = np.random.default_rng(2)
    N, k = E.N, E.k
    c0, c1 = uniform_residues(rng, E.q_primes, N), uniform_residues(rng, E.q_primes, N)
    scale = 1 << 40
    ct = aoa.Ciphertext.from_residues(ctx, c0, c1, slots=8, scale=scale)
    out = aoa.Ciphertext(ctx)
    aoa.ckks_mul_const(ctx, out, ct, val, rescale=False)
    x = int(round(abs(val) * scale))
    want = [np.array([[int(v) * (x if val > 0 else q - x % q) % q for v in c[i]] for i, q in enumerate(E.q_primes)],
                     dtype=np.uint64) for c in (c0, c1)]
    g0, g1 = out.download(domain=aoa.AOA_COEF)
    assert np.array_equal(g0, want[0]) and np.array_equal(g1, want[1])
    assert out.scale == scale * scale // E.q_primes[k - 1] and out.level == k - 1
    # add a constant, ciphertext in coefficients and in the transform domain
    cnst = int(abs(val) * scale)
    for dom in (aoa.AOA_COEF, aoa.AOA_NTT):
        ct = aoa.Ciphertext.from_residues(ctx, c0, c1, slots=8, scale=scale)
        if dom == aoa.AOA_NTT:
            ct = aoa.Ciphertext.from_residues(ctx, o.ntt_fwd(c0), o.ntt_fwd(c1), slots=8, scale=scale, domain=dom)
        aoa.ckks_add_const(ctx, out, ct, val)
        w0 = c0.copy()
        for i, q in enumerate(E.q_primes):
            w0[i, 0] = (int(c0[i, 0]) + (cnst if val > 0 else -cnst)) % q
        g0, g1 = out.download(domain=aoa.AOA_COEF)
        assert np.array_equal(g0, w0) and np.array_equal(g1, c1), dom


@pytest.mark.parametrize("transform", [None, 3])
def test_sumslots_matches_oracle(transform):
    require_gpu()
    aoa, E, ctx, o = _setup(transform)
    steps = (1, 2, 4)
    keys = make_keys(o, seed=9, rotations=steps)
    rtks = {}
    for r in steps:
        b, a = keys["rtk"][r]
        rtks[r] = aoa.SwitchKey(ctx, o.ntt_inv(b), o.ntt_inv(a), domain=aoa.AOA_COEF)
    rng = np.random.default_rng(3)
    N, k = E.N, E.k
    c0, c1 = uniform_residues(rng, E.q_primes, N), uniform_residues(rng, E.q_primes, N)
    ct = aoa.Ciphertext.from_residues(ctx, c0, c1, slots=8)
    out = aoa.Ciphertext(ctx)
    aoa.ckks_sumslots(ctx, out, ct, rtks)
    w = (c0, c1)
    for r in (4, 2, 1):
        rot = o.rotate_left(w, r, keys["rtk"][r], k - 1)
        w = tuple(np.array([[(int(x) + int(y)) % q for x, y in zip(w[p][i], rot[p][i])]
                            for i, q in enumerate(E.q_primes)], dtype=np.uint64) for p in (0, 1))
    g0, g1 = out.download(domain=aoa.AOA_COEF)
    assert np.array_equal(g0, w[0]) and np.array_equal(g1, w[1])
