"""GPU parity of the DGT variant (aoa-dgt) against the CPU oracle, through the C ABI.

Transform-domain values must equal the oracle's restatement of the
reference's DGT bit for bit on the reference's own primes, generators and
twist roots (tests/golden/dgt_roots.json); evaluation results (HMult,
rotation, conjugation) must equal the oracle's in coefficients."""
import json
import os
from types import SimpleNamespace

import numpy as np
import pytest

import oracle
from oracle import DgtOracle, Oracle, dgt_prime_set, dgt_roots, fold, unfold
from tests.ckks_inputs import make_keys, uniform_residues
from tests.gpu_util import require_gpu

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.fixture(scope="module")
def dgt_table():
    with open(os.path.join(HERE, "golden", "dgt_roots.json")) as f:
        return json.load(f)


def _setup(dgt_table, log_n, k, kl, prec, transform=None):
    import aoa_b200
    Q, B = dgt_prime_set(dgt_table, k, kl, prec)
    primes = Q + B
    g, r = dgt_roots(dgt_table, primes, (1 << log_n) // 2)
    E = aoa_b200.Engine(log_n, Q, B, generators=g, dgt_roots=r)
    ctx = aoa_b200.Context(E)
    if transform is not None:
        ctx.set_transform(transform)
    return aoa_b200, E, ctx, DgtOracle((1 << log_n) // 2, primes, g, r), Oracle(1 << log_n, Q, B, proots=g)


@pytest.mark.parametrize("log_n,prec", [(10, 55), (11, 45), (12, 48), (13, 52), (16, 55)])
def test_dgt_bit_exact(dgt_table, log_n, prec):
    require_gpu()
    aoa, E, ctx, D, _ = _setup(dgt_table, log_n, 3, 2, prec)
    rng = np.random.default_rng(log_n)
    x = uniform_residues(rng, E.primes, E.N)            # planar GI limbs = coefficients
    d = ctx.upload(x)
    ctx.dgt_fwd(d, 1, 0, E.k + E.kl)
    got = d.numpy()
    want = unfold(D.fwd(fold(x)))
    assert np.array_equal(got, want)
    ctx.dgt_inv(d, 1, 0, E.k + E.kl)
    assert np.array_equal(d.numpy(), x)
    # strided batch: 3 polys of 5 limbs, limbs 1..3 only (the pointer names
    # limb 1 of poly 0, as for the NTT entry points)
    xs = np.stack([uniform_residues(rng, E.primes, E.N) for _ in range(3)])
    d = ctx.upload(xs)
    ctx.dgt_fwd(SimpleNamespace(ptr=d.offset(E.N)), 3, 1, 3, poly_stride=E.k + E.kl)
    got = d.numpy()
    for p in range(3):
        assert np.array_equal(got[p, 1:4], unfold(D.fwd(fold(xs[p, 1:4]), first=1)))
        assert np.array_equal(got[p, 0], xs[p, 0]) and np.array_equal(got[p, 4], xs[p, 4])


@pytest.mark.parametrize("log_n", [12, 16])
def test_dgt_split_knob_keeps_results(dgt_table, log_n):
    """The DGT's cyclic limb transforms take their own R x C split (knob
    dgt_split, default 1); every split gives the oracle's DGT."""
    require_gpu()
    aoa, E, ctx, D, _ = _setup(dgt_table, log_n, 3, 2, 55)
    assert E.tune_get("dgt_split") == 1
    rng = np.random.default_rng(log_n + 3)
    x = uniform_residues(rng, E.primes, E.N)
    want = unfold(D.fwd(fold(x)))
    for split in (-1, 0, 1, 2):
        E.tune("dgt_split", split)
        d = ctx.upload(x)
        ctx.dgt_fwd(d, 1, 0, E.k + E.kl)
        assert np.array_equal(d.numpy(), want), split
        ctx.dgt_inv(d, 1, 0, E.k + E.kl)
        assert np.array_equal(d.numpy(), x), split
    E.tune("dgt_split", 1)


def test_gi_layout_and_mul(dgt_table):
    require_gpu()
    aoa, E, ctx, D, _ = _setup(dgt_table, 12, 2, 2, 55)
    lib = aoa.capi.load()
    rng = np.random.default_rng(3)
    a = uniform_residues(rng, E.primes, E.N)
    b = uniform_residues(rng, E.primes, E.N)
    inter = fold(a)                                      # reference layout [limb][N/2][2]
    src = ctx.upload(inter)
    dst = ctx.alloc(a.shape)
    aoa.capi.check(lib.aoa_gi_to_planar(ctx.handle, dst.ptr, src.ptr, 4))
    assert np.array_equal(dst.numpy(), a)
    back = ctx.alloc(inter.shape)
    aoa.capi.check(lib.aoa_gi_from_planar(ctx.handle, back.ptr, dst.ptr, 4))
    assert np.array_equal(back.numpy(), inter)
    da, db, dc = ctx.upload(a), ctx.upload(b), ctx.alloc(a.shape)
    aoa.capi.check(lib.aoa_gi_mul(ctx.handle, dc.ptr, da.ptr, db.ptr, 0, 4))
    assert np.array_equal(dc.numpy(), unfold(D.gi_mul(fold(a), fold(b))))


def test_dgt_product_is_negacyclic(dgt_table):
    require_gpu()
    aoa, E, ctx, D, o = _setup(dgt_table, 11, 2, 1, 55)
    lib = aoa.capi.load()
    rng = np.random.default_rng(4)
    a = uniform_residues(rng, E.primes, E.N)
    b = uniform_residues(rng, E.primes, E.N)
    da, db = ctx.upload(a), ctx.upload(b)
    ctx.dgt_fwd(da, 1, 0, 3)
    ctx.dgt_fwd(db, 1, 0, 3)
    aoa.capi.check(lib.aoa_gi_mul(ctx.handle, da.ptr, da.ptr, db.ptr, 0, 3))
    ctx.dgt_inv(da, 1, 0, 3)
    fa, fb = o.ntt_fwd(a), o.ntt_fwd(b)
    prod = np.array([[int(u) * int(v) % q for u, v in zip(fa[i], fb[i])] for i, q in enumerate(E.primes)],
                    dtype=np.uint64)
    assert np.array_equal(da.numpy(), o.ntt_inv(prod))


def test_engine_reports_roots_and_derives_its_own(dgt_table):
    require_gpu()
    import aoa_b200
    aoa, E, ctx, D, _ = _setup(dgt_table, 12, 2, 1, 55)
    out = np.zeros(2 * len(E.primes), dtype=np.uint64)
    aoa.capi.check(aoa.capi.load().aoa_engine_dgt_roots(E.handle, out.ctypes.data))
    _, r = dgt_roots(dgt_table, E.primes, E.N // 2)
    assert [tuple(int(v) for v in out[2 * i:2 * i + 2]) for i in range(len(E.primes))] == r
    # without given roots the engine derives r from the generator; products agree
    E2 = aoa_b200.Engine(12, E.q_primes, E.b_primes)
    ctx2 = aoa_b200.Context(E2)
    rng = np.random.default_rng(8)
    a = uniform_residues(rng, E.primes, E.N)
    b = uniform_residues(rng, E.primes, E.N)
    res = []
    for c in (ctx, ctx2):
        da, db = c.upload(a), c.upload(b)
        c.dgt_fwd(da, 1, 0, 3)
        c.dgt_fwd(db, 1, 0, 3)
        aoa.capi.check(aoa.capi.load().aoa_gi_mul(c.handle, da.ptr, da.ptr, db.ptr, 0, 3))
        c.dgt_inv(da, 1, 0, 3)
        res.append(da.numpy())
    assert np.array_equal(res[0], res[1])


@pytest.mark.parametrize("log_n", [11, 16])
def test_dgt_on_primes_one_mod_2_32(log_n):
    """The twist (three Shoup products per Gaussian integer) and the cyclic
    limb transforms on primes q = 1 mod 2^32, which take the shorter Shoup
    remainder, next to another prime below 2^60 and one above it, with the
    roots the engine derives: the forward DGT equals the oracle's on the same
    generators and roots, and the inverse undoes it."""
    require_gpu()
    import aoa_b200 as aoa
    from aoa_b200 import params
    n = 1 << log_n
    q1 = oracle.gen_ntt_primes(60, 1 << 32, 2)
    other = [q for q in oracle.gen_ntt_primes(59, 2 * n, 8) if q % (1 << 32) != 1][:1]
    big = oracle.gen_ntt_primes(62, 2 * n, 1)
    Q, B = [q1[0], other[0], big[0]], [q1[1]]
    primes = Q + B
    E = aoa.Engine(log_n, Q, B)
    ctx = aoa.Context(E)
    out = np.zeros(2 * len(primes), dtype=np.uint64)
    aoa.capi.check(aoa.capi.load().aoa_engine_dgt_roots(E.handle, out.ctypes.data))
    r = [tuple(int(v) for v in out[2 * i:2 * i + 2]) for i in range(len(primes))]
    g = [params.primitive_root(q) for q in primes]
    D = DgtOracle(n // 2, primes, g, r)
    rng = np.random.default_rng(log_n + 60)
    xs = np.stack([uniform_residues(rng, primes, n) for _ in range(2)])
    xs[1] = np.array([[q - 1] * n for q in primes], dtype=np.uint64)
    d = ctx.upload(xs)
    ctx.dgt_fwd(d, 2, 0, len(primes))
    got = d.numpy()
    for p in range(2):
        assert np.array_equal(got[p], unfold(D.fwd(fold(xs[p])))), p
    ctx.dgt_inv(d, 2, 0, len(primes))
    assert np.array_equal(d.numpy(), xs)


def test_dgt_hmult_on_primes_one_mod_2_32():
    """ckks_mul and ckks_mul_batch on a DGT context over primes q = 1 mod 2^32
    (the benchmark's kind: short Shoup remainders in the twist, the limb
    transforms and the basis conversion), roots derived by the engine: the
    oracle's HMult residues in coefficients."""
    require_gpu()
    import aoa_b200 as aoa
    log_n, k, kl = 12, 4, 4
    ps = oracle.gen_ntt_primes(60, 1 << 32, k + kl)
    Q, B = ps[:k], ps[k:]
    E = aoa.Engine(log_n, Q, B)
    ctx = aoa.Context(E)
    ctx.set_transform(aoa.AOA_DGT)
    o = Oracle(1 << log_n, Q, B)
    keys = make_keys(o, seed=33)
    evk = aoa.SwitchKey(ctx, o.ntt_inv(keys["evk"][0]), o.ntt_inv(keys["evk"][1]), domain=aoa.AOA_COEF)
    rng = np.random.default_rng(77)
    N = 1 << log_n
    pairs = [tuple(uniform_residues(rng, Q, N) for _ in range(4)) for _ in range(3)]
    sa, sb = 1 << 40, (1 << 40) + 77
    level = k - 1
    w = [o.hmult((a0, a1), (b0, b1), keys["evk"], level, sa, sb) for a0, a1, b0, b1 in pairs]
    cts = [(aoa.Ciphertext.from_residues(ctx, a0, a1, slots=N // 2, scale=sa),
            aoa.Ciphertext.from_residues(ctx, b0, b1, slots=N // 2, scale=sb)) for a0, a1, b0, b1 in pairs]
    out = aoa.Ciphertext(ctx)
    aoa.ckks_mul(ctx, out, cts[0][0], cts[0][1], evk)
    g0, g1 = out.download(nlimbs=level, domain=aoa.AOA_COEF)
    assert out.scale == w[0][2]
    assert np.array_equal(g0, w[0][0][:level]) and np.array_equal(g1, w[0][1][:level])
    cts = [(aoa.Ciphertext.from_residues(ctx, a0, a1, slots=N // 2, scale=sa),
            aoa.Ciphertext.from_residues(ctx, b0, b1, slots=N // 2, scale=sb)) for a0, a1, b0, b1 in pairs]
    outs = [aoa.Ciphertext(ctx) for _ in pairs]
    aoa.ckks_mul_batch(ctx, outs, [c[0] for c in cts], [c[1] for c in cts], evk)
    for ob, (w0, w1, _) in zip(outs, w):
        g0, g1 = ob.download(nlimbs=level, domain=aoa.AOA_COEF)
        assert np.array_equal(g0, w0[:level]) and np.array_equal(g1, w1[:level])


@pytest.mark.parametrize("log_n,prec,in_domain", [(12, 55, "coef"), (13, 52, "dgt"), (11, 45, "coef")])
def test_dgt_hmult_matches_oracle(dgt_table, log_n, prec, in_domain):
    """ckks_mul of the DGT library (aoa-dgt src/ckks.cpp:275-358): the same
    residues as the oracle's HMult (the transform only changes the domain of
    exact products)."""
    require_gpu()
    aoa, E, ctx, D, o = _setup(dgt_table, log_n, 4, 4, prec, transform=3)
    keys = make_keys(o, seed=31)
    evk = aoa.SwitchKey(ctx, o.ntt_inv(keys["evk"][0]), o.ntt_inv(keys["evk"][1]), domain=aoa.AOA_COEF)
    rng = np.random.default_rng(log_n + prec)
    N, k = E.N, E.k
    a0, a1 = uniform_residues(rng, E.q_primes, N), uniform_residues(rng, E.q_primes, N)
    b0, b1 = uniform_residues(rng, E.q_primes, N), uniform_residues(rng, E.q_primes, N)
    sa, sb = 1 << 40, (1 << 40) + 77
    if in_domain == "coef":
        ca = aoa.Ciphertext.from_residues(ctx, a0, a1, slots=N // 2, scale=sa)
        cb = aoa.Ciphertext.from_residues(ctx, b0, b1, slots=N // 2, scale=sb)
    else:
        ca = aoa.Ciphertext.from_residues(ctx, unfold(D.fwd(fold(a0))), unfold(D.fwd(fold(a1))), slots=N // 2,
                                          scale=sa, domain=aoa.AOA_DGT)
        cb = aoa.Ciphertext.from_residues(ctx, unfold(D.fwd(fold(b0))), unfold(D.fwd(fold(b1))), slots=N // 2,
                                          scale=sb, domain=aoa.AOA_DGT)
    for level, rescale in ((k - 1, True), (2, False)):
        ca.set(level, N // 2, sa, ca.domain)
        cb.set(level, N // 2, sb, cb.domain)
        out = aoa.Ciphertext(ctx)
        if rescale:
            aoa.ckks_mul(ctx, out, ca, cb, evk)
        else:
            aoa.ckks_mul_without_rescale(ctx, out, ca, cb, evk)
        w0, w1, wscale = o.hmult((a0, a1), (b0, b1), keys["evk"], level, sa, sb, rescale=rescale)
        nl = level if rescale else level + 1
        assert out.domain == aoa.AOA_DGT and out.scale == wscale
        g0, g1 = out.download(nlimbs=nl, domain=aoa.AOA_COEF)
        assert np.array_equal(g0, w0[:nl]) and np.array_equal(g1, w1[:nl]), (level, rescale)
        gd0, _ = out.download(nlimbs=nl, domain=aoa.AOA_DGT)
        assert np.array_equal(gd0, unfold(D.fwd(fold(w0[:nl]))))


def test_dgt_rotate_conjugate_match_oracle(dgt_table):
    require_gpu()
    aoa, E, ctx, D, o = _setup(dgt_table, 12, 3, 3, 55, transform=3)
    keys = make_keys(o, seed=41, rotations=(1, 5), conjugation=True)
    rng = np.random.default_rng(6)
    N = E.N
    c0, c1 = uniform_residues(rng, E.q_primes, N), uniform_residues(rng, E.q_primes, N)
    for step in (1, 5):
        rk = keys["rtk"][step]
        key = aoa.SwitchKey(ctx, o.ntt_inv(rk[0]), o.ntt_inv(rk[1]), domain=aoa.AOA_COEF)
        ct = aoa.Ciphertext.from_residues(ctx, c0, c1, slots=N // 2)
        out = aoa.Ciphertext(ctx)
        aoa.ckks_rotate_left(ctx, out, ct, step, key)
        w0, w1 = o.rotate_left((c0, c1), step, rk, E.k - 1)
        g0, g1 = out.download(domain=aoa.AOA_COEF)
        assert np.array_equal(g0, w0) and np.array_equal(g1, w1), step
    cj = keys["cjk"]
    key = aoa.SwitchKey(ctx, o.ntt_inv(cj[0]), o.ntt_inv(cj[1]), domain=aoa.AOA_COEF)
    ct = aoa.Ciphertext.from_residues(ctx, c0, c1, slots=N // 2)
    out = aoa.Ciphertext(ctx)
    aoa.ckks_conjugate(ctx, out, ct, key)
    w0, w1 = o.conjugate((c0, c1), cj, E.k - 1)
    g0, g1 = out.download(domain=aoa.AOA_COEF)
    assert np.array_equal(g0, w0) and np.array_equal(g1, w1)


def test_dgt_context_rejects_ntt_key(dgt_table):
    require_gpu()
    aoa, E, ctx, D, o = _setup(dgt_table, 12, 3, 2, 55)
    keys = make_keys(o, seed=5)
    evk_ntt = aoa.SwitchKey(ctx, keys["evk"][0], keys["evk"][1], domain=aoa.AOA_NTT)
    ctx.set_transform(aoa.AOA_DGT)
    rng = np.random.default_rng(1)
    N = E.N
    ca = aoa.Ciphertext.from_residues(ctx, *(uniform_residues(rng, E.q_primes, N) for _ in range(2)), slots=N // 2)
    out = aoa.Ciphertext(ctx)
    with pytest.raises(aoa.AoaError) as ei:
        aoa.ckks_mul(ctx, out, ca, ca, evk_ntt)
    assert ei.value.status == 1


@pytest.mark.parametrize("rescale", [True, False])
def test_dgt_hmult_batch_matches_oracle_and_per_call(dgt_table, rescale):
    """Batched HMult on a DGT context (aoa-dgt ckks_mul, src/ckks.cpp:275-360,
    one launch per stage over the batch; 10 products at mixed levels, inputs
    in coefficients and in the DGT domain, an output aliasing an input; the
    group of 8 runs as two halves on two streams): every product equals the
    per-call DGT HMult and the oracle."""
    require_gpu()
    aoa, E, ctx, D, o = _setup(dgt_table, 12, 4, 4, 55, transform=3)
    keys = make_keys(o, seed=33)
    evk = aoa.SwitchKey(ctx, o.ntt_inv(keys["evk"][0]), o.ntt_inv(keys["evk"][1]), domain=aoa.AOA_COEF)
    rng = np.random.default_rng(12)
    N, k = E.N, E.k
    levels = [3, 3, 2, 3, 3, 3, 3, 3, 2, 3]
    data = [tuple(uniform_residues(rng, E.q_primes, N) for _ in range(4)) for _ in levels]

    def make(z, x):
        dom = aoa.AOA_DGT if z % 2 else aoa.AOA_COEF
        conv = (lambda v: unfold(D.fwd(fold(v)))) if dom == aoa.AOA_DGT else (lambda v: v)
        ca = aoa.Ciphertext.from_residues(ctx, conv(x[0]), conv(x[1]), slots=8, scale=1 << 40, domain=dom)
        cb = aoa.Ciphertext.from_residues(ctx, conv(x[2]), conv(x[3]), slots=8, scale=(1 << 40) + 3, domain=dom)
        ca.set(levels[z], 8, 1 << 40, dom)
        cb.set(levels[z], 8, (1 << 40) + 3, dom)
        return ca, cb

    pairs = [make(z, x) for z, x in enumerate(data)]
    outs = [aoa.Ciphertext(ctx) for _ in data]
    outs[4] = pairs[4][0]                                  # output aliases an input
    aoa.ckks_mul_batch(ctx, outs, [p[0] for p in pairs], [p[1] for p in pairs], evk, rescale=rescale)
    for z, x in enumerate(data):
        lv = levels[z]
        nl = lv if rescale else lv + 1
        pad = lambda v: np.concatenate([v[: lv + 1], np.zeros((k - lv - 1, N), dtype=np.uint64)])
        w0, w1, wsc = o.hmult((pad(x[0]), pad(x[1])), (pad(x[2]), pad(x[3])), keys["evk"], lv, 1 << 40,
                              (1 << 40) + 3, rescale=rescale)
        assert outs[z].domain == aoa.AOA_DGT and outs[z].level == nl - 1 and outs[z].scale == wsc, z
        g0, g1 = outs[z].download(nlimbs=nl, domain=aoa.AOA_COEF)
        assert np.array_equal(g0, w0[:nl]) and np.array_equal(g1, w1[:nl]), z
        ca, cb = make(z, x)
        single = aoa.Ciphertext(ctx)
        (aoa.ckks_mul if rescale else aoa.ckks_mul_without_rescale)(ctx, single, ca, cb, evk)
        s0, s1 = single.download(nlimbs=nl, domain=aoa.AOA_DGT)
        b0, b1 = outs[z].download(nlimbs=nl, domain=aoa.AOA_DGT)
        assert np.array_equal(s0, b0) and np.array_equal(s1, b1), z
