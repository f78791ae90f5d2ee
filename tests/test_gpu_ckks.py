"""GPU parity of the CKKS hot path against the CPU oracle, through the C ABI.

Every residue of every live output limb must be bit-exact.  Inputs are seeded
synthetic ciphertexts / keys (tests/ckks_inputs.py)."""
import numpy as np
import pytest

import oracle
from oracle import Oracle, reference_prime_set, ST_COEF, ST_NTT
from tests.ckks_inputs import make_keys, encrypt_values, uniform_residues
from tests.gpu_util import require_gpu

pytestmark = pytest.mark.gpu


def _setup(log_n, Q, B, scale_bits=0):
    import aoa_b200
    E = aoa_b200.Engine(log_n, Q, B, scale_bits=scale_bits)
    ctx = aoa_b200.Context(E)
    return aoa_b200, E, ctx, Oracle(1 << log_n, Q, B)


def _sets(ref_table):
    q55, b55 = reference_prime_set(ref_table, 4, 4, 55)
    p60 = oracle.gen_ntt_primes(60, 1 << 17, 11)
    return {"ref55": (q55, b55), "p60": (p60[:5], p60[5:])}


@pytest.mark.parametrize("pset", ["ref55", "p60"])
def test_modup_moddown_rescale(ref_table, pset):
    require_gpu()
    Q, B = _sets(ref_table)[pset]
    aoa, E, ctx, o = _setup(12, Q, B)
    rng = np.random.default_rng(3)
    N, k, kl = E.N, E.k, E.kl
    xq = uniform_residues(rng, Q, N)
    xb = uniform_residues(rng, B, N)
    dq = ctx.upload(xq)
    dqb = ctx.upload(np.concatenate([xq, xb]))
    for level in range(k):
        out_b = ctx.alloc((kl, N))
        aoa.capi.check(aoa.capi.load().aoa_modup(ctx.handle, dq.ptr, out_b.ptr, level))
        assert np.array_equal(out_b.numpy(), o.modup(xq, level)), "modup level %d" % level
        out_q = ctx.alloc((k, N))
        aoa.capi.check(aoa.capi.load().aoa_moddown(ctx.handle, dqb.ptr, out_q.ptr, level))
        assert np.array_equal(out_q.numpy()[: level + 1], o.moddown(np.concatenate([xq, xb]), level)[: level + 1])
    for level in range(1, k):
        d = ctx.upload(np.stack([xq, xq[::-1].copy()]))
        aoa.capi.check(aoa.capi.load().aoa_rescale_polys(ctx.handle, d.ptr, 2, k, level))
        got = d.numpy()
        w0, w1 = o.rescale(xq, xq[::-1].copy(), level)
        assert np.array_equal(got[0, :level], w0[:level]) and np.array_equal(got[1, :level], w1[:level])


def _rand_ct(rng, primes, N, nlimbs):
    return uniform_residues(rng, primes[:nlimbs], N), uniform_residues(rng, primes[:nlimbs], N)


@pytest.mark.parametrize("pset,log_n", [("ref55", 12), ("p60", 12), ("p60", 13)])
@pytest.mark.parametrize("in_domain", ["coef", "ntt"])
def test_hmult_relin_rescale_bit_exact(ref_table, pset, log_n, in_domain):
    require_gpu()
    Q, B = _sets(ref_table)[pset]
    aoa, E, ctx, o = _setup(log_n, Q, B)
    keys = make_keys(o, seed=21)
    evk = aoa.SwitchKey(ctx, keys["evk"][0], keys["evk"][1], domain=aoa.AOA_NTT)
    rng = np.random.default_rng(log_n)
    N, k = E.N, E.k
    a0, a1 = _rand_ct(rng, Q, N, k)
    b0, b1 = _rand_ct(rng, Q, N, k)
    dom = aoa.AOA_COEF if in_domain == "coef" else aoa.AOA_NTT
    st = ST_COEF if in_domain == "coef" else ST_NTT
    sa, sb = 1 << 40, (1 << 40) + 12345
    ca = aoa.Ciphertext.from_residues(ctx, a0, a1, slots=N // 2, scale=sa, domain=dom)
    cb = aoa.Ciphertext.from_residues(ctx, b0, b1, slots=N // 2, scale=sb, domain=dom)
    for level in (k - 1, 2):
        ca.set(level, N // 2, sa, ca.domain)
        cb.set(level, N // 2, sb, cb.domain)
        out = aoa.Ciphertext(ctx)
        aoa.ckks_mul(ctx, out, ca, cb, evk)
        # the oracle is not level aware: hand it the live limbs and stale zeros above
        pad = lambda x: np.concatenate([x[: level + 1], np.zeros((k - level - 1, N), dtype=np.uint64)])
        A = [pad(v) for v in (ca.download(domain=aoa.AOA_COEF if st == ST_COEF else aoa.AOA_NTT, nlimbs=k))]
        Bc = [pad(v) for v in (cb.download(domain=aoa.AOA_COEF if st == ST_COEF else aoa.AOA_NTT, nlimbs=k))]
        w0, w1, wsc = o.hmult(A, Bc, keys["evk"], level, sa, sb, rescale=True, a_state=st, b_state=st)
        g0, g1 = out.download(nlimbs=level)
        assert out.level == level - 1 and out.scale == wsc
        assert np.array_equal(g0, w0[:level]) and np.array_equal(g1, w1[:level])


@pytest.mark.parametrize("pset", ["ref55", "p60"])
def test_hmult_plain_path_matches_oracle(ref_table, pset):
    """The reference-structured per-call path gives the same residues."""
    require_gpu()
    Q, B = _sets(ref_table)[pset]
    aoa, E, ctx, o = _setup(12, Q, B)
    keys = make_keys(o, seed=31)
    evk = aoa.SwitchKey(ctx, *keys["evk"])
    rng = np.random.default_rng(77)
    N, k = E.N, E.k
    a = _rand_ct(rng, Q, N, k)
    b = _rand_ct(rng, Q, N, k)
    ca = aoa.Ciphertext.from_residues(ctx, *a, slots=8, scale=1 << 40)
    cb = aoa.Ciphertext.from_residues(ctx, *b, slots=8, scale=1 << 41)
    out = aoa.Ciphertext(ctx)
    aoa.ckks_mul_plain(ctx, out, ca, cb, evk)
    w0, w1, wsc = o.hmult(a, b, keys["evk"], k - 1, 1 << 40, 1 << 41, rescale=True)
    g0, g1 = out.download(nlimbs=k - 1)
    assert out.level == k - 2 and out.scale == wsc and out.domain == aoa.AOA_COEF
    assert np.array_equal(g0, w0[: k - 1]) and np.array_equal(g1, w1[: k - 1])


def test_hmult_chain_in_transform_domain(ref_table):
    """Three chained HMults stay in the transform domain and match the oracle chain."""
    require_gpu()
    Q, B = _sets(ref_table)["p60"]
    aoa, E, ctx, o = _setup(12, Q, B)
    keys = make_keys(o, seed=5)
    evk = aoa.SwitchKey(ctx, *keys["evk"])
    rng = np.random.default_rng(3)
    N, k = E.N, E.k
    x = _rand_ct(rng, Q, N, k)
    cx = aoa.Ciphertext.from_residues(ctx, *x, slots=4, scale=1 << 30)
    cur, sc = (x[0].copy(), x[1].copy()), 1 << 30
    lvl = k - 1
    for _ in range(3):
        aoa.ckks_mul(ctx, cx, cx, cx, evk)
        assert cx.domain == aoa.AOA_NTT
        pad = lambda v: np.concatenate([v[: lvl + 1], np.zeros((k - lvl - 1, N), dtype=np.uint64)])
        w0, w1, sc = o.hmult((pad(cur[0]), pad(cur[1])), (pad(cur[0]), pad(cur[1])), keys["evk"], lvl, sc, sc)
        lvl -= 1
        cur = (w0, w1)
        g0, g1 = cx.download(nlimbs=lvl + 1)
        assert cx.level == lvl and cx.scale == sc
        assert np.array_equal(g0, w0[: lvl + 1]) and np.array_equal(g1, w1[: lvl + 1])


def test_hmult_without_rescale_and_aliasing(ref_table):
    require_gpu()
    Q, B = _sets(ref_table)["p60"]
    aoa, E, ctx, o = _setup(12, Q, B)
    keys = make_keys(o, seed=4)
    evk = aoa.SwitchKey(ctx, *keys["evk"])
    rng = np.random.default_rng(8)
    N, k = E.N, E.k
    a0, a1 = _rand_ct(rng, Q, N, k)
    ca = aoa.Ciphertext.from_residues(ctx, a0, a1, slots=4, scale=1 << 30)
    w0, w1, wsc = o.hmult((a0, a1), (a0, a1), keys["evk"], k - 1, 1 << 30, 1 << 30, rescale=False)
    aoa.ckks_mul_without_rescale(ctx, ca, ca, ca, evk)       # out aliases both inputs
    g0, g1 = ca.download(nlimbs=k)
    assert np.array_equal(g0, w0) and np.array_equal(g1, w1) and ca.scale == wsc


@pytest.mark.parametrize("pset", ["ref55", "p60"])
def test_rotate_conjugate_bit_exact(ref_table, pset):
    require_gpu()
    Q, B = _sets(ref_table)[pset]
    aoa, E, ctx, o = _setup(12, Q, B)
    keys = make_keys(o, seed=9, rotations=(1, 2, 64), conjugation=True)
    rng = np.random.default_rng(1)
    N, k = E.N, E.k
    c0, c1 = _rand_ct(rng, Q, N, k)
    for r in (1, 2, 64):
        rtk = aoa.SwitchKey(ctx, *keys["rtk"][r])
        ct = aoa.Ciphertext.from_residues(ctx, c0, c1, slots=N // 2)
        out = aoa.Ciphertext(ctx)
        aoa.ckks_rotate_left(ctx, out, ct, r, rtk)
        w0, w1 = o.rotate_left((c0, c1), r, keys["rtk"][r], k - 1, state=ST_COEF)
        g0, g1 = out.download(nlimbs=k)
        assert np.array_equal(g0, w0) and np.array_equal(g1, w1), r
        # the reference's per-call sequence, from coefficient and transform-domain inputs
        for dom in (aoa.AOA_COEF, aoa.AOA_NTT):
            ct = aoa.Ciphertext.from_residues(ctx, c0, c1, slots=N // 2)
            ct.upload(*(ct.download(nlimbs=k, domain=dom)), domain=dom)
            out = aoa.Ciphertext(ctx)
            aoa.ckks_rotate_plain(ctx, out, ct, r, rtk)
            assert out.domain == aoa.AOA_COEF and ct.domain == dom
            g0, g1 = out.download(nlimbs=k)
            assert np.array_equal(g0, w0) and np.array_equal(g1, w1), (r, dom)
    cjk = aoa.SwitchKey(ctx, *keys["cjk"])
    ct = aoa.Ciphertext.from_residues(ctx, c0, c1, slots=N // 2)
    out = aoa.Ciphertext(ctx)
    aoa.ckks_conjugate(ctx, out, ct, cjk)
    w0, w1 = o.conjugate((c0, c1), keys["cjk"], k - 1, state=ST_COEF)
    g0, g1 = out.download(nlimbs=k)
    assert np.array_equal(g0, w0) and np.array_equal(g1, w1)
    ct = aoa.Ciphertext.from_residues(ctx, c0, c1, slots=N // 2)
    out = aoa.Ciphertext(ctx)
    aoa.ckks_conjugate_plain(ctx, out, ct, cjk)
    g0, g1 = out.download(nlimbs=k)
    assert np.array_equal(g0, w0) and np.array_equal(g1, w1)
    with pytest.raises(aoa.capi.AoaError):
        aoa.ckks_rotate_plain(ctx, out, ct, 1, None)              # no key


def test_add_sub_mixed_domains(ref_table):
    require_gpu()
    Q, B = _sets(ref_table)["ref55"]
    aoa, E, ctx, o = _setup(12, Q, B)
    rng = np.random.default_rng(2)
    N, k = E.N, E.k
    a = _rand_ct(rng, Q, N, k)
    b = _rand_ct(rng, Q, N, k)
    for sub in (False, True):
        ca = aoa.Ciphertext.from_residues(ctx, *a, domain=aoa.AOA_NTT)
        cb = aoa.Ciphertext.from_residues(ctx, *b, domain=aoa.AOA_COEF)
        out = aoa.Ciphertext(ctx)
        (aoa.ckks_sub if sub else aoa.ckks_add)(ctx, out, ca, cb)
        w0, w1, st = o.add(a, b, subtract=sub, a_state=ST_NTT, b_state=ST_COEF)
        assert st == ST_COEF and out.domain == aoa.AOA_COEF
        g0, g1 = out.download(nlimbs=k, domain=aoa.AOA_COEF)
        assert np.array_equal(g0, w0) and np.array_equal(g1, w1)


def test_error_statuses(ref_table):
    require_gpu()
    Q, B = _sets(ref_table)["p60"]
    aoa, E, ctx, o = _setup(12, Q, B)
    rng = np.random.default_rng(0)
    a = _rand_ct(rng, Q, E.N, E.k)
    ca = aoa.Ciphertext.from_residues(ctx, *a, slots=8)
    cb = aoa.Ciphertext.from_residues(ctx, *a, slots=16)
    out = aoa.Ciphertext(ctx)
    keys = make_keys(o, seed=1)
    evk = aoa.SwitchKey(ctx, *keys["evk"])
    with pytest.raises(aoa.AoaError) as ei:
        aoa.ckks_mul(ctx, out, ca, cb, evk)
    assert ei.value.name == "AOA_ERR_SLOT_MISMATCH"
    with pytest.raises(aoa.AoaError) as ei:
        aoa.ckks_mul(ctx, out, ca, ca, None)
    assert ei.value.name == "AOA_ERR_NO_KEY"
    ca.set(0, 8, 1 << 20, aoa.AOA_COEF)
    with pytest.raises(aoa.AoaError) as ei:
        aoa.ckks_mul(ctx, out, ca, ca, evk)
    assert ei.value.name == "AOA_ERR_LEVEL_EXHAUSTED"
    with pytest.raises(aoa.AoaError) as ei:
        aoa.ckks_rescale(ctx, ca)
    assert ei.value.name == "AOA_ERR_LEVEL_EXHAUSTED"
    with pytest.raises(aoa.AoaError) as ei:
        aoa.ckks_rotate_left(ctx, out, cb, 1, None)
    assert ei.value.name == "AOA_ERR_NO_KEY"


def test_encrypted_hmult_decodes_full_size():
    """N = 2^16, 30 x 60-bit Q primes, 31 special primes, scale 2^50: the
    decrypted product matches the FP64 cleartext product (size-independent
    property at the benchmark's full size)."""
    require_gpu()
    import aoa_b200 as aoa
    ps = oracle.gen_ntt_primes(60, 1 << 17, 61)
    Q, B = ps[:30], ps[30:]
    log_n = 16
    E = aoa.Engine(log_n, Q, B, scale_bits=50)
    ctx = aoa.Context(E)
    o = Oracle(1 << log_n, Q, B)
    keys = make_keys(o, seed=2)
    evk = aoa.SwitchKey(ctx, *keys["evk"])
    rng = np.random.default_rng(1)
    slots = 1 << 15
    r1, t1 = np.sqrt(rng.uniform(0, 1, slots)), rng.uniform(0, 2 * np.pi, slots)
    r2, t2 = np.sqrt(rng.uniform(0, 1, slots)), rng.uniform(0, 2 * np.pi, slots)
    v1, v2 = r1 * np.exp(1j * t1), r2 * np.exp(1j * t2)
    scale = 1 << 50
    c1 = encrypt_values(o, keys, v1, scale, seed=3)
    c2 = encrypt_values(o, keys, v2, scale, seed=4)
    g1 = aoa.Ciphertext.from_residues(ctx, *c1, slots=slots, scale=scale, domain=aoa.AOA_NTT)
    g2 = aoa.Ciphertext.from_residues(ctx, *c2, slots=slots, scale=scale, domain=aoa.AOA_NTT)
    out = aoa.Ciphertext(ctx)
    aoa.ckks_mul(ctx, out, g1, g2, evk)
    d0, d1 = out.download(nlimbs=out.level + 1)
    pad = lambda x: np.concatenate([x, np.zeros((30 - x.shape[0], 1 << log_n), dtype=np.uint64)])
    m = o.decrypt((pad(d0), pad(d1)), keys["s"][:30], state=ST_COEF)
    got = o.decode(m[0], slots, out.scale)
    err = np.abs(got - v1 * v2)
    assert err.max() < 2.0 ** -20, err.max()


@pytest.mark.parametrize("rescale", [True, False])
def test_hmult_batch_matches_single_calls(ref_table, rescale):
    """Grouped batched HMult (mixed levels, aliased outputs) equals per-call HMult and the oracle."""
    require_gpu()
    Q, B = _sets(ref_table)["p60"]
    aoa, E, ctx, o = _setup(12, Q, B)
    keys = make_keys(o, seed=17)
    evk = aoa.SwitchKey(ctx, *keys["evk"])
    rng = np.random.default_rng(11)
    N, k = E.N, E.k
    levels = [4, 2, 4, 3, 2, 4]
    pairs = [(_rand_ct(rng, Q, N, k), _rand_ct(rng, Q, N, k)) for _ in levels]
    cts_a, cts_b, outs = [], [], []
    for (a, b), lv in zip(pairs, levels):
        ca = aoa.Ciphertext.from_residues(ctx, *a, slots=8, scale=1 << 35, domain=aoa.AOA_NTT)
        cb = aoa.Ciphertext.from_residues(ctx, *b, slots=8, scale=1 << 36, domain=aoa.AOA_COEF)
        ca.set(lv, 8, 1 << 35, aoa.AOA_NTT)
        cb.set(lv, 8, 1 << 36, aoa.AOA_COEF)
        cts_a.append(ca)
        cts_b.append(cb)
    outs = [aoa.Ciphertext(ctx) for _ in levels]
    outs[1] = cts_a[1]                                   # output aliases an input
    aoa.ckks_mul_batch(ctx, outs, cts_a, cts_b, evk, rescale=rescale)
    for z, ((a, b), lv) in enumerate(zip(pairs, levels)):
        pad = lambda x: np.concatenate([x[: lv + 1], np.zeros((k - lv - 1, N), dtype=np.uint64)])
        w0, w1, wsc = o.hmult((pad(a[0]), pad(a[1])), (pad(b[0]), pad(b[1])), keys["evk"], lv, 1 << 35, 1 << 36,
                              rescale=rescale, a_state=ST_NTT, b_state=ST_COEF)
        nl = lv if rescale else lv + 1
        g0, g1 = outs[z].download(nlimbs=nl)
        assert outs[z].level == nl - 1 and outs[z].scale == wsc, z
        assert np.array_equal(g0, w0[:nl]) and np.array_equal(g1, w1[:nl]), z


def test_hmult_batch_full_size_equals_pipeline():
    """N = 2^16, 30 + 31 primes: batched and per-call pipeline residues agree."""
    require_gpu()
    import aoa_b200 as aoa
    ps = oracle.gen_ntt_primes(60, 1 << 17, 61)
    E = aoa.Engine(16, ps[:30], ps[30:])
    ctx = aoa.Context(E)
    rng = np.random.default_rng(4)
    N = E.N
    evk = aoa.SwitchKey(ctx, uniform_residues(rng, ps, N), uniform_residues(rng, ps, N))
    xs = [(_rand_ct(rng, ps, N, 30), _rand_ct(rng, ps, N, 30)) for _ in range(3)]
    A = [aoa.Ciphertext.from_residues(ctx, *x[0], slots=4, scale=1 << 50, domain=aoa.AOA_NTT) for x in xs]
    Bc = [aoa.Ciphertext.from_residues(ctx, *x[1], slots=4, scale=1 << 50, domain=aoa.AOA_NTT) for x in xs]
    outs = [aoa.Ciphertext(ctx) for _ in xs]
    aoa.ckks_mul_batch(ctx, outs, A, Bc, evk)
    for z, x in enumerate(xs):
        a1 = aoa.Ciphertext.from_residues(ctx, *x[0], slots=4, scale=1 << 50, domain=aoa.AOA_NTT)
        b1 = aoa.Ciphertext.from_residues(ctx, *x[1], slots=4, scale=1 << 50, domain=aoa.AOA_NTT)
        o1 = aoa.Ciphertext(ctx)
        aoa.ckks_mul(ctx, o1, a1, b1, evk)
        g = outs[z].download(nlimbs=29, domain=aoa.AOA_NTT)
        w = o1.download(nlimbs=29, domain=aoa.AOA_NTT)
        assert np.array_equal(g[0], w[0]) and np.array_equal(g[1], w[1])


@pytest.mark.parametrize("log_n", [10, 12])
@pytest.mark.parametrize("fuse", [1, 2, 4, 7])
@pytest.mark.parametrize("pset", ["p60", "ref55"])
def test_fused_transform_ends_equal_separate_kernels(ref_table, log_n, fuse, pset):
    """Key products, key-switch combine and out-of-place inverses fused into the
    transforms give the same residues as the separate kernels and the oracle;
    on the reference's set (63-bit q0, 55-bit rest) the transforms run as a
    strict run (q0) and a lazy run, each with its source and epilogue offset."""
    require_gpu()
    Q, B = _sets(ref_table)[pset]
    aoa, E, ctx, o = _setup(log_n, Q, B)
    keys = make_keys(o, seed=5, rotations=(3,))
    evk = aoa.SwitchKey(ctx, *keys["evk"])
    rtk = aoa.SwitchKey(ctx, *keys["rtk"][3])
    rng = np.random.default_rng(2)
    N, k = E.N, E.k
    a, b = _rand_ct(rng, Q, N, k), _rand_ct(rng, Q, N, k)

    def run():
        ca = aoa.Ciphertext.from_residues(ctx, *a, slots=N // 2, scale=1 << 35)
        cb = aoa.Ciphertext.from_residues(ctx, *b, slots=N // 2, scale=1 << 35)
        res = []
        for rescale in (True, False):
            ca.set(k - 1, N // 2, 1 << 35, ca.domain)
            cb.set(k - 1, N // 2, 1 << 35, cb.domain)
            o1 = aoa.Ciphertext(ctx)
            (aoa.ckks_mul if rescale else aoa.ckks_mul_without_rescale)(ctx, o1, ca, cb, evk)
            res.append(o1.download(nlimbs=o1.level + 1, domain=aoa.AOA_COEF))
        outs = [aoa.Ciphertext(ctx), aoa.Ciphertext(ctx)]
        ca.set(k - 1, N // 2, 1 << 35, ca.domain)
        cb.set(k - 1, N // 2, 1 << 35, cb.domain)
        aoa.ckks_mul_batch(ctx, outs, [ca, cb], [cb, ca], evk)
        res += [x.download(nlimbs=x.level + 1, domain=aoa.AOA_COEF) for x in outs]
        ca.set(k - 1, N // 2, 1 << 35, ca.domain)
        r = aoa.Ciphertext(ctx)
        aoa.ckks_rotate_left(ctx, r, ca, 3, rtk)
        res.append(r.download(nlimbs=k, domain=aoa.AOA_COEF))
        return res

    E.tune("fuse", fuse)
    fused = run()
    E.tune("fuse", 0)
    separate = run()
    for f, s in zip(fused, separate):
        assert np.array_equal(f[0], s[0]) and np.array_equal(f[1], s[1])
    w0, w1, _ = o.hmult(a, b, keys["evk"], k - 1, 1 << 35, 1 << 35, rescale=True, a_state=ST_COEF, b_state=ST_COEF)
    assert np.array_equal(fused[0][0], w0[:k - 1]) and np.array_equal(fused[0][1], w1[:k - 1])
    r0, r1 = o.rotate_left(a, 3, keys["rtk"][3], k - 1, state=ST_COEF)
    assert np.array_equal(fused[4][0], r0) and np.array_equal(fused[4][1], r1)


def test_hmult_batch_two_streams_equal_one_stream(ref_table):
    """A large batch split over the context's two streams (halves forked and
    joined by events) gives the residues of the single-stream batch, with an
    output aliasing an operand inside a half and across halves."""
    require_gpu()
    Q, B = _sets(ref_table)["p60"]
    aoa, E, ctx, o = _setup(12, Q, B)
    keys = make_keys(o, seed=19)
    evk = aoa.SwitchKey(ctx, *keys["evk"])
    rng = np.random.default_rng(12)
    N, k = E.N, E.k
    data = [(_rand_ct(rng, Q, N, k), _rand_ct(rng, Q, N, k)) for _ in range(12)]

    def run(streams, cross):
        E.tune("batch_streams", streams)
        A = [aoa.Ciphertext.from_residues(ctx, *x[0], slots=8, scale=1 << 35, domain=aoa.AOA_NTT) for x in data]
        Bc = [aoa.Ciphertext.from_residues(ctx, *x[1], slots=8, scale=1 << 36, domain=aoa.AOA_NTT) for x in data]
        outs = [aoa.Ciphertext(ctx) for _ in data]
        outs[2] = A[2]                                   # aliasing inside a half
        if cross:
            outs[1] = Bc[9]                              # an output is an operand of the other half
        aoa.ckks_mul_batch(ctx, outs, A, Bc, evk)
        return [x.download(nlimbs=k - 1, domain=aoa.AOA_COEF) for x in outs]

    for cross in (False, True):
        one, two = run(1, cross), run(2, cross)
        for x, y in zip(one, two):
            assert np.array_equal(x[0], y[0]) and np.array_equal(x[1], y[1])


@pytest.mark.parametrize("count", [5, 12])
def test_rotate_batch_equals_single_rotations(ref_table, count):
    """Batched rotations (one key, mixed levels, an output aliasing its input;
    12 ops take the two-stream split) give the per-call residues, and the
    oracle's for one op."""
    require_gpu()
    Q, B = _sets(ref_table)["p60"]
    aoa, E, ctx, o = _setup(12, Q, B)
    keys = make_keys(o, seed=14, rotations=(3,), conjugation=True)
    rtk = aoa.SwitchKey(ctx, *keys["rtk"][3])
    cjk = aoa.SwitchKey(ctx, *keys["cjk"])
    rng = np.random.default_rng(15)
    N, k = E.N, E.k
    data = [_rand_ct(rng, Q, N, k) for _ in range(count)]
    levels = [k - 1 - (z % 3) for z in range(count)]

    def make():
        cts = []
        for x, lv in zip(data, levels):
            c = aoa.Ciphertext.from_residues(ctx, *x, slots=N // 2, scale=1 << 40,
                                             domain=aoa.AOA_NTT if lv % 2 else aoa.AOA_COEF)
            c.set(lv, N // 2, 1 << 40, c.domain)
            cts.append(c)
        return cts

    for batch_fn, single_fn, key in ((lambda o_, c_: aoa.ckks_rotate_batch(ctx, o_, c_, 3, rtk),
                                      lambda o_, c_: aoa.ckks_rotate_left(ctx, o_, c_, 3, rtk), rtk),
                                     (lambda o_, c_: aoa.ckks_conjugate_batch(ctx, o_, c_, cjk),
                                      lambda o_, c_: aoa.ckks_conjugate(ctx, o_, c_, cjk), cjk)):
        cts = make()
        outs = [aoa.Ciphertext(ctx) for _ in cts]
        outs[0] = cts[0]                                   # in place
        batch_fn(outs, cts)
        got = [x.download(nlimbs=x.level + 1, domain=aoa.AOA_COEF) for x in outs]
        ref = make()
        for z, (c, lv) in enumerate(zip(ref, levels)):
            w = aoa.Ciphertext(ctx)
            single_fn(w, c)
            assert outs[z].level == lv == w.level
            want = w.download(nlimbs=lv + 1, domain=aoa.AOA_COEF)
            assert np.array_equal(got[z][0], want[0]) and np.array_equal(got[z][1], want[1]), z
    # op 0 is at level k - 1 in coefficients: the oracle's rotation of the same residues
    w0, w1 = o.rotate_left(data[0], 3, keys["rtk"][3], k - 1, state=ST_COEF)
    cts = make()
    outs = [aoa.Ciphertext(ctx) for _ in cts]
    aoa.ckks_rotate_batch(ctx, outs, cts, 3, rtk)
    g0, g1 = outs[0].download(nlimbs=k, domain=aoa.AOA_COEF)
    assert np.array_equal(g0, w0) and np.array_equal(g1, w1)


@pytest.mark.parametrize("count", [7, 20])
def test_rotate_batch_steps_equals_single_rotations(ref_table, count):
    """Rotations with a step and key per op in one batched call (grouped by
    level only: ops of different steps and keys share the launches; a right
    rotation; an output aliasing its input; 20 ops take the two-stream split)
    give the per-call residues, and the oracle's for two ops."""
    require_gpu()
    Q, B = _sets(ref_table)["p60"]
    aoa, E, ctx, o = _setup(12, Q, B)
    N, k = E.N, E.k
    rots = (1, 2, 4, 64, N // 2 - 3)
    keys = make_keys(o, seed=24, rotations=rots)
    rtk = {r: aoa.SwitchKey(ctx, *keys["rtk"][r]) for r in rots}
    rng = np.random.default_rng(25)
    data = [_rand_ct(rng, Q, N, k) for _ in range(count)]
    levels = [k - 1 - (z % 3) for z in range(count)]
    steps = [rots[z % len(rots)] for z in range(count)]
    steps[1] = -3                                          # right by 3 = left by N/2 - 3

    def make():
        cts = []
        for x, lv in zip(data, levels):
            c = aoa.Ciphertext.from_residues(ctx, *x, slots=N // 2, scale=1 << 40,
                                             domain=aoa.AOA_NTT if lv % 2 else aoa.AOA_COEF)
            c.set(lv, N // 2, 1 << 40, c.domain)
            cts.append(c)
        return cts

    key_of = lambda s: rtk[s if s > 0 else N // 2 + s]
    cts = make()
    outs = [aoa.Ciphertext(ctx) for _ in cts]
    outs[2] = cts[2]                                       # in place
    aoa.ckks_rotate_batch_steps(ctx, outs, cts, steps, [key_of(s) for s in steps])
    got = [x.download(nlimbs=x.level + 1, domain=aoa.AOA_COEF) for x in outs]
    ref = make()
    for z, (c, lv) in enumerate(zip(ref, levels)):
        w = aoa.Ciphertext(ctx)
        aoa.ckks_rotate_left(ctx, w, c, steps[z], key_of(steps[z]))
        assert outs[z].level == lv == w.level
        want = w.download(nlimbs=lv + 1, domain=aoa.AOA_COEF)
        assert np.array_equal(got[z][0], want[0]) and np.array_equal(got[z][1], want[1]), z
    for z in (0, 1):                                       # level k - 1 ops in coefficients
        if levels[z] != k - 1 or z % 2:
            continue
        r = steps[z] if steps[z] > 0 else N // 2 + steps[z]
        w0, w1 = o.rotate_left(data[z], r, keys["rtk"][r], k - 1, state=ST_COEF)
        assert np.array_equal(got[z][0], w0) and np.array_equal(got[z][1], w1), z
    with pytest.raises(aoa.capi.AoaError):                  # a missing key is refused
        aoa.ckks_rotate_batch_steps(ctx, outs[:2], make()[:2], steps[:2], [rtk[1], None])


def test_tensor_core_and_cuda_core_conversions_agree(ref_table):
    """The int8 tensor-core basis conversion and the CUDA-core kernel give the
    same residues (ModUp, ModDown and the merged ModDown + rescale of HMult)."""
    require_gpu()
    Q, B = _sets(ref_table)["p60"]
    aoa, E, ctx, o = _setup(12, Q, B)
    keys = make_keys(o, seed=23)
    evk = aoa.SwitchKey(ctx, *keys["evk"])
    rng = np.random.default_rng(24)
    N, k = E.N, E.k
    a, b = _rand_ct(rng, Q, N, k), _rand_ct(rng, Q, N, k)
    res = []
    for tc in (1, 0):
        E.tune("conv_tensor_cores", tc)
        outs = []
        for rescale in (True, False):
            ca = aoa.Ciphertext.from_residues(ctx, *a, slots=8, scale=1 << 35)
            cb = aoa.Ciphertext.from_residues(ctx, *b, slots=8, scale=1 << 35)
            o1 = aoa.Ciphertext(ctx)
            (aoa.ckks_mul if rescale else aoa.ckks_mul_without_rescale)(ctx, o1, ca, cb, evk)
            outs.append(o1.download(nlimbs=o1.level + 1))
        res.append(outs)
    for x, y in zip(res[0], res[1]):
        assert np.array_equal(x[0], y[0]) and np.array_equal(x[1], y[1])


@pytest.mark.parametrize("bits", [33, 34, 40, 60, 61, 62])
def test_hmult_prime_sizes_bit_exact(bits):
    """Per-call and batched HMult + relinearise + rescale at prime sizes on
    both sides of every arithmetic switch: Montgomery products below 2^33,
    Barrett from 2^33 (funnel-shift quotient), the one-reduction cross term up
    to 61 bits, two reductions at 62 bits, lazy transforms below 2^60."""
    require_gpu()
    ps = oracle.gen_ntt_primes(bits, 1 << 13, 11)
    Q, B = ps[:5], ps[5:]
    aoa, E, ctx, o = _setup(12, Q, B)
    keys = make_keys(o, seed=bits)
    evk = aoa.SwitchKey(ctx, *keys["evk"])
    rng = np.random.default_rng(bits)
    N, k = E.N, E.k
    pairs = [(_rand_ct(rng, Q, N, k), _rand_ct(rng, Q, N, k)) for _ in range(3)]
    # all-(q - 1) residues for the first pair: the largest products
    full = tuple(np.array([[q - 1] * N for q in Q], dtype=np.uint64) for _ in range(2))
    pairs[0] = (full, full)
    sa, sb = 1 << 30, 1 << 31
    cts = [(aoa.Ciphertext.from_residues(ctx, *a, slots=8, scale=sa, domain=aoa.AOA_NTT),
            aoa.Ciphertext.from_residues(ctx, *b, slots=8, scale=sb, domain=aoa.AOA_NTT)) for a, b in pairs]
    outs = [aoa.Ciphertext(ctx) for _ in pairs]
    aoa.ckks_mul_batch(ctx, outs, [c[0] for c in cts], [c[1] for c in cts], evk)
    single = aoa.Ciphertext(ctx)
    aoa.ckks_mul(ctx, single, cts[1][0], cts[1][1], evk)
    for z, (a, b) in enumerate(pairs):
        w0, w1, _ = o.hmult(a, b, keys["evk"], k - 1, sa, sb, rescale=True, a_state=ST_NTT, b_state=ST_NTT)
        g0, g1 = outs[z].download(nlimbs=k - 1)
        assert np.array_equal(g0, w0[:k - 1]) and np.array_equal(g1, w1[:k - 1]), z
        if z == 1:
            s0, s1 = single.download(nlimbs=k - 1)
            assert np.array_equal(s0, w0[:k - 1]) and np.array_equal(s1, w1[:k - 1])
