"""Bit-exact parity at the benchmarked configuration, through the C ABI.

The benchmark runs HMult + relinearise + rescale at N = 2^16 with 30 Q primes
and 31 special primes of 60 bits (q = 1 mod 2^32, a subset of the primes
q = 1 mod 2N; the tests also run the largest primes q = 1 mod 2^17), dnum = 1 (the reference's
ckks_mul, aoa-ntt src/ckks/ckks.cpp:273-347, with the conversions of
src/cuda/manager.cu:180-223 and 312-341).  There the tensor-core basis
conversion runs its full shapes: ModUp 30 -> 31 (8 K-steps of the int8 GEMM),
ModDown and the merged ModDown + rescale 31 -> 29/30.  Every live residue of
every output below must equal the CPU oracle's.

Besides uniform residues, inputs are crafted so that the conversion's scaled
inputs z_i = [x_i (P/p_i)^-1]_{p_i} are all p_i - 1: the byte sums of the
tensor-core product are then at their largest for the given table.
"""
import numpy as np
import pytest

import oracle
from oracle import Oracle, ST_COEF, ST_NTT
from tests.ckks_inputs import make_keys, uniform_residues
from tests.gpu_util import require_gpu

pytestmark = pytest.mark.gpu

LOG_N, K, KL = 16, 30, 31
# the two 60-bit prime families: the largest q = 1 mod 2^17, and the largest
# q = 1 mod 2^32 (the benchmark's set), whose transforms take the shorter Shoup
# remainder
FAMILIES = (1 << 17, 1 << 32)


def _primes(count=K + KL, modulus=1 << 17):
    return oracle.gen_ntt_primes(60, modulus, count)


@pytest.fixture(scope="module", params=FAMILIES, ids=["q=1 mod 2^17", "q=1 mod 2^32"])
def full(request):
    require_gpu()
    import aoa_b200 as aoa
    ps = _primes(modulus=request.param)
    Q, B = ps[:K], ps[K:]
    E = aoa.Engine(LOG_N, Q, B, scale_bits=50)
    ctx = aoa.Context(E)
    o = Oracle(1 << LOG_N, Q, B)
    keys = make_keys(o, seed=40, rotations=(1, 1 << 12))
    evk = aoa.SwitchKey(ctx, *keys["evk"])
    return {"aoa": aoa, "E": E, "ctx": ctx, "o": o, "keys": keys, "evk": evk, "Q": Q, "B": B}


def _max_z_inputs(primes, level_primes, N):
    """x_i with [x_i (P/p_i)^-1]_{p_i} = p_i - 1, P the product of `level_primes`."""
    P = 1
    for p in level_primes:
        P *= p
    rows = []
    for p in primes:
        c = pow((P // p) % p, -1, p)
        x = (p - 1) * pow(c, -1, p) % p
        rows.append(np.full(N, x, dtype=np.uint64))
    return np.array(rows, dtype=np.uint64)


def _extend(live, rng, Q, level, N):
    """Live limbs 0..level, uniform residues in the stale limbs above."""
    if level + 1 >= len(Q):
        return live
    return np.concatenate([live, uniform_residues(rng, Q[level + 1:], N)])


def _inputs(kind, rng, primes, level_primes, N):
    if kind == "uniform":
        return uniform_residues(rng, primes, N)
    if kind == "all_q_minus_1":
        return np.array([np.full(N, p - 1, dtype=np.uint64) for p in primes])
    return _max_z_inputs(primes, level_primes, N)


@pytest.mark.parametrize("kind", ["uniform", "all_q_minus_1", "max_z"])
@pytest.mark.parametrize("level", [29, 3])
def test_modup_full_size(full, level, kind):
    aoa, ctx, o, Q = full["aoa"], full["ctx"], full["o"], full["Q"]
    N = 1 << LOG_N
    rng = np.random.default_rng(100 + level)
    live = _inputs(kind, rng, Q[: level + 1], Q[: level + 1], N)
    xq = _extend(live, rng, Q, level, N)
    dq = ctx.upload(xq)
    out_b = ctx.alloc((KL, N))
    aoa.capi.check(aoa.capi.load().aoa_modup(ctx.handle, dq.ptr, out_b.ptr, level))
    want = o.modup(xq, level)
    assert np.array_equal(out_b.numpy(), want)


@pytest.mark.parametrize("kind", ["uniform", "all_q_minus_1", "max_z"])
@pytest.mark.parametrize("level", [29, 3])
def test_moddown_full_size(full, level, kind):
    aoa, ctx, o, Q, B = full["aoa"], full["ctx"], full["o"], full["Q"], full["B"]
    N = 1 << LOG_N
    rng = np.random.default_rng(200 + level)
    xq = uniform_residues(rng, Q, N)
    xb = _inputs(kind, rng, B, B, N)
    xqb = np.concatenate([xq, xb])
    d = ctx.upload(xqb)
    out_q = ctx.alloc((K, N))
    aoa.capi.check(aoa.capi.load().aoa_moddown(ctx.handle, d.ptr, out_q.ptr, level))
    want = o.moddown(xqb, level)
    assert np.array_equal(out_q.numpy()[: level + 1], want[: level + 1])


def _ct(rng, Q, N):
    return uniform_residues(rng, Q, N), uniform_residues(rng, Q, N)


def _pad(x, level, N):
    return np.concatenate([x[: level + 1], np.zeros((K - level - 1, N), dtype=np.uint64)])


@pytest.mark.parametrize("in_domain,level", [("coef", 29), ("ntt", 29), ("ntt", 6)])
def test_hmult_full_size_bit_exact(full, in_domain, level):
    """Per-call ckks_mul (HMult + relinearise + rescale) at N = 2^16, k = 30, kl = 31."""
    aoa, ctx, o, keys, evk, Q = full["aoa"], full["ctx"], full["o"], full["keys"], full["evk"], full["Q"]
    N = 1 << LOG_N
    rng = np.random.default_rng(300 + level)
    a, b = _ct(rng, Q, N), _ct(rng, Q, N)
    dom = aoa.AOA_COEF if in_domain == "coef" else aoa.AOA_NTT
    st = ST_COEF if in_domain == "coef" else ST_NTT
    sa, sb = 1 << 50, (1 << 50) + 777
    ca = aoa.Ciphertext.from_residues(ctx, *a, slots=N // 2, scale=sa, domain=dom)
    cb = aoa.Ciphertext.from_residues(ctx, *b, slots=N // 2, scale=sb, domain=dom)
    ca.set(level, N // 2, sa, dom)
    cb.set(level, N // 2, sb, dom)
    out = aoa.Ciphertext(ctx)
    aoa.ckks_mul(ctx, out, ca, cb, evk)
    A = [_pad(v, level, N) for v in a]
    Bc = [_pad(v, level, N) for v in b]
    w0, w1, wsc = o.hmult(A, Bc, keys["evk"], level, sa, sb, rescale=True, a_state=st, b_state=st)
    g0, g1 = out.download(nlimbs=level)
    assert out.level == level - 1 and out.scale == wsc
    assert np.array_equal(g0, w0[:level]) and np.array_equal(g1, w1[:level])


def test_hmult_batch_16_full_size_bit_exact(full):
    """ckks_mul_batch of 16 products at level 29 in the transform domain (the
    benchmark's step; the batch runs as two halves on the context's two
    streams), every product against the oracle."""
    aoa, ctx, o, keys, evk, Q = full["aoa"], full["ctx"], full["o"], full["keys"], full["evk"], full["Q"]
    N = 1 << LOG_N
    rng = np.random.default_rng(400)
    sc = 1 << 50
    pairs = [(_ct(rng, Q, N), _ct(rng, Q, N)) for _ in range(16)]
    A = [aoa.Ciphertext.from_residues(ctx, *p[0], slots=N // 2, scale=sc, domain=aoa.AOA_NTT) for p in pairs]
    Bc = [aoa.Ciphertext.from_residues(ctx, *p[1], slots=N // 2, scale=sc, domain=aoa.AOA_NTT) for p in pairs]
    outs = [aoa.Ciphertext(ctx) for _ in pairs]
    assert full["E"].tune_get("batch_streams") == 2
    aoa.ckks_mul_batch(ctx, outs, A, Bc, evk)
    got = [x.download(nlimbs=K - 1) for x in outs]
    for z, (a, b) in enumerate(pairs):
        w0, w1, wsc = o.hmult(a, b, keys["evk"], K - 1, sc, sc, rescale=True, a_state=ST_NTT, b_state=ST_NTT)
        assert outs[z].level == K - 2 and outs[z].scale == wsc, z
        assert np.array_equal(got[z][0], w0[: K - 1]) and np.array_equal(got[z][1], w1[: K - 1]), z


@pytest.mark.parametrize("r", [1, 1 << 12])
def test_rotate_full_size_bit_exact(full, r):
    aoa, ctx, o, keys, Q = full["aoa"], full["ctx"], full["o"], full["keys"], full["Q"]
    N = 1 << LOG_N
    rng = np.random.default_rng(500 + r)
    c = _ct(rng, Q, N)
    rtk = aoa.SwitchKey(ctx, *keys["rtk"][r])
    ct = aoa.Ciphertext.from_residues(ctx, *c, slots=N // 2)
    out = aoa.Ciphertext(ctx)
    aoa.ckks_rotate_left(ctx, out, ct, r, rtk)
    w0, w1 = o.rotate_left(c, r, keys["rtk"][r], K - 1, state=ST_COEF)
    g0, g1 = out.download(nlimbs=K)
    assert np.array_equal(g0, w0) and np.array_equal(g1, w1)


@pytest.mark.parametrize("modulus", FAMILIES, ids=["q=1 mod 2^17", "q=1 mod 2^32"])
@pytest.mark.parametrize("kind", ["all_q_minus_1", "max_z"])
def test_conversion_32_inputs(kind, modulus):
    """The tensor-core conversion at its own maximum of 32 inputs and 32
    outputs (32 Q + 32 special primes at N = 2^12): ModUp at level 31 and
    ModDown, against the oracle and against the CUDA-core kernel."""
    require_gpu()
    import aoa_b200 as aoa
    ps = _primes(64, modulus)
    Q, B = ps[:32], ps[32:]
    E = aoa.Engine(12, Q, B)
    ctx = aoa.Context(E)
    o = Oracle(1 << 12, Q, B)
    N = 1 << 12
    rng = np.random.default_rng(7)
    xq = _inputs(kind, rng, Q, Q, N)
    xb = _inputs(kind, rng, B, B, N)
    xqb = np.concatenate([xq, xb])
    want_up, want_down = o.modup(xq, 31), o.moddown(xqb, 31)
    lib = aoa.capi.load()
    for tc in (1, 0):
        E.tune("conv_tensor_cores", tc)
        dq, dqb = ctx.upload(xq), ctx.upload(xqb)
        up, down = ctx.alloc((32, N)), ctx.alloc((32, N))
        aoa.capi.check(lib.aoa_modup(ctx.handle, dq.ptr, up.ptr, 31))
        aoa.capi.check(lib.aoa_moddown(ctx.handle, dqb.ptr, down.ptr, 31))
        assert np.array_equal(up.numpy(), want_up), tc
        assert np.array_equal(down.numpy(), want_down), tc


@pytest.mark.parametrize("modulus", FAMILIES, ids=["q=1 mod 2^17", "q=1 mod 2^32"])
@pytest.mark.parametrize("level", [29, 17, 8, 2])
def test_conversion_kernels_agree_at_benchmark_shapes(level, modulus):
    """30 Q + 31 special 60-bit primes at N = 2^12 (the benchmark's conversion
    shapes on a small ring): ModUp, ModDown and HMult with its merged ModDown +
    rescale, tensor-core kernel vs CUDA-core kernel vs oracle, with all-(q-1)
    inputs (ciphertexts and conversion inputs) and max-z conversion inputs."""
    require_gpu()
    import aoa_b200 as aoa
    ps = _primes(modulus=modulus)
    Q, B = ps[:K], ps[K:]
    E = aoa.Engine(12, Q, B)
    ctx = aoa.Context(E)
    o = Oracle(1 << 12, Q, B)
    N = 1 << 12
    keys = make_keys(o, seed=41)
    evk = aoa.SwitchKey(ctx, *keys["evk"])
    rng = np.random.default_rng(level)
    lib = aoa.capi.load()
    full_ct = tuple(np.array([np.full(N, q - 1, dtype=np.uint64) for q in Q]) for _ in range(2))
    cases = [(full_ct, full_ct), (_ct(rng, Q, N), full_ct)]
    conv_in = [(_inputs("max_z", rng, Q[: level + 1], Q[: level + 1], N), _inputs("max_z", rng, B, B, N)),
               (_inputs("all_q_minus_1", rng, Q[: level + 1], None, N), _inputs("all_q_minus_1", rng, B, None, N))]
    res = {}
    for tc in (1, 0):
        E.tune("conv_tensor_cores", tc)
        outs = []
        for live_q, xb in conv_in:
            xq = _extend(live_q, np.random.default_rng(1), Q, level, N)
            xqb = np.concatenate([xq, xb])
            up, down = ctx.alloc((KL, N)), ctx.alloc((K, N))
            aoa.capi.check(lib.aoa_modup(ctx.handle, ctx.upload(xq).ptr, up.ptr, level))
            aoa.capi.check(lib.aoa_moddown(ctx.handle, ctx.upload(xqb).ptr, down.ptr, level))
            outs.append(up.numpy())
            outs.append(down.numpy()[: level + 1])
            if tc == 1:
                assert np.array_equal(outs[-2], o.modup(xq, level))
                assert np.array_equal(outs[-1], o.moddown(xqb, level)[: level + 1])
        for a, b in cases:
            ca = aoa.Ciphertext.from_residues(ctx, *a, slots=8, scale=1 << 40)
            cb = aoa.Ciphertext.from_residues(ctx, *b, slots=8, scale=1 << 40)
            ca.set(level, 8, 1 << 40, aoa.AOA_COEF)
            cb.set(level, 8, 1 << 40, aoa.AOA_COEF)
            out = aoa.Ciphertext(ctx)
            aoa.ckks_mul(ctx, out, ca, cb, evk)
            g = out.download(nlimbs=level, domain=aoa.AOA_COEF)
            outs += [g[0], g[1]]
            if tc == 1:
                A = [_pad(v, level, N) for v in a]
                Bc = [_pad(v, level, N) for v in b]
                w0, w1, _ = o.hmult(A, Bc, keys["evk"], level, 1 << 40, 1 << 40, rescale=True)
                assert np.array_equal(g[0], w0[:level]) and np.array_equal(g[1], w1[:level])
        res[tc] = outs
    for x, y in zip(res[1], res[0]):
        assert np.array_equal(x, y)
