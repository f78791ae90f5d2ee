"""Compositions (aoa-ntt src/ckks/ckks.cpp:423-455 inner products, 732-761
power, 778-796 Horner polynomial evaluation, 813-906 Maclaurin functions) on
the GPU: residues equal the reference's operation sequence run step by step
through the oracle, metadata follows its rules, and encrypted evaluations
decode to the FP64 polynomial values."""
import numpy as np
import pytest

import oracle
from oracle import Oracle, ST_COEF
from tests.ckks_inputs import make_keys, uniform_residues, ternary_hw, gaussian
from tests.gpu_util import require_gpu

pytestmark = pytest.mark.gpu


def _setup(log_n=12, k=6, kl=4, scale_bits=40):
    import aoa_b200
    ps = oracle.gen_ntt_primes(60, 2 << log_n, k + kl)
    E = aoa_b200.Engine(log_n, ps[:k], ps[k:], scale_bits=scale_bits)
    return aoa_b200, E, aoa_b200.Context(E), Oracle(1 << log_n, ps[:k], ps[k:])


def _pad(x, lv, k):
    return np.concatenate([x[: lv + 1], np.zeros((k - lv - 1, x.shape[1]), dtype=np.uint64)])


def _o_add_const(o, ct, val, scale, lv):
    """ckks_add(ct, double) on coefficient residues (ckks.cpp:512-530)."""
    c0, c1 = ct[0].copy(), ct[1]
    cnst = int(abs(val) * scale)
    for i in range(lv + 1):
        q = o.primes[i]
        c0[i, 0] = (int(c0[i, 0]) + (cnst if val >= 0 else -cnst)) % q
    return c0, c1


def _o_mul(o, keys, a, b, la, lb, sa, sb):
    lv = min(la, lb)
    k = o.k
    r0, r1, sc = o.hmult((_pad(a[0], lv, k), _pad(a[1], lv, k)), (_pad(b[0], lv, k), _pad(b[1], lv, k)),
                         keys["evk"], lv, sa, sb, rescale=True, a_state=ST_COEF, b_state=ST_COEF)
    return (r0, r1), lv - 1, sc


def test_eval_polynomial_follows_horner_sequence():
    require_gpu()
    aoa, E, ctx, o = _setup()
    keys = make_keys(o, seed=3)
    evk = aoa.SwitchKey(ctx, *keys["evk"])
    rng = np.random.default_rng(5)
    N, k = E.N, E.k
    x = (uniform_residues(rng, E.q_primes, N), uniform_residues(rng, E.q_primes, N))
    ct = aoa.Ciphertext.from_residues(ctx, *x, slots=N // 2, scale=1 << 40)
    coeffs = [0.5, -0.25, 0.125]
    out = aoa.Ciphertext(ctx)
    aoa.ckks_eval_polynomial(ctx, out, ct, coeffs, evk)
    # the reference sequence on the oracle: r = 0 (level k-1, scale 2^40); r = r*x, r += c_i
    r = (np.zeros((k, N), np.uint64), np.zeros((k, N), np.uint64))
    lr, sr = k - 1, 1 << 40
    for c in reversed(coeffs):
        r, lr, sr = _o_mul(o, keys, r, x, lr, k - 1, sr, 1 << 40)
        r = _o_add_const(o, r, c, sr, lr)
    assert out.level == lr and out.scale == sr and out.slots == N // 2
    g0, g1 = out.download(nlimbs=lr + 1, domain=aoa.AOA_COEF)
    assert np.array_equal(g0, r[0][: lr + 1]) and np.array_equal(g1, r[1][: lr + 1])


def test_power_and_inner_products_follow_reference_sequence():
    require_gpu()
    aoa, E, ctx, o = _setup()
    keys = make_keys(o, seed=4)
    evk = aoa.SwitchKey(ctx, *keys["evk"])
    rng = np.random.default_rng(6)
    N, k = E.N, E.k
    xs = [(uniform_residues(rng, E.q_primes, N), uniform_residues(rng, E.q_primes, N)) for _ in range(3)]
    cts = [aoa.Ciphertext.from_residues(ctx, *x, slots=64, scale=1 << 40) for x in xs]
    # power x = 5 = 101b: out = 0 + x, then out = out * x^4; the running square is squared 3 times
    out = aoa.Ciphertext(ctx)
    aoa.ckks_power(ctx, out, cts[0], 5, evk)
    sq, lsq, ssq = xs[0], k - 1, 1 << 40
    acc = None
    for bit in (1, 0, 1):
        if bit:
            if acc is None:
                acc, la, sa = sq, lsq, 1 << 40            # ckks_add keeps the cleared accumulator's scale
            else:
                acc, la, sa = _o_mul(o, keys, acc, sq, la, lsq, sa, ssq)
        sq, lsq, ssq = _o_mul(o, keys, sq, sq, lsq, lsq, ssq, ssq)
    assert out.level == la and out.scale == sa
    g0, g1 = out.download(nlimbs=la + 1, domain=aoa.AOA_COEF)
    assert np.array_equal(g0, acc[0][: la + 1]) and np.array_equal(g1, acc[1][: la + 1])
    # inner product of ciphertext pairs: sum of products without rescale, one rescale, scale 2^40
    ip = aoa.Ciphertext(ctx)
    aoa.ckks_inner_prod(ctx, ip, cts[:2], [cts[2], cts[1]], evk)
    w = [np.zeros((k, N), np.uint64), np.zeros((k, N), np.uint64)]
    for a, b in ((xs[0], xs[2]), (xs[1], xs[1])):
        r0, r1, _ = o.hmult(a, b, keys["evk"], k - 1, 1 << 40, 1 << 40, rescale=False, a_state=ST_COEF,
                            b_state=ST_COEF)
        w = [np.array([[(int(p) + int(q_)) % q for p, q_ in zip(w[j][i], (r0, r1)[j][i])]
                       for i, q in enumerate(E.q_primes)], dtype=np.uint64) for j in (0, 1)]
    w0, w1 = o.rescale(w[0], w[1], k - 1)
    assert ip.level == k - 2 and ip.scale == 1 << 40
    g0, g1 = ip.download(nlimbs=k - 1, domain=aoa.AOA_COEF)
    assert np.array_equal(g0, w0[: k - 1]) and np.array_equal(g1, w1[: k - 1])
    # with real weights: each product is a constant multiply without rescale
    ipc = aoa.Ciphertext(ctx)
    aoa.ckks_inner_prod(ctx, ipc, cts[:2], [0.5, -2.0])
    parts = []
    for z, wv in zip(cts[:2], (0.5, -2.0)):
        t = aoa.Ciphertext(ctx)
        z.set(k - 1, 64, 1 << 40, z.domain)
        aoa.ckks_mul_const(ctx, t, z, wv, rescale=False)
        parts.append(t)
    acc_ct = aoa.Ciphertext(ctx)
    aoa.ckks_add(ctx, acc_ct, parts[0], parts[1])
    aoa.ckks_rescale(ctx, acc_ct)
    want = acc_ct.download(nlimbs=k - 1, domain=aoa.AOA_COEF)
    got = ipc.download(nlimbs=k - 1, domain=aoa.AOA_COEF)
    assert np.array_equal(got[0], want[0]) and np.array_equal(got[1], want[1])


@pytest.mark.parametrize("fn", ["sigmoid", "exp"])
def test_encrypted_function_approximations_decode(fn):
    """Keys and encryptions on the GPU; 50-bit primes track the 2^50 scale so
    the Horner chain keeps its precision over 8-11 products."""
    require_gpu()
    import aoa_b200 as aoa
    from aoa_b200 import params
    log_n = 13
    q0 = params.ntt_primes(60, 2 << log_n, 1)
    qs = params.ntt_primes(50, 2 << log_n, 12)
    bs = params.ntt_primes(61, 2 << log_n, 14)
    Q, B = q0 + qs, bs
    E = aoa.Engine(log_n, Q, B, scale_bits=50)
    ctx = aoa.Context(E)
    rng = np.random.default_rng(8)
    N = E.N
    primes = Q + B
    s_int = ternary_hw(rng, N)
    s = ctx.upload(np.array([(s_int % q).astype(np.uint64) for q in primes]))
    unif = lambda: np.array([rng.integers(0, q, N, dtype=np.uint64) for q in primes])
    draws = {"pk": (ctx.upload(unif()), ctx.upload(gaussian(rng, N))),
             "evk": (ctx.upload(unif()), ctx.upload(gaussian(rng, N)))}
    keys = aoa.ckks_keygen(ctx, s, draws)
    vals = rng.uniform(-0.5, 0.5, N // 2)
    ct = aoa.ckks_encrypt(ctx, vals, keys["pk"], rng.integers(-1, 2, N).astype(np.int64), gaussian(rng, N),
                          gaussian(rng, N), scale=1 << 50)
    out = aoa.Ciphertext(ctx)
    getattr(aoa, "ckks_" + fn)(ctx, out, ct, keys["evk"])
    sk = ctx.upload(np.array([(s_int % q).astype(np.uint64) for q in Q]))
    dec = aoa.ckks_decrypt(ctx, out, sk)
    coeffs, n = aoa.MACLAURIN[fn]
    want = np.polyval(np.array(coeffs[:n])[::-1], vals)
    assert out.level == len(Q) - 1 - n
    assert np.max(np.abs(dec.real - want)) < 1e-6 and np.max(np.abs(dec.imag)) < 1e-6
