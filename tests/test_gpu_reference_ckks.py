"""The CUDA engine's CKKS layer against outputs of the reference evaluators.

The golden outputs of pdroalves/aoa's own aoa-ntt and aoa-dgt CKKS layers that
pin the oracle (tests/test_oracle_reference_ckks.py) are compared here with
this library's kernels, through the C ABI, on each reference's primes (the
aoa-dgt records on a context whose transform is the DGT): HMult with and
without rescale (per call, batched, and the reference's own per-call
sequence), rotations and conjugation (the same three ways), addition,
subtraction and the encoder on seeded operands, then HMult and decryption of
ciphertexts the reference encrypted under its own keys, word for word."""
import numpy as np
import pytest

from tests.gpu_util import require_gpu
from tests.test_oracle_reference_ckks import (FIXTURES, HERE, LEVELS, ROTATIONS, SCALE_A, SCALE_B, ct_record,
                                              decoded, load, seeded_ct, seeded_key, splitmix_values)

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", params=FIXTURES)
def env(request):
    require_gpu()
    import json
    import os
    import aoa_b200 as aoa
    from oracle import dgt_roots
    g, N, k, kl, prec, primes = load(request.param)
    if "dgt" in request.param:                   # the AOADGT evaluator: a DGT context on aoa-dgt's roots
        with open(os.path.join(HERE, "golden", "dgt_roots.json")) as f:
            gens, roots = dgt_roots(json.load(f), primes, N // 2)
        E = aoa.Engine(N.bit_length() - 1, primes[:k], primes[k:], scale_bits=prec, generators=gens, dgt_roots=roots)
        ctx = aoa.Context(E)
        ctx.set_transform(aoa.AOA_DGT)
        ctx.is_dgt = True
    else:
        E = aoa.Engine(N.bit_length() - 1, primes[:k], primes[k:], scale_bits=prec)
        ctx = aoa.Context(E)
        ctx.is_dgt = False
    return aoa, g, N, k, kl, prec, primes, ctx


def _ct(aoa, ctx, pair, level, scale, slots):
    return aoa.Ciphertext.from_residues(ctx, pair[0], pair[1], level=level, slots=slots, scale=scale)


def _key(aoa, ctx, pair):
    return aoa.SwitchKey(ctx, pair[0], pair[1], domain=aoa.AOA_COEF)


def _check(out, words, N, name):
    _, scale, slots, r0, r1 = ct_record(words, N)
    n = r0.shape[0]
    assert out.level == n - 1 and out.scale == scale and out.slots == slots, name
    g0, g1 = out.download(nlimbs=n)
    assert np.array_equal(g0, r0) and np.array_equal(g1, r1), name


@pytest.mark.parametrize("level", LEVELS)
def test_hmult_equals_reference(env, level):
    aoa, g, N, k, kl, prec, primes, ctx = env
    evk = _key(aoa, ctx, seeded_key(111, 112, primes, N))
    a_in, b_in = seeded_ct(101, 102, primes[:k], N), seeded_ct(103, 104, primes[:k], N)
    for rescale in (True, False):
        name = ("hmult_l%d" % (level - 1)) if rescale else ("hmult_norescale_l%d" % level)
        a, b = _ct(aoa, ctx, a_in, level, SCALE_A, N // 2), _ct(aoa, ctx, b_in, level, SCALE_B, N // 2)
        out = aoa.Ciphertext(ctx)
        (aoa.ckks_mul if rescale else aoa.ckks_mul_without_rescale)(ctx, out, a, b, evk)
        _check(out, g["n1024_" + name], N, name)
        if rescale and not ctx.is_dgt:   # the reference's own per-call op sequence (NTT contexts)
            out = aoa.Ciphertext(ctx)
            aoa.ckks_mul_plain(ctx, out, _ct(aoa, ctx, a_in, level, SCALE_A, N // 2),
                               _ct(aoa, ctx, b_in, level, SCALE_B, N // 2), evk)
            _check(out, g["n1024_" + name], N, name + " per-call sequence")
        # the batched path (fused kernels, one launch per stage for the batch)
        a2 = [_ct(aoa, ctx, a_in, level, SCALE_A, N // 2) for _ in range(3)]
        b2 = [_ct(aoa, ctx, b_in, level, SCALE_B, N // 2) for _ in range(3)]
        outs = [aoa.Ciphertext(ctx) for _ in range(3)]
        aoa.ckks_mul_batch(ctx, outs, a2, b2, evk, rescale=rescale)
        for o in outs:
            _check(o, g["n1024_" + name], N, name + " batched")


@pytest.mark.parametrize("level", LEVELS)
def test_rotations_and_conjugation_equal_reference(env, level):
    aoa, g, N, k, kl, prec, primes, ctx = env
    c_in = seeded_ct(105, 106, primes[:k], N)
    for r in ROTATIONS:
        rtk = _key(aoa, ctx, seeded_key(113 + 10 * r, 114 + 10 * r, primes, N))
        out = aoa.Ciphertext(ctx)
        aoa.ckks_rotate_left(ctx, out, _ct(aoa, ctx, c_in, level, SCALE_A, N // 2), r, rtk)
        _check(out, g["n1024_rotate%d_l%d" % (r, level)], N, "rotate %d" % r)
        if ctx.is_dgt:          # batched rotations and the reference-sequence path: NTT contexts
            continue
        outs = [aoa.Ciphertext(ctx) for _ in range(2)]
        aoa.ckks_rotate_batch(ctx, outs, [_ct(aoa, ctx, c_in, level, SCALE_A, N // 2) for _ in range(2)], r, rtk)
        for o in outs:
            _check(o, g["n1024_rotate%d_l%d" % (r, level)], N, "rotate %d batched" % r)
        out = aoa.Ciphertext(ctx)                # the reference's own per-call sequence
        aoa.ckks_rotate_plain(ctx, out, _ct(aoa, ctx, c_in, level, SCALE_A, N // 2), r, rtk)
        assert out.domain == aoa.AOA_COEF
        _check(out, g["n1024_rotate%d_l%d" % (r, level)], N, "rotate %d per-call sequence" % r)
    cjk = _key(aoa, ctx, seeded_key(115, 116, primes, N))
    out = aoa.Ciphertext(ctx)
    aoa.ckks_conjugate(ctx, out, _ct(aoa, ctx, c_in, level, SCALE_A, N // 2), cjk)
    _check(out, g["n1024_conjugate_l%d" % level], N, "conjugate")
    if not ctx.is_dgt:
        out = aoa.Ciphertext(ctx)
        aoa.ckks_conjugate_plain(ctx, out, _ct(aoa, ctx, c_in, level, SCALE_A, N // 2), cjk)
        _check(out, g["n1024_conjugate_l%d" % level], N, "conjugate per-call sequence")


@pytest.mark.parametrize("level", LEVELS)
def test_add_sub_equal_reference(env, level):
    aoa, g, N, k, kl, prec, primes, ctx = env
    a_in, c_in = seeded_ct(101, 102, primes[:k], N), seeded_ct(105, 106, primes[:k], N)
    for name, fn in (("add", aoa.ckks_add), ("sub", aoa.ckks_sub)):
        out = aoa.Ciphertext(ctx)
        fn(ctx, out, _ct(aoa, ctx, a_in, level, SCALE_A, N // 2), _ct(aoa, ctx, c_in, level, SCALE_A, N // 2))
        _check(out, g["n1024_%s_l%d" % (name, level)], N, name)


@pytest.mark.parametrize("slots", [512, 8])
def test_encode_equals_reference(env, slots):
    aoa, g, N, k, kl, prec, primes, ctx = env
    poly, scale = aoa.ckks_encode(ctx, splitmix_values(200 + slots, slots), scale=SCALE_A)
    w = g["n1024_encode_s%d" % slots]
    assert scale == int(w[0])
    assert np.array_equal(poly.numpy(), w[1:].reshape(k, N))


def test_reference_keys_hmult_and_decryptions(env):
    """Ciphertexts the reference encrypted under its own keys: this engine's
    HMult with the reference's evaluation key equals the reference's ckks_mul
    output word for word, and its decryptions equal the reference's."""
    aoa, g, N, k, kl, prec, primes, ctx = env
    slots = N // 2
    evk_w = g["n1024_evk"].reshape(2, k + kl, N)
    evk = _key(aoa, ctx, (evk_w[0], evk_w[1]))
    cts = {}
    for name in ("enc300", "enc301", "mul_keys", "rot1_keys"):
        _, sc, sl, c0, c1 = ct_record(g["n1024_" + name], N)
        pad = np.zeros((k - c0.shape[0], N), np.uint64)
        cts[name] = aoa.Ciphertext.from_residues(ctx, np.vstack([c0, pad]), np.vstack([c1, pad]),
                                                 level=c0.shape[0] - 1, slots=sl, scale=sc)
    out = aoa.Ciphertext(ctx)
    aoa.ckks_mul(ctx, out, cts["enc300"], cts["enc301"], evk)
    _check(out, g["n1024_mul_keys"], N, "HMult under the reference's keys")
    s = g["n1024_sk"].view(np.int64)
    s_res = np.array([np.where(s >= 0, s, s + p).astype(np.uint64) for p in primes[:k]])
    sk = ctx.upload(s_res)
    v1, v2 = splitmix_values(300, slots), splitmix_values(301, slots)
    for name, dec, expect, tol in (("enc300", "dec300", v1, 1e-9), ("mul_keys", "dec_mul", v1 * v2, 1e-6),
                                   ("rot1_keys", "dec_rot1", np.roll(v1, -1), 1e-6)):
        got = aoa.ckks_decrypt(ctx, cts[name], sk)
        want = decoded(g["n1024_" + dec])
        assert np.max(np.abs(got - want)) <= 1e-12 * max(1.0, np.max(np.abs(want))), name
        assert np.max(np.abs(got - expect)) < tol, name
