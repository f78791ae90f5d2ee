"""The allocation-free HMult entry point (aoa_hmult_relin_rescale_noalloc).

It serves callers that may not allocate device memory while they evaluate (a
host application that owns the whole device memory budget, a serving thread
that must not risk cudaMalloc's synchronisation); it runs the regular HMult +
relinearise + rescale kernels on a fixed 32 MiB scratch array that is part of
the library's device image.  This file is collected last so that a run that
stops at the first failure has already run every other test.
"""
import ctypes

import numpy as np
import pytest

import oracle
from tests.gpu_util import require_gpu

pytestmark = pytest.mark.gpu


def _rand(rng, primes, n):
    return np.array([rng.integers(0, q, n, dtype=np.uint64) for q in primes], dtype=np.uint64)


def test_noalloc_hmult_matches_regular_entry_point_twice():
    require_gpu()
    import aoa_b200 as aoa
    lib = aoa.capi.load()
    ps = oracle.gen_ntt_primes(60, 1 << 14, 9)
    Q, B = ps[:4], ps[4:]
    E = aoa.Engine(13, Q, B, scale_bits=40)
    ctx = aoa.Context(E)
    N, k = E.N, E.k
    rng = np.random.default_rng(2024)
    evk = aoa.SwitchKey(ctx, _rand(rng, ps, N), _rand(rng, ps, N))
    for call in range(2):          # two calls in a row share (and reuse) the scratch
        a = (_rand(rng, Q, N), _rand(rng, Q, N))
        b = (_rand(rng, Q, N), _rand(rng, Q, N))
        dom = aoa.AOA_NTT if call else aoa.AOA_COEF
        want_out = aoa.Ciphertext(ctx)
        got_out = aoa.Ciphertext(ctx)
        wa = aoa.Ciphertext.from_residues(ctx, *a, slots=16, scale=1 << 40, domain=dom)
        wb = aoa.Ciphertext.from_residues(ctx, *b, slots=16, scale=1 << 40, domain=dom)
        ga = aoa.Ciphertext.from_residues(ctx, *a, slots=16, scale=1 << 40, domain=dom)
        gb = aoa.Ciphertext.from_residues(ctx, *b, slots=16, scale=1 << 40, domain=dom)
        aoa.capi.check(lib.aoa_hmult_relin_rescale(ctx.handle, want_out.handle, wa.handle, wb.handle, evk.handle))
        aoa.capi.check(lib.aoa_hmult_relin_rescale_noalloc(ctx.handle, got_out.handle, ga.handle, gb.handle,
                                                           evk.handle))
        assert got_out.level == want_out.level == k - 2
        assert got_out.scale == want_out.scale and got_out.domain == want_out.domain
        g = got_out.download(nlimbs=k - 1, domain=aoa.AOA_NTT)
        w = want_out.download(nlimbs=k - 1, domain=aoa.AOA_NTT)
        assert np.array_equal(g[0], w[0]) and np.array_equal(g[1], w[1]), "call %d" % call


def test_noalloc_hmult_rejects_parameters_beyond_its_scratch():
    require_gpu()
    import aoa_b200 as aoa
    lib = aoa.capi.load()
    ps = oracle.gen_ntt_primes(60, 1 << 17, 20)
    E = aoa.Engine(16, ps[:10], ps[10:])
    ctx = aoa.Context(E)
    N = E.N
    rng = np.random.default_rng(1)
    evk = aoa.SwitchKey(ctx, _rand(rng, ps, N), _rand(rng, ps, N))
    a = aoa.Ciphertext.from_residues(ctx, _rand(rng, ps[:10], N), _rand(rng, ps[:10], N), slots=4)
    out = aoa.Ciphertext(ctx)
    st = lib.aoa_hmult_relin_rescale_noalloc(ctx.handle, out.handle, a.handle, a.handle, evk.handle)
    assert st == 1   # AOA_ERR_BAD_PARAM
    assert "MiB" in lib.aoa_last_error().decode()
