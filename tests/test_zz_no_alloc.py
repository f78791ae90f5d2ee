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

CU_MEMPOOL_ATTR_RESERVED_MEM_CURRENT = 5
CU_MEMPOOL_ATTR_USED_MEM_CURRENT = 7


def _rand(rng, primes, n):
    return np.array([rng.integers(0, q, n, dtype=np.uint64) for q in primes], dtype=np.uint64)


def _default_pool_usage(ordinal):
    """(used, reserved) bytes of the device's default memory pool, the pool
    every stream-ordered allocation of the library draws from (driver API)."""
    cu = ctypes.CDLL("libcuda.so.1")
    dev = ctypes.c_int()
    pool = ctypes.c_void_p()
    assert cu.cuDeviceGet(ctypes.byref(dev), ordinal) == 0
    assert cu.cuDeviceGetDefaultMemPool(ctypes.byref(pool), dev) == 0
    out = []
    for attr in (CU_MEMPOOL_ATTR_USED_MEM_CURRENT, CU_MEMPOOL_ATTR_RESERVED_MEM_CURRENT):
        v = ctypes.c_uint64()
        assert cu.cuMemPoolGetAttribute(pool, attr, ctypes.byref(v)) == 0
        out.append(v.value)
    return tuple(out)


def test_noalloc_hmult_matches_regular_entry_point_twice():
    """Two no-alloc calls in a row, made first, on a context that has never
    allocated a workspace: the device's memory pool holds exactly as much
    before as after them, and each result equals the regular (allocating)
    entry point's on the same inputs, residue for residue."""
    require_gpu()
    import torch
    import aoa_b200 as aoa
    lib = aoa.capi.load()
    ps = oracle.gen_ntt_primes(60, 1 << 14, 9)
    Q, B = ps[:4], ps[4:]
    E = aoa.Engine(13, Q, B, scale_bits=40)
    owner = aoa.Context(E)            # holds the inputs, outputs and key
    fresh = aoa.Context(E)            # runs the no-alloc calls: no workspace ever allocated
    N, k = E.N, E.k
    rng = np.random.default_rng(2024)
    evk = aoa.SwitchKey(owner, _rand(rng, ps, N), _rand(rng, ps, N))
    calls = []
    for call in range(2):
        a = (_rand(rng, Q, N), _rand(rng, Q, N))
        b = (_rand(rng, Q, N), _rand(rng, Q, N))
        dom = aoa.AOA_NTT if call else aoa.AOA_COEF
        mk = lambda x: aoa.Ciphertext.from_residues(owner, *x, slots=16, scale=1 << 40, domain=dom)
        calls.append({"got": (mk(a), mk(b), aoa.Ciphertext(owner)), "want": (mk(a), mk(b), aoa.Ciphertext(owner))})
    owner.sync()
    fresh.sync()
    torch.cuda.synchronize()
    before = _default_pool_usage(torch.cuda.current_device())
    for c in calls:                   # two calls in a row share (and reuse) the scratch
        ga, gb, gout = c["got"]
        aoa.capi.check(lib.aoa_hmult_relin_rescale_noalloc(fresh.handle, gout.handle, ga.handle, gb.handle,
                                                           evk.handle))
    fresh.sync()
    after = _default_pool_usage(torch.cuda.current_device())
    assert after == before, "the no-alloc HMult changed the memory pool: %s -> %s" % (before, after)
    for z, c in enumerate(calls):
        wa, wb, wout = c["want"]
        aoa.capi.check(lib.aoa_hmult_relin_rescale(owner.handle, wout.handle, wa.handle, wb.handle, evk.handle))
        gout = c["got"][2]
        assert gout.level == wout.level == k - 2
        assert gout.scale == wout.scale and gout.domain == wout.domain
        g = gout.download(nlimbs=k - 1, domain=aoa.AOA_NTT)
        w = wout.download(nlimbs=k - 1, domain=aoa.AOA_NTT)
        assert np.array_equal(g[0], w[0]) and np.array_equal(g[1], w[1]), "call %d" % z


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
