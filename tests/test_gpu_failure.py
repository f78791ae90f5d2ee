"""Failure detection without a GPU fault: bounded device waits that run out.

Every mbarrier wait in the engine's kernels is bounded; a wait that expires
sets a bit in the engine's device error word, lets its own copies and MMAs
in flight land (with the default bound) and returns, and aoa_ctx_sync
reports AOA_ERR_TIMEOUT (the reference has no such path: its
cudaCheckError() exits the process, include/newckks/cuda/htrans/common.h:
20-29).  Here waits are made to run out on purpose: on a barrier that
nothing ever completes, and in the real transform and conversion kernels
with a spin limit of zero.  The context must stay usable afterwards.
"""
import numpy as np
import pytest

import oracle
from oracle import Oracle, ST_NTT
from tests.ckks_inputs import make_keys, uniform_residues
from tests.gpu_util import require_gpu

pytestmark = pytest.mark.gpu


def _setup(log_n=12):
    import aoa_b200 as aoa
    ps = oracle.gen_ntt_primes(60, 1 << 17, 9)
    Q, B = ps[:5], ps[5:]
    E = aoa.Engine(log_n, Q, B)
    return aoa, E, aoa.Context(E), Oracle(1 << log_n, Q, B), Q, B


def _expect_timeout(aoa, ctx):
    with pytest.raises(aoa.AoaError) as ei:
        ctx.sync()
    assert ei.value.name == "AOA_ERR_TIMEOUT"
    ctx.sync()                                     # the record is cleared by the report


def test_wait_on_a_barrier_nothing_completes_reports_timeout():
    require_gpu()
    aoa, E, ctx, o, Q, B = _setup()
    lib = aoa.capi.load()
    aoa.capi.check(lib.aoa_ctx_wait_check(ctx.handle, 256))
    _expect_timeout(aoa, ctx)
    assert lib.aoa_ctx_wait_check(ctx.handle, -1) == 1          # AOA_ERR_BAD_PARAM
    # the context is usable: a transform on it is still bit-exact
    rng = np.random.default_rng(1)
    x = uniform_residues(rng, Q + B, E.N)
    d = ctx.upload(x)
    ctx.ntt_fwd(d, 1, 0, len(Q + B))
    assert np.array_equal(d.numpy(), o.ntt_fwd(x))


@pytest.mark.parametrize("cols_kind", [0, 1])
def test_zero_spin_limit_in_transform_kernels_reports_timeout(cols_kind):
    """With spin_limit 0 the column and row passes give up on their first tile
    (both column-pass kinds), drain the copy in flight and return."""
    require_gpu()
    aoa, E, ctx, o, Q, B = _setup()
    E.tune("ntt_cols_kind", cols_kind)
    rng = np.random.default_rng(2)
    x = np.stack([uniform_residues(rng, Q + B, E.N) for _ in range(4)])
    d = ctx.upload(x)
    E.tune("spin_limit", 0)
    assert E.tune_get("spin_limit") == 0
    ctx.ntt_fwd(d, 4, 0, len(Q + B))
    _expect_timeout(aoa, ctx)
    E.tune("spin_limit", 1 << 20)
    d = ctx.upload(x)
    ctx.ntt_fwd(d, 4, 0, len(Q + B))
    got = d.numpy()
    for p in range(4):
        assert np.array_equal(got[p], o.ntt_fwd(x[p]))


def test_zero_spin_limit_in_hmult_reports_timeout_then_recovers():
    """HMult's transforms and tensor-core conversions (which wait on their
    table image and on their MMAs) give up with spin_limit 0; with the
    default limit the same context then computes the oracle's residues."""
    require_gpu()
    aoa, E, ctx, o, Q, B = _setup()
    keys = make_keys(o, seed=3)
    evk = aoa.SwitchKey(ctx, *keys["evk"])
    rng = np.random.default_rng(4)
    N, k = E.N, E.k
    a = (uniform_residues(rng, Q, N), uniform_residues(rng, Q, N))
    b = (uniform_residues(rng, Q, N), uniform_residues(rng, Q, N))
    E.tune("spin_limit", 0)
    for tc in (1, 0):
        E.tune("conv_tensor_cores", tc)
        ca = aoa.Ciphertext.from_residues(ctx, *a, slots=8, scale=1 << 40, domain=aoa.AOA_NTT)
        cb = aoa.Ciphertext.from_residues(ctx, *b, slots=8, scale=1 << 40, domain=aoa.AOA_NTT)
        out = aoa.Ciphertext(ctx)
        aoa.capi.check(aoa.capi.load().aoa_hmult_relin_rescale(ctx.handle, out.handle, ca.handle, cb.handle,
                                                               evk.handle))
        _expect_timeout(aoa, ctx)
    E.tune("spin_limit", 1 << 20)
    E.tune("conv_tensor_cores", 1)
    ca = aoa.Ciphertext.from_residues(ctx, *a, slots=8, scale=1 << 40, domain=aoa.AOA_NTT)
    cb = aoa.Ciphertext.from_residues(ctx, *b, slots=8, scale=1 << 40, domain=aoa.AOA_NTT)
    out = aoa.Ciphertext(ctx)
    aoa.ckks_mul(ctx, out, ca, cb, evk)
    w0, w1, _ = o.hmult(a, b, keys["evk"], k - 1, 1 << 40, 1 << 40, rescale=True, a_state=ST_NTT, b_state=ST_NTT)
    g0, g1 = out.download(nlimbs=k - 1)
    assert np.array_equal(g0, w0[: k - 1]) and np.array_equal(g1, w1[: k - 1])
