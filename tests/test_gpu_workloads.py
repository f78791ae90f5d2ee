"""CUDA-graph replay, the batched uneven workload and the serving loop on the GPU.

The grouped / captured schedules must give the same residues as the plain
per-call path, and every served request the same result in the mix as when it
runs alone (integer arithmetic: equal bit for bit)."""
import numpy as np
import pytest

import oracle
from tests.ckks_inputs import uniform_residues
from tests.gpu_util import require_gpu

pytestmark = pytest.mark.gpu


def test_graph_replay_matches_direct_calls():
    require_gpu()
    import aoa_b200 as aoa
    ps = oracle.gen_ntt_primes(60, 1 << 13, 9)
    E = aoa.Engine(12, ps[:5], ps[5:], scale_bits=40)
    ctx = aoa.Context(E)
    rng = np.random.default_rng(0)
    N = E.N
    res = lambda qs: uniform_residues(rng, qs, N)
    evk = aoa.SwitchKey(ctx, res(ps), res(ps))
    rtk = aoa.SwitchKey(ctx, res(ps), res(ps))
    a = [aoa.Ciphertext.from_residues(ctx, res(ps[:5]), res(ps[:5]), slots=N // 2, domain=aoa.AOA_NTT)
         for _ in range(4)]
    outs = [aoa.Ciphertext(ctx) for _ in range(4)]

    def chain():
        for x in a:
            x.set(4, N // 2, 1 << 40, aoa.AOA_NTT)
        aoa.ckks_mul_batch(ctx, outs[:2], a[:2], a[2:], evk)
        aoa.ckks_rotate_left(ctx, outs[2], a[0], 4, rtk)
        aoa.ckks_add(ctx, outs[3], a[1], a[3])

    chain()
    want = [o.download(nlimbs=o.level + 1, domain=aoa.AOA_COEF) for o in outs]
    g = aoa.Graph.capture(ctx, chain)
    assert g.nodes > 10
    for o in outs:                       # clobber the outputs, then replay twice
        o.upload(np.zeros((5, N), np.uint64), np.zeros((5, N), np.uint64), domain=aoa.AOA_NTT)
    g.launch()
    g.launch()
    ctx.sync()
    for o, (w0, w1), lvl in zip(outs, want, (3, 3, 4, 4)):
        o.set(lvl, N // 2, o.scale, aoa.AOA_NTT)
        g0, g1 = o.download(nlimbs=lvl + 1, domain=aoa.AOA_COEF)
        assert np.array_equal(g0, w0) and np.array_equal(g1, w1)


def test_uneven_batch_grouped_and_captured_equal_plain():
    require_gpu()
    from aoa_b200.workloads import UnevenBatch
    wb = UnevenBatch(n_ops=24, seed=4, log_ns=(11, 12), k=6, kl=7, min_limbs=2)
    wb.run_plain()
    wb.sync()
    plain = [o.download(nlimbs=o.level + 1, domain=1) for o in wb.outs]
    levels = [o.level for o in wb.outs]
    nodes = wb.capture()
    assert nodes > len(wb.ops)
    wb.launch_graphs()
    wb.sync()
    for z, (o, want, lvl) in enumerate(zip(wb.outs, plain, levels)):
        assert o.level == lvl
        got = o.download(nlimbs=lvl + 1, domain=1)
        assert np.array_equal(got[0], want[0]) and np.array_equal(got[1], want[1]), (z, wb.ops[z])


def test_serving_results_alone_equal_in_mix():
    require_gpu()
    from aoa_b200.workloads import Server
    srv = Server(log_ns=(11, 12), k=6, kl=5, slots_per_degree=3, hbm_budget=1 << 30, n_slots_used=8)
    mixed = srv.make_requests(10, seed=6)
    lat, wall = srv.run(mixed, rate=None)
    assert np.all(lat >= 0) and wall > 0
    got = [r["out"].download(nlimbs=r["out"].level + 1, domain=1) for r in mixed]
    alone = srv.make_requests(10, seed=6)
    for r, (g0, g1) in zip(alone, got):
        srv.submit(0, r)
        srv.pool[r["log_n"]][0].sync()
        w0, w1 = r["out"].download(nlimbs=r["out"].level + 1, domain=1)
        assert np.array_equal(g0, w0) and np.array_equal(g1, w1)


def test_batched_serving_results_alone_equal_in_mix():
    """Iteration-level batching (rotations of requests at the same stage in one
    batched launch sequence): every result equals the request run alone."""
    require_gpu()
    from aoa_b200.workloads import BatchServer
    srv = BatchServer(log_ns=(11, 12), k=6, kl=5, hbm_budget=1 << 30, n_slots_used=8)
    mixed = srv.make_requests(10, seed=7)
    lat, wall = srv.run(mixed, rate=2000.0)
    assert np.all(lat >= 0) and wall > 0
    got = [r["out"].download(nlimbs=r["out"].level + 1, domain=1) for r in mixed]
    alone = srv.make_requests(10, seed=7)
    for r, (g0, g1) in zip(alone, got):
        srv.submit(0, r)
        srv.pool[r["log_n"]][0].sync()
        w0, w1 = r["out"].download(nlimbs=r["out"].level + 1, domain=1)
        assert np.array_equal(g0, w0) and np.array_equal(g1, w1)
