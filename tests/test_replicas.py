"""Multi-process replica plumbing on CPU (gloo, world size 2): the timed
region's max-over-ranks reduction, the whole-job rate, per-rank inputs and
the barrier, as bench.py uses them over NCCL on GPUs."""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

WORKER = r'''
import json, os, sys, time
sys.path.insert(0, os.environ["AOA_ROOT"])
import numpy as np
from aoa_b200 import replicas
world, rank, local = replicas.ranks()
pg = replicas.init("gloo", timeout_s=30)
seed = replicas.replica_seed(1000, rank)
x = np.random.default_rng(seed).integers(0, 1 << 60, 4, dtype=np.uint64)
replicas.barrier(pg)
ms = 10.0 * (rank + 1)                    # rank 1 is the slowest
mx = replicas.max_over_ranks(ms, pg)
rate = replicas.job_rate(16, world, mx)
if rank == 0:
    print(json.dumps({"world": world, "max_ms": mx, "rate": rate, "seed": seed, "x0": int(x[0])}), flush=True)
else:
    print(json.dumps({"rank": rank, "seed": seed, "x0": int(x[0])}), flush=True)
replicas.finish(pg)
'''


def _run(world, port):
    procs = []
    for r in range(world):
        env = dict(os.environ, WORLD_SIZE=str(world), RANK=str(r), LOCAL_RANK=str(r), MASTER_ADDR="127.0.0.1",
                   MASTER_PORT=str(port), AOA_ROOT=ROOT, CUDA_VISIBLE_DEVICES="")
        procs.append(subprocess.Popen([sys.executable, "-c", WORKER], env=env, stdout=subprocess.PIPE,
                                      stderr=subprocess.PIPE, text=True))
    outs = []
    for p in procs:
        o, e = p.communicate(timeout=120)
        assert p.returncode == 0, e[-2000:]
        outs.append(json.loads(o.strip().splitlines()[-1]))
    return outs


def test_two_gloo_replicas_max_over_ranks():
    pytest.importorskip("torch.distributed")
    r0, r1 = _run(2, 29517)
    assert r0["world"] == 2 and r0["max_ms"] == 20.0            # the slowest rank's time
    assert abs(r0["rate"] - 2 * 16 / 0.020) < 1e-6              # all ranks' units over that time
    assert r0["seed"] != r1["seed"] and r0["x0"] != r1["x0"]     # each replica draws its own inputs


def test_single_process_needs_no_group():
    from aoa_b200 import replicas
    assert replicas.init("gloo") is None or int(os.environ.get("WORLD_SIZE", "1")) > 1
    assert replicas.max_over_ranks(3.5, None) == 3.5
    assert replicas.job_rate(10, 1, 500.0) == 20.0
