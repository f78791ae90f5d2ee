#!/usr/bin/env python3
"""Benchmark: batched HMult + relinearise + rescale at N = 2^16, L = 30.

Workload (one "step"): B independent ckks_mul calls (HMult + relinearisation
with the dnum = 1 evaluation key + rescale) on ciphertext pairs at level 29
(30 live 60-bit Q primes and 31 special 60-bit primes, the largest with
q = 1 mod 2^32, a subset of the NTT primes q = 1 mod 2N; scale 2^50).  Inputs are seeded uniform residues in the state the path's own
previous HMult leaves them in (the steady state of a multiplication chain):
the transform domain for this engine's pipeline, coefficients for the plain
per-call path (the reference's ckks_mul op sequence on the same kernels),
which is timed on the same batch as the comparison.  Each pair occupies
60 MiB; a step touches far more than the 126 MB L2, so no L2 flush is needed
between steps.

Prints one JSON line (rank 0).  --impl reference times the CPU restatement of
the reference algorithm (oracle/) on the host cores instead.
Multi-GPU (torchrun): replicas only — each rank runs its own batch, no
collective on the data path; value = all ranks' ops / max-over-ranks time.
"""
import argparse
import json
import os
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

LOG_N, K, KL, SCALE_BITS = 16, 30, 31, 50
METRIC = "Batched HMult+relin+rescale/s at N=2^16 L=30"
UNIT = "HMult/s"


# The workload's primes: the largest 60-bit primes q = 1 mod 2^32 (q = 1 mod
# 2N holds for every ring degree up to 2^31); their transforms take the
# shorter Shoup remainder.  The transform rate on the largest primes
# q = 1 mod 2N (the general remainder) is reported beside it.
PRIME_MODULUS = 1 << 32


def primes():
    from aoa_b200 import params
    return params.ntt_primes(60, PRIME_MODULUS, K + KL)


def oracle_primes():
    """The same primes from the oracle's own prime search (the reference arm
    loads no library of the product)."""
    import oracle
    return oracle.gen_ntt_primes(60, PRIME_MODULUS, K + KL)


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clock / throttle sampling during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index, self.proc, self.path = index, None, None

    def start(self):
        try:
            self.path = "/tmp/aoa_clocks_%d.csv" % os.getpid()
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.Q,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if not self.proc:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        if not sm:
            return None
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def issue_roofline(issue, clk, sms):
    """The transform against the instruction issue peak: sms x 4 warp
    instructions per SM clock, at the median SM clock of the timed region;
    and against its integer multiply pipe: the pipe cycles its instruction mix
    needs over the cycles of the pipes of all SM sub-partitions in the
    measured time."""
    if not issue:
        return None
    mhz = (clk or {}).get("sm_mhz") or 1965.0
    peak = sms * 4 * mhz * 1e6
    out = dict(issue, peak_per_s=peak, sm_mhz=mhz, frac=issue["achieved_per_s"] / peak)
    if "fma_pipe_cycles" in issue:
        avail = sms * 4 * mhz * 1e6 * issue["seconds"]
        out["fma_pipe_frac"] = issue["fma_pipe_cycles"] / avail
    return out


def dist_setup():
    """(world_size, rank, local_rank) from the launcher's environment."""
    return (int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")),
            int(os.environ.get("LOCAL_RANK", "0")))


def workload_config(batch):
    return {"workload": "hmult_relin_rescale", "log_n": LOG_N, "q_limbs": K, "special_limbs": KL,
            "dnum": 1, "level": K - 1, "prime_bits": 60, "primes": "largest 60-bit q = 1 mod 2^32",
            "scale_bits": SCALE_BITS,
            "batch_per_gpu": batch, "parallelism": "replicas",
            "l2": "inputs exceed L2 (60 MiB per ciphertext pair, %d pairs)" % batch}


def run_reference(args, world, rank):
    """CPU restatement of the reference path (oracle/), all host threads."""
    if rank != 0:
        return
    import oracle
    from oracle import Oracle
    threads = os.cpu_count() or 1
    oracle.lib().oc_set_threads(threads)
    ps = oracle_primes()
    o = Oracle(1 << LOG_N, ps[:K], ps[K:])
    rng = np.random.default_rng(1)
    N = 1 << LOG_N
    rr = lambda qs: np.array([rng.integers(0, q, N, dtype=np.uint64) for q in qs], dtype=np.uint64)
    a, b = (rr(ps[:K]), rr(ps[:K])), (rr(ps[:K]), rr(ps[:K]))
    evk = (rr(ps), rr(ps))
    for _ in range(args.warmup):
        o.hmult(a, b, evk, K - 1, 1 << SCALE_BITS, 1 << SCALE_BITS)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        o.hmult(a, b, evk, K - 1, 1 << SCALE_BITS, 1 << SCALE_BITS)
    dt = time.perf_counter() - t0
    v = args.steps / dt
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000 * dt / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u64",
            "data": "synthetic",
            "config": workload_config(args.batch),
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": threads, "kind": "port",
                             "sample": "1 of the step's %d HMult+relin+rescale per timed step (bounded sample; "
                                       "reference op sequence restated in oracle/ckks_oracle.cpp, OpenMP)"
                                       % args.batch},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def profile_case(args, aoa, ctx, rr, ps):
    """Small fixed cases for ncu: `ntt` / `dgt` = forward + inverse NTT / DGT
    over args.polys polys of 30 limbs (args.polys * 15 MiB); `hmult` = 2
    HMult+relin+rescale; `batch` = 2 batched calls of args.batch
    HMult+relin+rescale."""
    N = 1 << LOG_N
    if args.profile_case == "dgt":
        ctx.set_transform(aoa.AOA_DGT)
        buf = ctx.alloc((args.polys, K, N))
        xs = rr(ps[:K])
        for p in range(args.polys):
            aoa.capi.check(aoa.capi.load().aoa_memcpy_h2d(ctx.handle, buf.offset(p * K * N), aoa.capi.ptr(xs),
                                                          xs.nbytes))
        for _ in range(2):
            ctx.dgt_fwd(buf, args.polys, 0, K)
            ctx.dgt_inv(buf, args.polys, 0, K)
        ctx.sync()
        assert np.array_equal(buf.numpy()[0], xs), "inverse(forward(x)) != x"
    elif args.profile_case == "ntt":
        buf = ctx.alloc((args.polys, K, N))
        xs = rr(ps[:K])
        for p in range(args.polys):
            aoa.capi.check(aoa.capi.load().aoa_memcpy_h2d(ctx.handle, buf.offset(p * K * N), aoa.capi.ptr(xs),
                                                          xs.nbytes))
        for _ in range(2):
            ctx.ntt_fwd(buf, args.polys, 0, K)
            ctx.ntt_inv(buf, args.polys, 0, K)
        ctx.sync()
        assert np.array_equal(buf.numpy()[0], xs), "inverse(forward(x)) != x"
    elif args.profile_case == "batch":
        evk = aoa.SwitchKey(ctx, rr(ps), rr(ps))
        A = [aoa.Ciphertext.from_residues(ctx, rr(ps[:K]), rr(ps[:K]), slots=N // 2, scale=1 << SCALE_BITS,
                                          domain=aoa.AOA_NTT) for _ in range(args.batch)]
        Bs = [aoa.Ciphertext.from_residues(ctx, rr(ps[:K]), rr(ps[:K]), slots=N // 2, scale=1 << SCALE_BITS,
                                           domain=aoa.AOA_NTT) for _ in range(args.batch)]
        outs = [aoa.Ciphertext(ctx) for _ in range(args.batch)]
        for _ in range(2):
            for x in A + Bs:
                x.set(K - 1, N // 2, 1 << SCALE_BITS, aoa.AOA_NTT)
            aoa.ckks_mul_batch(ctx, outs, A, Bs, evk)
        ctx.sync()
    else:
        evk = aoa.SwitchKey(ctx, rr(ps), rr(ps))
        a = aoa.Ciphertext.from_residues(ctx, rr(ps[:K]), rr(ps[:K]), slots=N // 2, scale=1 << SCALE_BITS)
        b = aoa.Ciphertext.from_residues(ctx, rr(ps[:K]), rr(ps[:K]), slots=N // 2, scale=1 << SCALE_BITS)
        o = aoa.Ciphertext(ctx)
        for _ in range(2):
            a.set(K - 1, N // 2, 1 << SCALE_BITS, aoa.AOA_COEF)
            b.set(K - 1, N // 2, 1 << SCALE_BITS, aoa.AOA_COEF)
            aoa.ckks_mul(ctx, o, a, b, evk)
        ctx.sync()
    print("profile case done")


def accuracy(aoa, log_n, Q, B, scale_bits, seed):
    """encode -> encrypt -> HMult + relinearise + rescale -> decrypt -> decode,
    every stage on the GPU through the package API, keys generated on the GPU
    from sampled draws (ternary secret of Hamming weight 64, Gaussian errors of
    sigma 3.2, ternary u); slots = N/2 uniform in the unit disk.  Returns the
    max and mean absolute error of the decoded product against the FP64
    cleartext product."""
    primes = list(Q) + list(B)
    k, kl = len(Q), len(B)
    E = aoa.Engine(log_n, Q, B, scale_bits=scale_bits)
    ctx = aoa.Context(E)
    rng = np.random.default_rng(seed)
    N = 1 << log_n
    s_int = np.zeros(N, np.int64)
    idx = rng.choice(N, 64, replace=False)
    s_int[idx] = rng.choice([-1, 1], 64)
    s = ctx.upload(np.array([(s_int % q).astype(np.uint64) for q in primes]))
    gauss = lambda: np.rint(rng.normal(0.0, 3.2, N)).astype(np.int64)
    unif = lambda: np.array([rng.integers(0, q, N, dtype=np.uint64) for q in primes])
    draws = {"pk": (ctx.upload(unif()), ctx.upload(gauss())), "evk": (ctx.upload(unif()), ctx.upload(gauss()))}
    keys = aoa.ckks_keygen(ctx, s, draws)
    slots = N // 2
    vals = []
    for _ in range(2):
        r, t = np.sqrt(rng.uniform(0, 1, slots)), rng.uniform(0, 2 * np.pi, slots)
        vals.append(r * np.exp(1j * t))
    scale = 1 << scale_bits
    cts = [aoa.ckks_encrypt(ctx, v, keys["pk"], rng.integers(-1, 2, N).astype(np.int64), gauss(), gauss(),
                            scale=scale) for v in vals]
    out = aoa.Ciphertext(ctx)
    aoa.ckks_mul(ctx, out, cts[0], cts[1], keys["evk"])
    sk = ctx.upload(np.array([(s_int % q).astype(np.uint64) for q in primes[:k]]))
    dec = aoa.ckks_decrypt(ctx, out, sk)
    err = np.abs(dec - vals[0] * vals[1])
    return {"log_n": log_n, "q_limbs": k, "q_bits": [int(q).bit_length() for q in Q], "special_limbs": kl,
            "b_bits": int(B[0]).bit_length(), "scale_bits": scale_bits,
            "slots": slots, "max_abs_err": float(err.max()), "mean_abs_err": float(err.mean()),
            "max_abs_err_log2": float(np.log2(err.max())), "within_2^-20": bool(err.max() <= 2.0 ** -20)}


def reference_layout_n4096():
    """The primes the reference's CUDAManager::init(k = 3, kl = 4, N = 2^12,
    prec = 52) selects: its first 63-bit prime, two of its 52-bit bucket, and
    four of its 55-bit bucket as the special primes (a copy of its tables is
    the fixture tests/golden/reference_primes.json)."""
    from aoa_b200 import params
    with open(os.path.join(os.path.dirname(os.path.abspath(__file__)), "tests", "golden",
                           "reference_primes.json")) as f:
        table = json.load(f)
    return params.reference_prime_set(table, 3, 4, 52)


def cpu_chain(Q, B, scale_bits):
    """Config 1 on the host: the oracle (the reference's CPU path restated)
    runs encode -> encrypt -> HMult + relinearise + rescale -> decrypt -> decode
    at N = 2^12, single-threaded and on all host threads."""
    import oracle
    from oracle import Oracle
    from tests.ckks_inputs import make_keys, encrypt_values, decrypt_values
    o = Oracle(1 << 12, list(Q), list(B))
    keys = make_keys(o, seed=2)
    rng = np.random.default_rng(1)
    slots = 2048
    vals = []
    for _ in range(2):
        r, t = np.sqrt(rng.uniform(0, 1, slots)), rng.uniform(0, 2 * np.pi, slots)
        vals.append(r * np.exp(1j * t))
    scale = 1 << scale_bits
    out = {"slots": slots, "scale_bits": scale_bits, "q_bits": [int(q).bit_length() for q in Q]}
    for label, threads in (("single_thread", 1), ("all_threads", os.cpu_count() or 1)):
        oracle.lib().oc_set_threads(threads)
        t0 = time.perf_counter()
        ca = encrypt_values(o, keys, vals[0], scale, seed=3)
        cb = encrypt_values(o, keys, vals[1], scale, seed=4)
        r0, r1, rsc = o.hmult(ca, cb, keys["evk"], len(Q) - 1, scale, scale, rescale=True, a_state=oracle.ST_NTT,
                              b_state=oracle.ST_NTT)
        pad = lambda x: np.concatenate([x[: len(Q) - 1], np.zeros((1, x.shape[1]), np.uint64)])
        dec = decrypt_values(o, keys, (pad(r0), pad(r1)), slots, rsc, state=oracle.ST_COEF)
        ms = (time.perf_counter() - t0) * 1000
        err = np.abs(dec - vals[0] * vals[1])
        out[label] = {"threads": threads, "ms": ms, "max_abs_err": float(err.max()),
                      "mean_abs_err": float(err.mean())}
    out["cpu_model"] = cpu_model()
    return out


def cpu_model():
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def systems_workloads(aoa, torch):
    """Batched uneven mix (512 ops, N in {2^14, 2^15, 2^16}, live limbs 4..30,
    50% HMult+relin+rescale / 30% rotate by 2^j / 20% add): grouped launches
    captured in CUDA graphs vs the plain per-call path; then the serving loop
    (plaintext-weight multiply + rescale, rotate-and-sum, rescale; N in
    {2^15, 2^16}, live limbs 6..30) at 5 Poisson rates relative to its measured
    saturation throughput."""
    from aoa_b200.workloads import UnevenBatch, Server, BatchServer
    wb = UnevenBatch(n_ops=512, seed=4, autotune=True)

    def timed_multi(fn):
        wb.sync()
        torch.cuda.synchronize()
        evs = {ln: (torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for ln in wb.ctx}
        st = {ln: torch.cuda.ExternalStream(c.stream) for ln, c in wb.ctx.items()}
        first = next(iter(wb.ctx))
        evs[first][0].record(st[first])
        for ln in wb.ctx:
            if ln != first:
                evs[ln][0].record(st[ln])
        fn()
        for ln in wb.ctx:
            evs[ln][1].record(st[ln])
        wb.sync()
        torch.cuda.synchronize()
        return max(evs[first][0].elapsed_time(evs[ln][1]) for ln in wb.ctx)

    wb.run_plain()
    plain_ms = timed_multi(wb.run_plain)
    nodes = wb.capture()
    wb.launch_graphs()
    graph_ms = min(timed_multi(wb.launch_graphs) for _ in range(3))
    grouped_ms = timed_multi(lambda: [wb.run_grouped(ln) for ln in wb.ctx])
    n_ops = len(wb.ops)
    mix = {k: sum(1 for op in wb.ops if op["kind"] == k) for k in ("mul", "rot", "add")}
    uneven = {"ops": n_ops, "mix": mix, "seed": 4,
              "graph_ops_per_s": n_ops / (graph_ms / 1000.0), "grouped_ops_per_s": n_ops / (grouped_ms / 1000.0),
              "plain_ops_per_s": n_ops / (plain_ms / 1000.0), "speedup_vs_plain": plain_ms / graph_ms,
              "graph_nodes": nodes, "algorithmic_bytes": wb.bytes,
              "achieved_gbs": wb.bytes / (graph_ms / 1000.0) / 1e9,
              "rotation_keys": "a distinct key per step 2^j and degree",
              "plain": "one op at a time in input order: HMult and rotations through the reference's per-call "
                       "sequences on this engine (aoa_hmult_plain, aoa_rotate_plain), additions as ckks_add",
              "schedule": "one stream per N; HMults grouped by limb count (<=64 per launch), rotations in one "
                          "batched call per N (grouped by limb count, a step and key per op), additions; "
                          "one CUDA graph per stream"}
    del wb
    n_req = 500

    def serve(server, reqs, factors):
        server.run(reqs[:16], rate=None)                  # warm the contexts' workspaces
        lat, wall = server.run(reqs, rate=None)
        sat = len(reqs) / wall
        out = {"saturation_req_per_s": sat, "saturation_stats": dict(server.stats), "rates": []}
        for f in factors:
            lat, wall = server.run(reqs, rate=f * sat)
            out["rates"].append({"rate_factor": f, "offered_req_per_s": f * sat, "requests": len(reqs),
                                 "served_req_per_s": len(reqs) / wall,
                                 "p50_ms": float(np.percentile(lat, 50) * 1000),
                                 "p99_ms": float(np.percentile(lat, 99) * 1000),
                                 "max_ms": float(np.max(lat) * 1000), **server.stats})
        return out

    srv = Server(log_ns=(15, 16), slots_per_degree=4, hbm_budget=8 << 30, autotune=True)
    reqs = srv.make_requests(n_req, seed=6, templates=8)
    serving = serve(srv, reqs, (0.25, 0.5, 0.75, 0.9, 1.1))
    serving.update({"requests_per_rate": n_req, "streams_per_degree": 4, "hbm_budget_bytes": 8 << 30,
                    "resident_key_bytes": srv.resident_bytes,
                    "request": "ct*w (plaintext, rescale) + rotate-and-sum over N/2 slots + rescale; N in "
                               "{2^15,2^16}, live limbs 6..30; latency = arrival to completion (host clock)"})
    del srv, reqs
    # the same requests with iteration-level batching (one context per degree)
    bsrv = BatchServer(log_ns=(15, 16), hbm_budget=8 << 30, autotune=True)
    breqs = bsrv.make_requests(n_req, seed=6, templates=8)
    serving["iteration_batched"] = serve(bsrv, breqs, (0.25, 0.5, 0.75, 0.9, 1.1))
    serving["iteration_batched"]["schedule"] = (
        "one context per degree; each iteration advances every active request one stage, the rotations of a "
        "stage in one batched launch sequence (aoa_rotate_batch); arrivals join at the next iteration")
    # a budget that binds: the resident keys plus room for six 2^16 requests
    budget = bsrv.resident_bytes + 6 * bsrv.footprint(16)
    bsrv.hbm_budget = budget
    bound = serve(bsrv, breqs, (0.9,))
    bound.update({"hbm_budget_bytes": budget, "resident_key_bytes": bsrv.resident_bytes,
                  "note": "HBM budget = resident Galois keys and weights + 6 requests at 2^16; admission waits "
                          "for budget (deferred_by_budget), not for slots"})
    serving["iteration_batched_budget_bound"] = bound
    return uneven, serving


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--batch", type=int, default=48)
    ap.add_argument("--impl", default="aoa", choices=["aoa", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-systems", action="store_true", help="skip the uneven-batch and serving measurements")
    ap.add_argument("--profile-case", choices=["ntt", "dgt", "hmult", "batch"],
                    help="run a small fixed case for ncu captures (no timing, no JSON)")
    ap.add_argument("--polys", type=int, default=16, help="polys of 30 limbs for --profile-case ntt / dgt")
    ap.add_argument("--autotune", action="store_true",
                    help="run the transform autotuner first (default: the engine's measured-best shapes)")
    ap.add_argument("--no-autotune", action="store_true", help="(default) keep the engine's transform shapes")
    ap.add_argument("--knobs", default="", help="engine knobs name=value,... applied before the run")
    args = ap.parse_args()
    world, rank, local = dist_setup()     # the launcher's WORLD_SIZE / RANK / LOCAL_RANK
    if args.impl == "reference":
        run_reference(args, world, rank)
        return

    import torch
    torch.cuda.set_device(local)
    from aoa_b200 import replicas
    pg = replicas.init("nccl", timeout_s=120, device=torch.device("cuda", local))
    import aoa_b200 as aoa

    ps = primes()
    E = aoa.Engine(LOG_N, ps[:K], ps[K:], scale_bits=SCALE_BITS)
    source = "engine defaults (measured best on B200 at 2^16)"
    if args.knobs:
        for kv in args.knobs.split(","):
            k, v = kv.split("=")
            E.tune(k, float(v))
        source = "knobs " + args.knobs
    elif args.autotune and not args.profile_case:
        E.autotune()
        source = "autotuner"
    tuning = dict(E.transform_shapes(), source=source)
    ctx = aoa.Context(E)
    stream = torch.cuda.ExternalStream(ctx.stream)
    N = 1 << LOG_N
    B = args.batch
    rng = np.random.default_rng(replicas.replica_seed(1000, rank))
    rr = lambda qs: np.array([rng.integers(0, q, N, dtype=np.uint64) for q in qs], dtype=np.uint64)
    if args.profile_case:
        profile_case(args, aoa, ctx, rr, ps)
        return
    evk = aoa.SwitchKey(ctx, rr(ps), rr(ps))
    host_in = [(rr(ps[:K]), rr(ps[:K]), rr(ps[:K]), rr(ps[:K])) for _ in range(B)]
    cts = [(aoa.Ciphertext.from_residues(ctx, x[0], x[1], slots=N // 2, scale=1 << SCALE_BITS),
            aoa.Ciphertext.from_residues(ctx, x[2], x[3], slots=N // 2, scale=1 << SCALE_BITS)) for x in host_in]
    outs = [aoa.Ciphertext(ctx) for _ in range(B)]

    A = [x[0] for x in cts]
    Bs = [x[1] for x in cts]

    def step(mode="batch", dom=aoa.AOA_NTT):
        for a, b in cts:
            a.set(K - 1, N // 2, 1 << SCALE_BITS, dom)
            b.set(K - 1, N // 2, 1 << SCALE_BITS, dom)
        if mode == "batch":
            aoa.ckks_mul_batch(ctx, outs, A, Bs, evk)
        else:
            for (a, b), o in zip(cts, outs):
                (aoa.ckks_mul_plain if mode == "plain" else aoa.ckks_mul)(ctx, o, a, b, evk)

    def barrier():
        torch.cuda.synchronize()
        ctx.sync()
        replicas.barrier(pg)

    def maxt(ms):
        return replicas.max_over_ranks(ms, pg, device="cuda")

    # ---- device-resident throughput -------------------------------------------
    for _ in range(max(3, args.warmup)):
        step()
    barrier()
    clocks = ClockSampler(local)
    clocks.start()
    time.sleep(0.3)
    l0 = aoa.kernel_launches()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier()
    e0.record(stream)
    for _ in range(args.steps):
        step()
    e1.record(stream)
    barrier()
    launches = aoa.kernel_launches() - l0
    clk = clocks.stop()
    ms = maxt(e0.elapsed_time(e1))
    ms_step = ms / args.steps
    value = replicas.job_rate(B * args.steps, world, ms)

    def timed(fn, steps):
        fn()
        barrier()
        s0, s1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s0.record(stream)
        for _ in range(steps):
            fn()
        s1.record(stream)
        barrier()
        return maxt(s0.elapsed_time(s1)) / steps

    # the plain per-call path (reference op sequence) on the same batch
    plain_ms = timed(lambda: step("plain", dom=aoa.AOA_COEF), max(2, args.steps // 2))
    percall_ms = timed(lambda: step("per_call"), max(2, args.steps // 2))
    coef_ms = timed(lambda: step(dom=aoa.AOA_COEF), max(2, args.steps // 2))

    # ---- per-call latency (plain per-call path, one op at a time) -------------
    lat = []
    (a0, b0), o0 = cts[0], outs[0]
    for _ in range(max(20, args.steps)):
        a0.set(K - 1, N // 2, 1 << SCALE_BITS, aoa.AOA_NTT)
        b0.set(K - 1, N // 2, 1 << SCALE_BITS, aoa.AOA_NTT)
        s0, s1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s0.record(stream)
        aoa.ckks_mul(ctx, o0, a0, b0, evk)
        s1.record(stream)
        s1.synchronize()
        lat.append(s0.elapsed_time(s1))
    lat = np.array(lat)

    # ---- transform throughput: 256 polys x 30 limbs, forward then inverse ----------
    npolys = 256
    buf = ctx.alloc((npolys, K, N))
    xs = rr(ps[:K])
    for p in range(npolys):
        aoa.capi.check(aoa.capi.load().aoa_memcpy_h2d(ctx.handle, buf.offset(p * K * N), aoa.capi.ptr(xs), xs.nbytes))
    for _ in range(3):
        ctx.ntt_fwd(buf, npolys, 0, K)
        ctx.ntt_inv(buf, npolys, 0, K)
    barrier()
    reps = 5
    t0, t1, t2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
    t0.record(stream)
    for _ in range(reps):
        ctx.ntt_fwd(buf, npolys, 0, K)
    t1.record(stream)
    for _ in range(reps):
        ctx.ntt_inv(buf, npolys, 0, K)
    t2.record(stream)
    barrier()
    fwd_ms = t0.elapsed_time(t1) / reps
    inv_ms = t1.elapsed_time(t2) / reps
    # inverse(forward(x)) == x on the first and last poly, forward == oracle on one poly
    lib_ = aoa.capi.load()
    chk = np.empty((K, N), dtype=np.uint64)
    roundtrip_ok = True
    for p in (0, npolys - 1):
        aoa.capi.check(lib_.aoa_memcpy_d2h(ctx.handle, aoa.capi.ptr(chk), buf.offset(p * K * N), chk.nbytes))
        ctx.sync()
        roundtrip_ok = roundtrip_ok and bool(np.array_equal(chk, xs))
    ctx.ntt_fwd(buf, 1, 0, K)
    aoa.capi.check(lib_.aoa_memcpy_d2h(ctx.handle, aoa.capi.ptr(chk), buf.ptr, chk.nbytes))
    ctx.sync()
    ntt_cpu = None
    fwd_matches_oracle = None
    if rank == 0 and not args.no_cpu_baseline:
        import oracle
        from oracle import Oracle
        oracle.lib().oc_set_threads(os.cpu_count() or 1)
        o_ntt = Oracle(N, ps[:K], ps[K:])
        tc = time.perf_counter()
        want = o_ntt.ntt_fwd(xs)
        tc = time.perf_counter() - tc
        fwd_matches_oracle = bool(np.array_equal(chk, want))
        ntt_cpu = {"value": 16 * K * N / tc / 1e9, "unit": "GB/s", "cores": os.cpu_count() or 1, "kind": "port",
                   "sample": "forward transform of one 30-limb poly (oracle, OpenMP)"}
    ctx.ntt_inv(buf, 1, 0, K)
    # the DGT on the same data (folded to 2^15 Gaussian integers per limb)
    d0, d1, d2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
    ctx.dgt_fwd(buf, npolys, 0, K)
    ctx.dgt_inv(buf, npolys, 0, K)
    barrier()
    d0.record(stream)
    ctx.dgt_fwd(buf, npolys, 0, K)
    d1.record(stream)
    ctx.dgt_inv(buf, npolys, 0, K)
    d2.record(stream)
    barrier()
    dgt256_fwd_ms, dgt256_inv_ms = d0.elapsed_time(d1), d1.elapsed_time(d2)
    aoa.capi.check(lib_.aoa_memcpy_d2h(ctx.handle, aoa.capi.ptr(chk), buf.offset((npolys - 1) * K * N), chk.nbytes))
    ctx.sync()
    dgt_roundtrip_ok = bool(np.array_equal(chk, xs))
    algo_bytes = 16 * npolys * K * N          # read + write every coefficient once
    achieved = algo_bytes / (fwd_ms / 1000.0) / 1e9
    peak, peak_src = measured_peaks()
    traffic = None
    issue = None
    tfile = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tfile):
        with open(tfile) as f:
            tj = json.load(f)
        if "ntt_fwd_bytes_per_coef" in tj:
            traffic = tj["ntt_fwd_bytes_per_coef"] * npolys * K * N
        if "ntt_fwd_warp_instructions_per_limb" in tj:
            # the transform is bound by integer issue: the same launch against
            # the SMs' instruction issue peak (4 schedulers x 1 warp instruction
            # per clock per SM), at the SM clock sampled during the timed region
            wi = tj["ntt_fwd_warp_instructions_per_limb"] * npolys * K
            issue = {"warp_instructions": wi, "achieved_per_s": wi / (fwd_ms / 1000.0), "seconds": fwd_ms / 1000.0,
                     "source": "warp instructions per limb from an ncu capture of the same forward transform"}
            if "ntt_fwd_fma_pipe_cycles_per_limb" in tj:
                issue["fma_pipe_cycles"] = tj["ntt_fwd_fma_pipe_cycles_per_limb"] * npolys * K
    del buf

    # ---- DGT variant: transform rate and per-call HMult on a DGT context -----------
    ctxd = aoa.Context(E)
    ctxd.set_transform(aoa.AOA_DGT)
    streamd = torch.cuda.ExternalStream(ctxd.stream)

    def timed_on(st, c, fn, steps):
        fn()
        c.sync()
        s0, s1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s0.record(st)
        for _ in range(steps):
            fn()
        s1.record(st)
        c.sync()
        torch.cuda.synchronize()
        return maxt(s0.elapsed_time(s1)) / steps

    # the 256 x 30-limb transforms on the largest 60-bit primes q = 1 mod 2N
    # (general Shoup remainder), same shapes and defaults
    from aoa_b200 import params as params_
    gen_primes = params_.ntt_primes(60, 2 << LOG_N, K + 1)
    ctxg = aoa.Context(aoa.Engine(LOG_N, gen_primes[:K], gen_primes[K:], scale_bits=SCALE_BITS))
    streamg = torch.cuda.ExternalStream(ctxg.stream)
    gbuf = ctxg.alloc((npolys, K, N))
    xg = rr(gen_primes[:K])
    for p in range(npolys):
        aoa.capi.check(lib_.aoa_memcpy_h2d(ctxg.handle, gbuf.offset(p * K * N), aoa.capi.ptr(xg), xg.nbytes))
    gen_fwd_ms = timed_on(streamg, ctxg, lambda: ctxg.ntt_fwd(gbuf, npolys, 0, K), reps)
    gen_inv_ms = timed_on(streamg, ctxg, lambda: ctxg.ntt_inv(gbuf, npolys, 0, K), reps)
    del gbuf, ctxg

    dbuf = ctxd.alloc((8, K, N))
    dgt_fwd_ms = timed_on(streamd, ctxd, lambda: ctxd.dgt_fwd(dbuf, 8, 0, K), 5)
    dgt_inv_ms = timed_on(streamd, ctxd, lambda: ctxd.dgt_inv(dbuf, 8, 0, K), 5)
    dgt_bytes = 16 * 8 * K * N
    del dbuf
    evk_d = aoa.SwitchKey(ctxd, rr(ps), rr(ps), domain=aoa.AOA_COEF)

    def dgt_step():
        for (a, b), o in zip(cts, outs):
            a.set(K - 1, N // 2, 1 << SCALE_BITS, aoa.AOA_DGT)
            b.set(K - 1, N // 2, 1 << SCALE_BITS, aoa.AOA_DGT)
            aoa.ckks_mul(ctxd, o, a, b, evk_d)
    dgt_hmult_ms = timed_on(streamd, ctxd, dgt_step, max(2, args.steps // 2))

    def dgt_batch_step():
        for a, b in cts:
            a.set(K - 1, N // 2, 1 << SCALE_BITS, aoa.AOA_DGT)
            b.set(K - 1, N // 2, 1 << SCALE_BITS, aoa.AOA_DGT)
        aoa.ckks_mul_batch(ctxd, outs, A, Bs, evk_d)
    dgt_batch_ms = timed_on(streamd, ctxd, dgt_batch_step, max(2, args.steps // 2))
    # encoder: N/2 slots encoded into K limbs and decoded from limb 0
    vals = rng.uniform(-1, 1, N // 2) + 1j * rng.uniform(-1, 1, N // 2)
    t0 = time.perf_counter()
    for _ in range(5):
        m_enc, _ = aoa.ckks_encode(ctx, vals, scale=1 << SCALE_BITS)
        ctx.sync()
    enc_ms = (time.perf_counter() - t0) / 5 * 1000.0
    t0 = time.perf_counter()
    for _ in range(5):
        aoa.ckks_decode(ctx, m_enc, N // 2, 1 << SCALE_BITS)
    dec_ms = (time.perf_counter() - t0) / 5 * 1000.0

    # ---- batched uneven workload and serving loop ----------------------------------
    uneven = serving = None
    if not args.no_systems and world == 1:
        uneven, serving = systems_workloads(aoa, torch)

    # ---- end to end through the C ABI with host buffers -----------------------------
    # Every step uploads its B input pairs from pinned host memory, runs the
    # batched HMult + relinearise + rescale and queues the B results' copy
    # back (coefficient domain); steps alternate between two contexts
    # (streams), so one step's copies overlap the other's arithmetic, as a
    # serving loop would (three contexts measured slower: 668 vs ~700/s, the
    # copies in both directions share the host link).  All copies are inside
    # the timed region.
    lib = aoa.capi.load()
    pin_in = [aoa.PinnedArray((2, K, N)) for _ in range(2 * B)]
    for i, x in enumerate(host_in):
        pin_in[2 * i].array[0], pin_in[2 * i].array[1] = x[0], x[1]
        pin_in[2 * i + 1].array[0], pin_in[2 * i + 1].array[1] = x[2], x[3]
    lanes = []
    nlanes = 2
    for lane in range(nlanes):
        c2 = ctx if lane == 0 else aoa.Context(E)
        ins = [(aoa.Ciphertext(c2), aoa.Ciphertext(c2)) for _ in range(B)]
        los = [aoa.Ciphertext(c2) for _ in range(B)]
        pouts = [aoa.PinnedArray((2, K - 1, N)) for _ in range(B)]
        lanes.append((c2, ins, los, pouts, torch.cuda.ExternalStream(c2.stream)))

    def e2e_step(lane):
        c2, ins, los, pouts, _ = lanes[lane]
        for i, (a, b) in enumerate(ins):
            aoa.capi.check(lib.aoa_ct_upload(c2.handle, a.handle, pin_in[2 * i].ptr, K, aoa.AOA_COEF))
            aoa.capi.check(lib.aoa_ct_upload(c2.handle, b.handle, pin_in[2 * i + 1].ptr, K, aoa.AOA_COEF))
            a.set(K - 1, N // 2, 1 << SCALE_BITS, aoa.AOA_COEF)
            b.set(K - 1, N // 2, 1 << SCALE_BITS, aoa.AOA_COEF)
        aoa.ckks_mul_batch(c2, los, [x[0] for x in ins], [x[1] for x in ins], evk)
        for o, po in zip(los, pouts):
            aoa.capi.check(lib.aoa_ct_download_async(c2.handle, o.handle, po.ptr, K - 1, aoa.AOA_COEF))

    for lane in range(nlanes):
        e2e_step(lane)
    for lane in lanes:
        lane[0].sync()
    barrier()
    e2e_steps = max(2 * nlanes, args.steps // nlanes * nlanes)
    q0 = torch.cuda.Event(enable_timing=True)
    q_end = [torch.cuda.Event(enable_timing=True) for _ in lanes]
    q0.record(lanes[0][4])
    for lane in lanes[1:]:
        lane[4].wait_event(q0)
    for st_i in range(e2e_steps):
        e2e_step(st_i % nlanes)
    for ev, lane in zip(q_end, lanes):
        ev.record(lane[4])
    for lane in lanes:
        lane[0].sync()
    barrier()
    e2e_ms = maxt(max(q0.elapsed_time(ev) for ev in q_end))
    e2e_value = replicas.job_rate(B * e2e_steps, world, e2e_ms)
    h2d = B * 2 * 2 * K * N * 8
    d2h = B * 2 * (K - 1) * N * 8
    # the host-to-device copy rate alone (one step's uploads on one stream),
    # the ceiling of the end-to-end rate: h2d bytes per step / this rate
    c0, ins0 = lanes[0][0], lanes[0][1]
    h0, h1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    h0.record(lanes[0][4])
    for i, (a, b) in enumerate(ins0):
        aoa.capi.check(lib.aoa_ct_upload(c0.handle, a.handle, pin_in[2 * i].ptr, K, aoa.AOA_COEF))
        aoa.capi.check(lib.aoa_ct_upload(c0.handle, b.handle, pin_in[2 * i + 1].ptr, K, aoa.AOA_COEF))
    h1.record(lanes[0][4])
    c0.sync()
    h2d_gbs = h2d / (h0.elapsed_time(h1) * 1e-3) / 1e9
    # both directions at once, as in a step of the steady state: one step's
    # uploads on lane 0 and one step's downloads on lane 1, started together;
    # the host link's combined rate bounds the end-to-end rate
    c1, los1, pouts1, st1 = lanes[1][0], lanes[1][2], lanes[1][3], lanes[1][4]
    d0, d1 = torch.cuda.Event(enable_timing=True), [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    d0.record(lanes[0][4])
    st1.wait_event(d0)
    for i, (a, b) in enumerate(ins0):
        aoa.capi.check(lib.aoa_ct_upload(c0.handle, a.handle, pin_in[2 * i].ptr, K, aoa.AOA_COEF))
        aoa.capi.check(lib.aoa_ct_upload(c0.handle, b.handle, pin_in[2 * i + 1].ptr, K, aoa.AOA_COEF))
    for o, po in zip(los1, pouts1):
        aoa.capi.check(lib.aoa_ct_download_async(c1.handle, o.handle, po.ptr, K - 1, o.domain))
    d1[0].record(lanes[0][4])
    d1[1].record(st1)
    c0.sync()
    c1.sync()
    duplex_gbs = (h2d + d2h) / (max(d0.elapsed_time(e) for e in d1) * 1e-3) / 1e9
    # the last lane-0 result equals a per-call HMult of the same host inputs
    x = host_in[0]
    a1 = aoa.Ciphertext.from_residues(ctx, x[0], x[1], slots=N // 2, scale=1 << SCALE_BITS)
    b1 = aoa.Ciphertext.from_residues(ctx, x[2], x[3], slots=N // 2, scale=1 << SCALE_BITS)
    o1 = aoa.Ciphertext(ctx)
    aoa.ckks_mul(ctx, o1, a1, b1, evk)
    w0, w1 = o1.download(nlimbs=K - 1, domain=aoa.AOA_COEF)
    got = lanes[0][3][0].array
    e2e_check = bool(np.array_equal(got[0], w0) and np.array_equal(got[1], w1))

    # ---- CPU baseline (rank 0, N = 1): the oracle's reference op sequence ------
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        import oracle
        from oracle import Oracle
        threads = os.cpu_count() or 1
        oracle.lib().oc_set_threads(threads)
        o = Oracle(N, ps[:K], ps[K:])
        x = host_in[0]
        ek = (rr(ps), rr(ps))
        o.hmult((x[0], x[1]), (x[2], x[3]), ek, K - 1, 1 << SCALE_BITS, 1 << SCALE_BITS)   # warm
        n_cpu, tc = 0, time.perf_counter()
        while n_cpu < 2 or time.perf_counter() - tc < 10.0:
            o.hmult((x[0], x[1]), (x[2], x[3]), ek, K - 1, 1 << SCALE_BITS, 1 << SCALE_BITS)
            n_cpu += 1
            if n_cpu >= 20:
                break
        tc = time.perf_counter() - tc
        cpu = {"value": n_cpu / tc, "unit": UNIT, "cores": threads, "kind": "port",
               "sample": "%d HMult+relin+rescale on the same N=2^16, k=30, kl=31 workload "
                         "(reference op sequence, oracle/ckks_oracle.cpp, OpenMP)" % n_cpu}

    acc = None
    if rank == 0:
        from aoa_b200 import params
        p52 = params.ntt_primes(52, 2 << 12, 7)
        ref_q, ref_b = reference_layout_n4096()
        acc = {"plain_ckks_n4096": accuracy(aoa, 12, p52[:3], p52[3:], 40, seed=7),
               "plain_ckks_n4096_scale52": accuracy(aoa, 12, p52[:3], p52[3:], 52, seed=7),
               "reference_layout_n4096_scale52": accuracy(aoa, 12, ref_q, ref_b, 52, seed=7),
               "reference_layout_n4096_scale40": accuracy(aoa, 12, ref_q, ref_b, 40, seed=7),
               "hmult_n65536": accuracy(aoa, LOG_N, ps[:K], ps[K:], SCALE_BITS, seed=8),
               "reference": "decoded HMult+relin+rescale product vs the FP64 cleartext product (numpy)"}
        if cpu is not None:
            acc["cpu_chain_n4096"] = cpu_chain(p52[:3], p52[3:], 40)
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "u64", "data": "synthetic",
            "config": dict(workload_config(B), input_domain="transform (state left by the previous HMult)",
                           transform_tuning=tuning),
            "accuracy": acc,
            "latency_ms": {"p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99)),
                           "single_op_ops_per_s": float(1000.0 / np.mean(lat))},
            "plain_per_call": {"ops_per_s": world * B / (plain_ms / 1000.0),
                               "path": "reference ckks_mul op sequence (aoa_hmult_plain), coefficient inputs",
                               "speedup_of_value": value / (world * B / (plain_ms / 1000.0))},
            "pipeline_per_call_ops_per_s": world * B / (percall_ms / 1000.0),
            "batched_coefficient_inputs_ops_per_s": world * B / (coef_ms / 1000.0),
            "speedup_vs_plain": {
                "transform_domain_inputs": value / (world * B / (plain_ms / 1000.0)),
                "coefficient_inputs": plain_ms / coef_ms,
                "note": "plain path: reference op sequence with coefficient inputs; batched path with the "
                        "inputs its previous HMult leaves (transform domain) and with the same coefficient inputs"},
            "ntt": {"fwd_ms": fwd_ms, "inv_ms": inv_ms, "polys": npolys, "limbs": K,
                    "fwd_gbs": achieved, "inv_gbs": algo_bytes / (inv_ms / 1000.0) / 1e9,
                    "hbm_frac": achieved / peak, "inverse_of_forward_is_identity": roundtrip_ok,
                    "forward_equals_oracle": fwd_matches_oracle, "cpu_baseline": ntt_cpu,
                    "dgt_fwd_gbs": algo_bytes / (dgt256_fwd_ms / 1000.0) / 1e9,
                    "dgt_inv_gbs": algo_bytes / (dgt256_inv_ms / 1000.0) / 1e9,
                    "dgt_inverse_of_forward_is_identity": dgt_roundtrip_ok,
                    "general_primes": {"primes": "largest 60-bit q = 1 mod 2^17 (general Shoup remainder)",
                                       "fwd_gbs": algo_bytes / (gen_fwd_ms / 1000.0) / 1e9,
                                       "inv_gbs": algo_bytes / (gen_inv_ms / 1000.0) / 1e9}},
            "dgt": {"fwd_ms": dgt_fwd_ms, "inv_ms": dgt_inv_ms, "polys": 8, "limbs": K,
                    "fwd_gbs": dgt_bytes / (dgt_fwd_ms / 1000.0) / 1e9,
                    "inv_gbs": dgt_bytes / (dgt_inv_ms / 1000.0) / 1e9,
                    "hmult_per_call_ops_per_s": world * B / (dgt_hmult_ms / 1000.0),
                    "hmult_batched_ops_per_s": world * B / (dgt_batch_ms / 1000.0),
                    "path": "aoa-dgt ckks_mul on a DGT context (GI tensor and key products), inputs in the DGT domain; "
                            "batched: ckks_mul_batch of the same %d pairs on the DGT context" % B},
            "encoder": {"slots": N // 2, "limbs": K, "encode_ms_host_to_device": enc_ms,
                        "decode_ms_device_to_host": dec_ms},
            "uneven_batch": uneven,
            "serving": serving,
            "roofline": {"kernel": "ntt forward (column + row kernel pair), N=2^16", "bound": "hbm",
                         "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                         "peak_source": peak_src, "algorithmic_bytes": algo_bytes, "traffic": traffic},
            "issue_roofline": issue_roofline(issue, clk, torch.cuda.get_device_properties(local).multi_processor_count),
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                    "h2d_copy_gbs": h2d_gbs, "h2d_bound_ops_per_s": B * h2d_gbs * 1e9 / h2d,
                    "duplex_copy_gbs": duplex_gbs, "link_bound_ops_per_s": B * duplex_gbs * 1e9 / (h2d + d2h),
                    "path": "aoa_ct_upload (pinned) + aoa_hmult_batch + aoa_ct_download_async (coefficients) "
                            "per step, steps alternating over two contexts (streams)",
                    "result_equals_per_call": e2e_check},
            "gpu_launches": launches,
            "clocks": clk,
            "cpu_baseline": cpu,
        }
        print(json.dumps(line), flush=True)
    replicas.finish(pg)


if __name__ == "__main__":
    main()
