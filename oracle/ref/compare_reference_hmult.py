#!/usr/bin/env python3
"""HMult + relinearise + rescale, and the limb transforms: the reference's own
CUDA evaluators against this engine, on one GPU and the same primes.

Runs oracle/_ref/ref_ckks_harness in its timing mode (pdroalves/aoa aoa-ntt's
ckks_mul, built from its sources by oracle/ref/Makefile: seeded ciphertexts at
level k - 1, inputs left in the transform domain after the first call, host
clock around a device-synchronised loop), then times this engine on the
primes the reference chose: per-call ckks_mul, the reference's op sequence on
this engine's kernels (ckks_mul_plain), and batched HMult of 16 products
(CUDA events on the context's stream).  The reference supports a 63-bit q0
and 45/48/52/55-bit buckets only, so the comparison runs on its 55-bit set
(this engine runs the 63-bit q0's limbs with strict butterflies, the rest
lazy).
Transforms: oracle/_ref/ref_harness and ref_dgt_harness in their timing modes
run aoa-ntt's NTT (COMMONEngine::execute) and aoa-dgt's DGT
(DGTEngine::execute_dgt) one call per poly over `--polys` polys of k limbs,
forward then inverse; this engine runs the same shapes with ntt_fwd / ntt_inv
and dgt_fwd / dgt_inv over the whole batch (its DGT roots derived from the
primes).  Comparison tooling beside the fixture harnesses: it is not the
benchmark (bench.py) and nothing in the product runs it.

Usage (GPU machine, harness built):
    python oracle/ref/compare_reference_hmult.py [--log-n 16 --k 30 --kl 31 --prec 55 --reps 20]
prints one JSON line.
"""
import argparse
import json
import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
HARNESS = os.path.join(ROOT, "oracle", "_ref", "ref_ckks_harness")
NTT_HARNESS = os.path.join(ROOT, "oracle", "_ref", "ref_harness")
DGT_HARNESS = os.path.join(ROOT, "oracle", "_ref", "ref_dgt_harness")


def engine_times(log_n, q, b, reps, batch=16):
    sys.path.insert(0, ROOT)
    import torch
    import aoa_b200 as aoa
    E = aoa.Engine(log_n, q, b, scale_bits=40)
    ctx = aoa.Context(E)
    N, k = E.N, E.k
    rng = np.random.default_rng(1)
    res = lambda primes: np.array([rng.integers(0, p, N, dtype=np.uint64) for p in primes], dtype=np.uint64)
    evk = aoa.SwitchKey(ctx, res(q + b), res(q + b))
    st = torch.cuda.ExternalStream(ctx.stream)

    def pairs(n):
        return [(aoa.Ciphertext.from_residues(ctx, res(q), res(q), slots=N // 2, scale=1 << 40, domain=aoa.AOA_NTT),
                 aoa.Ciphertext.from_residues(ctx, res(q), res(q), slots=N // 2, scale=1 << 40, domain=aoa.AOA_NTT))
                for _ in range(n)]

    def timed(fn, n_iter):
        for _ in range(3):
            fn()
        ctx.sync()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        for _ in range(n_iter):
            fn()
        e1.record(st)
        ctx.sync()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / n_iter

    def reset(ps):
        for a, bb in ps:
            a.set(k - 1, N // 2, 1 << 40, aoa.AOA_NTT)
            bb.set(k - 1, N // 2, 1 << 40, aoa.AOA_NTT)

    one = pairs(1)
    out = aoa.Ciphertext(ctx)

    def per_call():
        reset(one)
        aoa.ckks_mul(ctx, out, one[0][0], one[0][1], evk)

    def plain():
        reset(one)
        aoa.ckks_mul_plain(ctx, out, one[0][0], one[0][1], evk)

    many = pairs(batch)
    outs = [aoa.Ciphertext(ctx) for _ in range(batch)]

    def batched():
        reset(many)
        aoa.ckks_mul_batch(ctx, outs, [p[0] for p in many], [p[1] for p in many], evk)

    return {"per_call_ms": timed(per_call, reps), "reference_sequence_ms": timed(plain, reps),
            "batched_ms_per_hmult": timed(batched, max(1, reps // 4)) / batch, "batch": batch,
            "lazy_primes": "%d of %d" % (sum(p < (1 << 60) for p in q + b), len(q + b))}


def run_json(cmd):
    out = subprocess.run(cmd, check=True, capture_output=True, text=True).stdout
    return json.loads([l for l in out.splitlines() if l.startswith("{")][-1])


def engine_transforms(log_n, primes, polys, dgt):
    sys.path.insert(0, ROOT)
    import torch
    import aoa_b200 as aoa
    k = len(primes)
    E = aoa.Engine(log_n, primes, [])
    ctx = aoa.Context(E)
    N = E.N
    rng = np.random.default_rng(2)
    big = ctx.alloc((polys, k, N))
    host = np.array([rng.integers(0, q, N, dtype=np.uint64) for q in primes], dtype=np.uint64)
    for p in range(polys):
        aoa.capi.check(aoa.capi.load().aoa_memcpy_h2d(ctx.handle, big.offset(p * k * N), aoa.capi.ptr(host),
                                                      host.nbytes))
    fwd, inv = (ctx.dgt_fwd, ctx.dgt_inv) if dgt else (ctx.ntt_fwd, ctx.ntt_inv)
    st = torch.cuda.ExternalStream(ctx.stream)
    fwd(big, polys, 0, k)
    inv(big, polys, 0, k)
    ctx.sync()
    e = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
    e[0].record(st)
    fwd(big, polys, 0, k)
    e[1].record(st)
    inv(big, polys, 0, k)
    e[2].record(st)
    ctx.sync()
    torch.cuda.synchronize()
    f, i = e[0].elapsed_time(e[1]), e[1].elapsed_time(e[2])
    by = 16.0 * polys * k * N
    big.free()
    return {"fwd_ms": f, "inv_ms": i, "fwd_gbs": by / f / 1e6, "inv_gbs": by / i / 1e6}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--log-n", type=int, default=16)
    ap.add_argument("--k", type=int, default=30)
    ap.add_argument("--kl", type=int, default=31)
    ap.add_argument("--prec", type=int, default=55)
    ap.add_argument("--reps", type=int, default=20)
    ap.add_argument("--polys", type=int, default=256)
    ap.add_argument("--what", default="hmult", help="hmult, ntt or dgt")
    a = ap.parse_args()
    if a.what in ("ntt", "dgt"):
        harness = NTT_HARNESS if a.what == "ntt" else DGT_HARNESS
        ref = run_json([harness, "--time", str(a.log_n), str(a.k), "1", str(a.prec), str(a.polys)])
        primes = [int(p) for p in ref.pop("primes")]
        ours = engine_transforms(a.log_n, primes, a.polys, a.what == "dgt")
        print(json.dumps({"workload": "%s forward + inverse, %d polys x %d limbs at N=2^%d (the reference's "
                                      "%d-bit set, 63-bit q0)" % (a.what.upper(), a.polys, a.k, a.log_n, a.prec),
                          "reference": ref, "engine": ours,
                          "speedup_fwd": ref["fwd_ms"] / ours["fwd_ms"], "speedup_inv": ref["inv_ms"] / ours["inv_ms"]}))
        return
    ref = run_json([HARNESS, "--time", str(a.log_n), str(a.k), str(a.kl), str(a.prec), str(a.reps)])
    primes = [int(p) for p in ref.pop("primes")]
    ours = engine_times(a.log_n, primes[:a.k], primes[a.k:], a.reps)
    line = {"workload": "HMult+relin+rescale, N=2^%d, %d Q + %d special primes (the reference's %d-bit set, "
                        "63-bit q0), level %d, inputs in the transform domain"
                        % (a.log_n, a.k, a.kl, a.prec, a.k - 1),
            "reference": {"ms_per_hmult": ref["ms_per_hmult"], "reps": ref["reps"],
                          "path": "aoa-ntt ckks_mul (its own CUDA kernels), host clock, device synchronised"},
            "engine": ours,
            "speedup_per_call": ref["ms_per_hmult"] / ours["per_call_ms"],
            "speedup_batched": ref["ms_per_hmult"] / ours["batched_ms_per_hmult"]}
    print(json.dumps(line))


if __name__ == "__main__":
    main()
