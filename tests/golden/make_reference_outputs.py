#!/usr/bin/env python3
"""Golden outputs of the reference evaluator's own kernels.

oracle/_ref/ref_harness runs pdroalves/aoa's aoa-ntt transform and RNS
kernels (built from its sources by oracle/ref/Makefile, where the reference
checkout exists) through the reference's API on seeded inputs.  This script
runs it on one GPU for each configuration below and packs its outputs into
tests/golden/reference_outputs.npz, which tests/test_oracle_reference_outputs.py
compares with the oracle (the inputs are regenerated there from the seeds the
harness documents, so the fixture holds outputs only).

oracle/_ref/ref_ckks_harness runs the reference's CKKS layer (HMult with and
without rescale, rotation, conjugation, addition, subtraction and the encoder
on seeded operands; then its own key generation, encryption, HMult, rotation
and decryption) for CKKS_CONFIGS; its records go to
tests/golden/reference_ckks_outputs.npz (tests/test_oracle_reference_ckks.py).

oracle/_ref/ref_dgt_harness runs aoa-dgt's DGT (single-kernel and
hierarchical), its product, and ModUp / ModDown / rescale on its DGT engine
for DGT_CONFIGS; its records go to tests/golden/reference_dgt_outputs.npz
(tests/test_oracle_reference_dgt.py).  oracle/_ref/ref_dgt_ckks_harness runs
aoa-dgt's CKKS layer with ref_ckks_harness's records for DGT_CKKS_CONFIGS
(tests/golden/reference_dgt_ckks_outputs.npz, tests/test_gpu_reference_dgt.py).

Usage (on a machine with a GPU and the built harnesses):
    python tests/golden/make_reference_outputs.py OUT_DIR
writes OUT_DIR/reference_outputs.npz, reference_ckks_outputs.npz,
reference_dgt_outputs.npz, reference_dgt_ckks_outputs.npz and
reference_digests.json (copy them into tests/golden/).  The digests are the
reference's ckks_mul and rotation at the headline shape (N = 2^16, 30 + 31
primes) on the seeded operands of the CKKS records, each output limb reduced
to a position-weighted sum, from both variants (ref_ckks_harness and
ref_dgt_ckks_harness --digest).
"""
import json
import os
import subprocess
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
HARNESS = os.path.join(ROOT, "oracle", "_ref", "ref_harness")
CKKS_HARNESS = os.path.join(ROOT, "oracle", "_ref", "ref_ckks_harness")
DGT_HARNESS = os.path.join(ROOT, "oracle", "_ref", "ref_dgt_harness")
DGT_CKKS_HARNESS = os.path.join(ROOT, "oracle", "_ref", "ref_dgt_ckks_harness")

# (log2 N, k, kl, prec, transforms only): the reference's hierarchical
# transforms at 2^10 (32 x 32) and 2^12 (64 x 64) on its own prime choice
# (a 63-bit q0, then its 55- or 52-bit bucket; special primes from the
# 55-bit bucket), ModUp / ModDown / rescale at 2^10
CONFIGS = [(10, 4, 5, 55, 0), (12, 3, 4, 52, 1)]
TAGS = {1: "ntt_fwd", 2: "ntt_inv", 3: "modup", 4: "moddown", 5: "rescale", 6: "modup_max", 7: "ntt_fwd_max"}

# (log2 nphi, k, kl, prec, transforms only) of the DGT records: aoa-dgt's
# single-kernel DGT at nphi = 2^10 (512 Gaussian integers) with its product,
# ModUp / ModDown / rescale on the DGT engine, and its hierarchical DGT at
# 2^13 (64 x 64)
DGT_CONFIGS = [(10, 3, 4, 45, 0), (13, 2, 2, 48, 1)]
DGT_TAGS = {1: "dgt_fwd", 2: "dgt_inv", 3: "mul", 4: "modup", 5: "moddown", 6: "rescale"}

# (log2 N, k, kl, prec) of the CKKS-layer records (aoa-ntt, then aoa-dgt)
CKKS_CONFIGS = [(10, 4, 5, 55)]
DGT_CKKS_CONFIGS = [(10, 4, 4, 48)]
# (log2 N, k, kl, prec) of the full-shape digests (ckks_mul and a rotation at
# the headline shape, too large to keep whole)
DIGEST_CONFIGS = [(16, 30, 31, 55)]
CKKS_TAGS = {20: "hmult_l%d", 21: "hmult_norescale_l%d", 23: "conjugate_l%d", 24: "add_l%d", 25: "sub_l%d",
             26: "encode_s%d", 40: "sk", 41: "evk", 42: "enc300", 43: "enc301", 44: "mul_keys", 45: "dec300",
             46: "dec_mul", 47: "rot1_keys", 48: "dec_rot1"}


def parse(path, magic=b"AOAREF01", tags=TAGS):
    w = np.fromfile(path, dtype=np.uint64)
    assert w[:1].tobytes() == magic, "not a harness output"
    N, k, kl, prec = (int(v) for v in w[1:5])
    primes = w[5:5 + k + kl].copy()
    at = 5 + k + kl
    recs = {}
    while at < w.size:
        tag, level, n = (int(v) for v in w[at:at + 3])
        recs["%s_l%d" % (tags[tag], level)] = w[at + 3:at + 3 + n].copy()
        at += 3 + n
    return N, k, kl, prec, primes, recs


def parse_ckks(path, magic=b"AOAREF02"):
    """Records of ref_ckks_harness / ref_dgt_ckks_harness; ciphertext records
    keep their [aux, scale, slots, c0 limbs, c1 limbs] words."""
    w = np.fromfile(path, dtype=np.uint64)
    assert w[:1].tobytes() == magic, "not a CKKS harness output"
    N, k, kl, prec = (int(v) for v in w[1:5])
    primes = w[5:5 + k + kl].copy()
    at = 5 + k + kl
    recs = {}
    while at < w.size:
        tag, level, n = (int(v) for v in w[at:at + 3])
        words = w[at + 3:at + 3 + n].copy()
        if tag == 22:
            name = "rotate%d_l%d" % (int(words[0]), level)
        else:
            name = CKKS_TAGS[tag] % level if "%d" in CKKS_TAGS[tag] else CKKS_TAGS[tag]
        assert name not in recs, name
        recs[name] = words
        at += 3 + n
    return N, k, kl, prec, primes, recs


def main():
    if len(sys.argv) != 2:
        sys.exit(__doc__)
    out_dir = sys.argv[1]
    os.makedirs(out_dir, exist_ok=True)
    arrays = {}
    for log_n, k, kl, prec, tonly in CONFIGS:
        path = os.path.join(out_dir, "ref_n%d.bin" % (1 << log_n))
        subprocess.check_call([HARNESS, path, str(log_n), str(k), str(kl), str(prec), str(tonly)])
        N, k2, kl2, prec2, primes, recs = parse(path)
        tag = "n%d" % N
        arrays[tag + "_params"] = np.array([N, k2, kl2, prec2], dtype=np.uint64)
        arrays[tag + "_primes"] = primes
        for name, v in recs.items():
            arrays["%s_%s" % (tag, name)] = v
    dst = os.path.join(out_dir, "reference_outputs.npz")
    np.savez_compressed(dst, **arrays)
    print("wrote", dst, sorted(arrays))
    arrays = {}
    for log_n, k, kl, prec in CKKS_CONFIGS:
        path = os.path.join(out_dir, "ref_ckks_n%d.bin" % (1 << log_n))
        subprocess.check_call([CKKS_HARNESS, path, str(log_n), str(k), str(kl), str(prec)])
        N, k2, kl2, prec2, primes, recs = parse_ckks(path)
        tag = "n%d" % N
        arrays[tag + "_params"] = np.array([N, k2, kl2, prec2], dtype=np.uint64)
        arrays[tag + "_primes"] = primes
        for name, v in recs.items():
            arrays["%s_%s" % (tag, name)] = v
    dst = os.path.join(out_dir, "reference_ckks_outputs.npz")
    np.savez_compressed(dst, **arrays)
    print("wrote", dst, sorted(arrays))
    arrays = {}
    for log_n, k, kl, prec, tonly in DGT_CONFIGS:
        path = os.path.join(out_dir, "ref_dgt_n%d.bin" % (1 << log_n))
        subprocess.check_call([DGT_HARNESS, path, str(log_n), str(k), str(kl), str(prec), str(tonly)])
        N, k2, kl2, prec2, primes, recs = parse(path, b"AOAREF03", DGT_TAGS)
        tag = "n%d" % N
        arrays[tag + "_params"] = np.array([N, k2, kl2, prec2], dtype=np.uint64)
        arrays[tag + "_primes"] = primes
        for name, v in recs.items():
            arrays["%s_%s" % (tag, name)] = v
    dst = os.path.join(out_dir, "reference_dgt_outputs.npz")
    np.savez_compressed(dst, **arrays)
    print("wrote", dst, sorted(arrays))
    arrays = {}
    for log_n, k, kl, prec in DGT_CKKS_CONFIGS:
        path = os.path.join(out_dir, "ref_dgt_ckks_n%d.bin" % (1 << log_n))
        subprocess.check_call([DGT_CKKS_HARNESS, path, str(log_n), str(k), str(kl), str(prec)])
        N, k2, kl2, prec2, primes, recs = parse_ckks(path, b"AOAREF04")
        tag = "n%d" % N
        arrays[tag + "_params"] = np.array([N, k2, kl2, prec2], dtype=np.uint64)
        arrays[tag + "_primes"] = primes
        for name, v in recs.items():
            arrays["%s_%s" % (tag, name)] = v
    dst = os.path.join(out_dir, "reference_dgt_ckks_outputs.npz")
    np.savez_compressed(dst, **arrays)
    print("wrote", dst, sorted(arrays))
    digests = []
    for log_n, k, kl, prec in DIGEST_CONFIGS:
        for variant, harness in (("aoa-ntt", CKKS_HARNESS), ("aoa-dgt", DGT_CKKS_HARNESS)):
            out = subprocess.run([harness, "--digest", str(log_n), str(k), str(kl), str(prec)], check=True,
                                 capture_output=True, text=True).stdout
            rec = json.loads([l for l in out.splitlines() if l.startswith("{")][-1])
            rec["variant"] = variant
            digests.append(rec)
    dst = os.path.join(out_dir, "reference_digests.json")
    with open(dst, "w") as f:
        json.dump(digests, f)
        f.write("\n")
    print("wrote", dst)


if __name__ == "__main__":
    main()
