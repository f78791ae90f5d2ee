#!/usr/bin/env python3
"""Extract the reference's RNS prime buckets and primitive roots into a fixture.

The reference evaluator picks its primes from fixed tables (aoa-ntt
src/cuda/htrans/coprimes.cu: COPRIMES_{45,48,52,55,63}_BUCKET and the PROOTS map)
following fill_ckks_coprimes_bucket (aoa-ntt src/cuda/manager.cu:426-464):
q0 = first 63-bit prime, then the prec-bit bucket for Q, then B primes.  The
primes fix the NTT twiddles, so bit-exact parity "on the reference prime set"
needs these numbers.  This script reads the table as text and writes a small
JSON fixture (a prefix of each bucket plus the generators); it runs only where
the reference checkout exists, the fixture it wrote is committed.

Usage: python tests/golden/make_reference_primes.py REFERENCE_ROOT
"""
import json
import os
import re
import sys

KEEP = {63: 4, 55: 128, 52: 30, 48: 64, 45: 32}


def main():
    if len(sys.argv) != 2:
        sys.exit("usage: %s REFERENCE_ROOT (the pdroalves/aoa checkout)" % sys.argv[0])
    root = sys.argv[1]
    src = open(os.path.join(root, "aoa-ntt/src/cuda/htrans/coprimes.cu")).read()
    proots = {int(a): int(b) for a, b in re.findall(r"\{\(uint64_t\)(\d+), (\d+)\}", src)}
    out = {"source": "aoa-ntt/src/cuda/htrans/coprimes.cu", "buckets": {}, "proots": {}}
    for bits, n in KEEP.items():
        m = re.search(r"COPRIMES_%d_BUCKET\[\] = \{(.*?)\};" % bits, src, re.S)
        vals = [int(x) for x in re.sub(r"\s", "", m.group(1)).split(",")][:n]
        out["buckets"][str(bits)] = vals
        for q in vals:
            out["proots"][str(q)] = proots[q]
    dst = os.path.join(os.path.dirname(os.path.abspath(__file__)), "reference_primes.json")
    with open(dst, "w") as f:
        json.dump(out, f, separators=(",", ":"))
        f.write("\n")
    print("wrote", dst, {b: len(v) for b, v in out["buckets"].items()})


if __name__ == "__main__":
    main()
