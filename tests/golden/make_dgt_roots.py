#!/usr/bin/env python3
"""Extract the reference DGT evaluator's primes, generators and GI roots.

The DGT variant (aoa-dgt) folds a degree-n polynomial into n/2 Gaussian
integers and twists them by powers of a fixed root r of i in GF(p)[i] with
r^(n/2) = i before its length-n/2 transform (compute_nthroot, aoa-dgt
src/cuda/dgt.cu).  r is not derived: it is looked up in a generated table,
NTHROOT[p][n/2] (aoa-dgt src/arithmetic/coprimes.cu), so bit-exact parity of
transform-domain values needs those numbers.  This script reads the table as
text and writes a JSON fixture: a prefix of each prime bucket, each prime's
generator (PROOTS) and its roots for every tabulated size.  INVNTHROOT is not
stored: it is the unique inverse of r, which the reference asserts.  It runs
only where the reference checkout exists; the fixture it wrote is committed.

Usage: python tests/golden/make_dgt_roots.py REFERENCE_ROOT
"""
import json
import os
import re
import sys

KEEP = {63: 1, 55: 40, 52: 30, 48: 40, 45: 40}


def main():
    if len(sys.argv) != 2:
        sys.exit("usage: %s REFERENCE_ROOT (the pdroalves/aoa checkout)" % sys.argv[0])
    root = sys.argv[1]
    src = open(os.path.join(root, "aoa-dgt/src/arithmetic/coprimes.cu")).read()
    i0 = src.index("std::map<uint64_t, std::map<int, GaussianInteger>> NTHROOT")
    i1 = src.index("std::map<uint64_t, std::map<int, GaussianInteger>> INVNTHROOT")
    roots, cur = {}, None
    for line in src[i0:i1].splitlines():
        m = re.match(r"\s*\{\(uint64_t\)(\d+), \{\s*$", line)
        if m:
            cur = roots.setdefault(int(m.group(1)), {})
            continue
        m = re.match(r"\s*\{(\d+), \(GaussianInteger\)\{\(uint64_t\)(\d+), \(uint64_t\)(\d+)\}\}", line)
        if m and cur is not None:
            cur[int(m.group(1))] = [int(m.group(2)), int(m.group(3))]
    pr_src = src[src.index("std::map<uint64_t, int> PROOTS"):]
    proots = {int(a): int(b) for a, b in re.findall(r"\{\(uint64_t\)(\d+), (\d+)\}", pr_src)}
    out = {"source": "aoa-dgt/src/arithmetic/coprimes.cu", "buckets": {}, "proots": {}, "nthroot": {}}
    for bits, n in KEEP.items():
        m = re.search(r"COPRIMES_%d_BUCKET\[\] = \{(.*?)\};" % bits, src, re.S)
        vals = [int(x) for x in re.sub(r"\s", "", m.group(1)).split(",") if x][:n]
        out["buckets"][str(bits)] = vals
        for q in vals:
            out["proots"][str(q)] = proots[q]
            out["nthroot"][str(q)] = {str(s): v for s, v in sorted(roots[q].items())}
    dst = os.path.join(os.path.dirname(os.path.abspath(__file__)), "dgt_roots.json")
    with open(dst, "w") as f:
        json.dump(out, f, separators=(",", ":"))
        f.write("\n")
    print("wrote", dst, {b: len(v) for b, v in out["buckets"].items()})


if __name__ == "__main__":
    main()
