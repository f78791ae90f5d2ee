#!/usr/bin/env python3
"""Generate the committed golden vectors from the independent Python model
(tests/pymodel.py), not from the oracle or the CUDA library.

  ntt_n1024.npz : N=1024, reference prime set (q0 + 55-bit bucket, k=3, kl=1),
                  seeded uniform residues x and their transform X (closed form).
  rns_n64.npz   : N=64, reference primes k=4, kl=3: ModUp / ModDown / rescale
                  inputs and outputs at level 3.

Usage: python tests/golden/make_golden.py
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
from tests import pymodel  # noqa: E402


def ref_set(table, k, kl):
    b = table["buckets"]
    return [b["63"][0]] + b["55"][: k - 1], b["55"][k - 1: k - 1 + kl]


def psi_of(q, g, n):
    return pow(g, (q - 1) // (2 * n), q)


def main():
    table = json.load(open(os.path.join(HERE, "reference_primes.json")))
    rng = np.random.default_rng(20240601)
    # --- NTT vectors
    N = 1024
    Q, B = ref_set(table, 3, 1)
    primes = Q + B
    x = np.array([rng.integers(0, q, N, dtype=np.uint64) for q in primes], dtype=np.uint64)
    X = np.array([pymodel.ntt_closed_form([int(v) for v in x[r]], q, psi_of(q, table["proots"][str(q)], N))
                  for r, q in enumerate(primes)], dtype=np.uint64)
    np.savez_compressed(os.path.join(HERE, "ntt_n1024.npz"), primes=np.array(primes, dtype=np.uint64), x=x, X=X)
    # --- RNS vectors
    N, k, kl, level = 64, 4, 3, 3
    Q, B = ref_set(table, k, kl)
    xq = [[int(rng.integers(0, q)) for _ in range(N)] for q in Q]
    xb = [[int(rng.integers(0, b)) for _ in range(N)] for b in B]
    up = pymodel.modup(xq, Q, B, level)
    down = pymodel.moddown(xq, xb, Q, B, level)
    resc = pymodel.rescale(xq, Q, level)
    np.savez_compressed(os.path.join(HERE, "rns_n64.npz"),
                        q=np.array(Q, dtype=np.uint64), b=np.array(B, dtype=np.uint64),
                        xq=np.array(xq, dtype=np.uint64), xb=np.array(xb, dtype=np.uint64),
                        modup=np.array(up, dtype=np.uint64), moddown=np.array(down, dtype=np.uint64),
                        rescale=np.array(resc, dtype=np.uint64), level=level)
    print("golden vectors written")


if __name__ == "__main__":
    main()
