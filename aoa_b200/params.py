"""Parameter sets: prime selection for the engine (host only).

* ntt_primes(bits, modulus, count): the `count` largest `bits`-bit primes
  q = 1 mod `modulus` (2N for ring degree N), descending — the prime rule used
  for the 60-bit workloads, which the reference's tables do not contain.
* reference_prime_set(table, k, kl, prec): the Q / B primes the reference's
  CUDAManager::init(k, kl, N, prec) would select (fill_ckks_coprimes_bucket,
  aoa-ntt src/cuda/manager.cu:426-464) from a prime table the caller supplies
  in the JSON layout {"buckets": {"63": [...], "55": [...], ...}} (its own copy
  of the reference's COPRIMES_*_BUCKET tables).
"""
import numpy as np

from . import capi


def ntt_primes(bits, modulus, count):
    out = np.zeros(count, dtype=np.uint64)
    n = capi.load().aoa_search_primes(bits, modulus, count, out.ctypes.data_as(capi.u64p))
    if n < count:
        raise ValueError("only %d primes of %d bits with q = 1 mod %d" % (max(n, 0), bits, modulus))
    return [int(v) for v in out]


def primitive_root(q):
    return int(capi.load().aoa_primitive_root(q))


def reference_prime_set(table, k, kl, prec):
    b = table["buckets"]
    q0 = int(b["63"][0])
    if prec in (45, 55):
        bucket = [int(v) for v in b[str(prec)]]
        return [q0] + bucket[: k - 1], bucket[k - 1: k - 1 + kl]
    if prec in (48, 52):
        return [q0] + [int(v) for v in b[str(prec)][: k - 1]], [int(v) for v in b["55"][:kl]]
    raise ValueError("the reference supports prec 45, 48, 52 and 55 only")
