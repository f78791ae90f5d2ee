// AOADGT/ckks.h — drop-in shim for callers of the reference's DGT evaluator.
//
// aoa-dgt (library AOADGT) keeps newckks's evaluator names and signatures
// (aoa-dgt include/AOADGT/ckks.h:23-304) on the Gaussian-integer DGT; its
// parameter set comes from CUDAEngine::init(k, kl, M, t)
// (include/AOADGT/cuda/cudaengine.h:93-107: M the cyclotomic index 2N, t the
// CKKS scaling factor).  This header is the newckks shim with every context
// on this library's DGT transform (aoa_ctx_set_transform(ctx, AOA_DGT)):
// results in coefficients are the NTT evaluator's, DGT-domain values are the
// reference's for the twist roots the engine was given (aoa_params.dgt_roots;
// without them the engine derives its own root of i, which changes
// DGT-domain values only).
#pragma once
#define AOA_SHIM_TRANSFORM AOA_DGT
#include "../newckks/ckks/ckks.h"

struct CUDAEngine {
  // init(k, kl, M, t): ring degree N = M / 2, scale 2^t; kl <= 0 means k + 1
  static void init(int k, int kl, int M, uint64_t t) { CUDAManager::init(k, kl, M / 2, (int)t); }
  static void init(int k, int kl, int M, uint64_t t, const std::vector<uint64_t>& primes) {
    CUDAManager::init(k, kl, M / 2, (int)t, primes);
  }
  static void destroy() { CUDAManager::destroy(); }
};
