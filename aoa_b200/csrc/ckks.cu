// CKKS ciphertext objects and the key-switching operations (HMult +
// relinearisation + rescale, rotation, conjugation, add/sub, rescale) behind
// the C ABI.  Semantics follow the reference evaluator (aoa-ntt
// src/ckks/ckks.cpp); residues of every output limb <= level are identical to
// the reference's.  The pipeline differs: it is level aware (only limbs
// 0..level and the kl special limbs are touched), keeps the transform-domain
// d2 for the Q part of the extended key-switch input instead of transforming
// it back and forth, and multiplies with the key in one kernel.
#include <cstring>

#include <functional>

#include "aoa_internal.h"

using namespace aoa;

namespace aoa {

// Workspace for one key switch / HMult at the engine's largest level (words):
//   D   [3][k]       tensor outputs d0 d1 d2 (transform domain)
//   T   [k]          coefficient-domain copy of the key-switch input
//   UB  [kl]         ModUp output (B limbs)
//   KS  [2][k + kl]  key products: Q limbs transform domain, B limbs coefficients
//   L4  [4]          single limbs (d0_l, d1_l, k0_l, k1_l) for the merged rescale
//   CL  [2]          c_l, limb l of the product in coefficients
//   Y   [2][k]       ModDown corrections
//   R0  [k]          automorphism of c0
struct Workspace {
  uint64_t *D, *T, *UB, *KS, *L4, *CL, *Y, *R0;
};

size_t workspace_words(const Engine& E) {
  return (size_t)E.N * (3 * E.k + E.k + std::max(E.kl, 1) + 2 * (E.k + E.kl) + 4 + 2 + 2 * E.k + E.k);
}

Workspace carve(const Engine& E, uint64_t* p) {
  const size_t limb = (size_t)E.N;
  Workspace w;
  w.D = p; p += 3 * E.k * limb;
  w.T = p; p += E.k * limb;
  w.UB = p; p += std::max(E.kl, 1) * limb;
  w.KS = p; p += 2 * (E.k + E.kl) * limb;
  w.L4 = p; p += 4 * limb;
  w.CL = p; p += 2 * limb;
  w.Y = p; p += 2 * E.k * limb;
  w.R0 = p;
  return w;
}

static Workspace get_ws(Ctx& C) {
  const size_t need = workspace_words(*C.E) * sizeof(uint64_t);
  if (C.scratch_bytes < need) {
    if (C.scratch) AOA_CUDA(cudaFreeAsync(C.scratch, C.stream));
    C.scratch = nullptr;
    C.scratch_bytes = 0;
    cudaError_t e = cudaMallocAsync(&C.scratch, need, C.stream);
    if (e != cudaSuccess) {
      cudaGetLastError();
      throw AoaError(AOA_ERR_OOM, "workspace allocation failed");
    }
    C.scratch_bytes = need;
  }
  return carve(*C.E, (uint64_t*)C.scratch);
}

// Limb transforms of the given kind (AOA_NTT: negacyclic NTT of aoa-ntt;
// AOA_DGT: folded Gaussian-integer DGT of aoa-dgt) on [npolys][stride][N].
void xform(const Engine& E, int kind, uint64_t* d, int npolys, int first_prime, int nlimbs, long stride, bool fwd,
           cudaStream_t st) {
  if (kind == AOA_DGT) dgt_batch(E, d, npolys, first_prime, nlimbs, stride, fwd, st);
  else ntt_batch(E, d, npolys, first_prime, nlimbs, stride, fwd, st);
}

// Brings limbs 0..nlimbs-1 of both polys of ct to `domain` in place.
void ct_to_domain(Ctx& C, aoa_ct* ct, int domain, int nlimbs) {
  const Engine& E = *C.E;
  if (ct->domain == domain) return;
  if (ct->domain != AOA_COEF) xform(E, ct->domain, ct->d, 2, 0, nlimbs, E.k, false, C.stream);
  if (domain != AOA_COEF) xform(E, domain, ct->d, 2, 0, nlimbs, E.k, true, C.stream);
  ct->domain = domain;
}

static void to_domain(Ctx& C, aoa_ct* ct, int domain, int nlimbs) { ct_to_domain(C, ct, domain, nlimbs); }

static void copy_limbs(Ctx& C, uint64_t* dst, const uint64_t* src, long words) {
  AOA_CUDA(cudaMemcpyAsync(dst, src, (size_t)words * 8, cudaMemcpyDeviceToDevice, C.stream));
}

// Key-switch core on the Q limbs 0..level of x, given in both domains
// (x_coef, x_ntt).  Leaves in w.KS = [x*b | x*a] (stride k + kl limbs): the Q
// limbs in the transform domain, the kl B limbs back in coefficients.
// (ModUp poly_modup, key products poly_mul, ckks.cpp:309-314.)
// Fused transform ends (out-of-place inverse, key products, key-switch
// combine; engine knob "fuse", a bit mask) on NTT contexts; DGT contexts take
// the separate kernels.
static bool fused(const Ctx& C, int what) { return C.transform == AOA_NTT && (C.E->tune.fuse & what); }

// Forward transform of the corrections Y (npolys polys of stride k limbs,
// limbs 0..nlimbs-1) with the key-switch combine as its epilogue.
static void combine_into(Ctx& C, uint64_t* Y, int npolys, int nlimbs, const uint64_t* base, long base_stride,
                         int base_polys, const uint64_t* KS, long ks_stride, int rescale_level, uint64_t* out,
                         long out_stride, const OutPtrs* outp, cudaStream_t st = nullptr) {
  const Engine& E = *C.E;
  NttIo io;
  io.epi.mode = kEpiCombine;
  io.epi.base = base;
  io.epi.base_stride = base_stride;
  io.epi.base_polys = base ? base_polys : 0;
  io.epi.ks = KS;
  io.epi.ks_stride = ks_stride;
  io.epi.binv = E.rns.moddown_binv;
  io.epi.resc = rescale_level > 0 ? E.rns.resc_inv + (long)rescale_level * E.k : nullptr;
  if (outp) {
    io.epi.use_ptrs = 1;
    io.epi.outp = *outp;
  } else {
    io.epi.out = out;
    io.epi.out_stride = out_stride;
  }
  ntt_batch_io(E, Y, npolys, 0, nlimbs, E.k, true, io, st ? st : C.stream);
}

static void keyswitch_core(Ctx& C, const Workspace& w, const uint64_t* x_coef, const uint64_t* x_ntt,
                           const aoa_swk* key, int level) {
  const Engine& E = *C.E;
  const long N = E.N;
  const int m = level + 1;
  const int tk = C.transform;
  if (key->domain != tk) throw AoaError(AOA_ERR_BAD_PARAM, "the switching key is in another transform domain");
  modup(E, x_coef, 0, w.UB, 0, 1, level, C.stream);
  const long ks = (long)(E.k + E.kl) * N;
  if (fused(C, kFuseKeyProduct)) {
    // forward transform of the special limbs with the key products as its epilogue
    NttIo io;
    io.epi.mode = kEpiKeyProduct;
    io.epi.out = w.KS + (long)m * N;
    io.epi.out_poly1 = ks;
    io.epi.key = key->d;
    io.epi.key_half = (long)E.nprimes * N;
    ntt_batch_io(E, w.UB, 1, E.k, E.kl, E.kl, true, io, C.stream);
    keyswitch_mul_op(E, x_ntt, nullptr, key->d, w.KS, w.KS + ks, m, C.stream, 0);
  } else {
    xform(E, tk, w.UB, 1, E.k, E.kl, E.kl, true, C.stream);
    if (tk == AOA_DGT) gi_keyswitch_mul_op(E, x_ntt, w.UB, key->d, w.KS, w.KS + ks, m, C.stream);
    else keyswitch_mul_op(E, x_ntt, w.UB, key->d, w.KS, w.KS + ks, m, C.stream);
  }
  xform(E, tk, w.KS + (long)m * N, 2, E.k, E.kl, E.k + E.kl, false, C.stream);
}

static uint64_t scale_after_mult(const Engine& E, uint64_t sa, uint64_t sb, int level) {
  unsigned __int128 p = (unsigned __int128)sa * sb;            // ckks.cpp:328-330
  return (uint64_t)(p / E.primes[level]);
}

// Finishes a key switch whose products sit in w.KS and writes the transform
// domain result to out (2 polys of stride `half`):
//   rescale:  out = Rescale(base + ModDown(KS))   (limbs 0..level-1)
//   else:     out = base + ModDown(KS)            (limbs 0..level)
// base = [b0 | b1] (stride `half`, transform domain) or b1 == nullptr (zero).
static void keyswitch_finish(Ctx& C, const Workspace& w, uint64_t* out, long half, const uint64_t* b0,
                             const uint64_t* b1, int level, bool do_rescale) {
  const Engine& E = *C.E;
  const long N = E.N;
  const int m = level + 1;
  const long ks_stride = (long)(E.k + E.kl) * N;
  const uint64_t* kb = w.KS + (long)m * N;
  if (do_rescale) {
    // u_l = limb l of (base + k B^-1) in coefficients, for both polys
    uint64_t* U = w.L4;
    if (b0 && b1 == b0 + half) {
      ks_combine(E, U, N, b0 + (long)level * N, half, w.KS + (long)level * N, ks_stride, nullptr, 0, 1, 2, 0,
                 C.stream, level);
    } else {
      ks_combine(E, U, 0, b0 ? b0 + (long)level * N : nullptr, 0, w.KS + (long)level * N, 0, nullptr, 0, 1, 1,
                 0, C.stream, level);
      ks_combine(E, U + N, 0, b1 ? b1 + (long)level * N : nullptr, 0, w.KS + ks_stride + (long)level * N, 0,
                 nullptr, 0, 1, 1, 0, C.stream, level);
    }
    xform(E, C.transform, U, 2, level, 1, 1, false, C.stream);
    rescale_corrections(E, kb, ks_stride, U, N, w.CL, N, w.Y, (long)E.k * N, 2, level, C.stream);
    if (fused(C, kFuseCombine) && (!b1 || b1 == b0 + half)) {
      combine_into(C, w.Y, 2, level, b0, half, b1 ? 2 : 1, w.KS, ks_stride, level, out, half, nullptr);
      return;
    }
    xform(E, C.transform, w.Y, 2, 0, level, E.k, true, C.stream);
    if (b0 && b1 == b0 + half) {
      ks_combine(E, out, half, b0, half, w.KS, ks_stride, w.Y, (long)E.k * N, level, 2, level, C.stream);
    } else {
      ks_combine(E, out, 0, b0, 0, w.KS, 0, w.Y, 0, level, 1, level, C.stream);
      ks_combine(E, out + half, 0, b1, 0, w.KS + ks_stride, 0, w.Y + (long)E.k * N, 0, level, 1, level, C.stream);
    }
  } else {
    moddown_conv(E, kb, ks_stride, w.Y, (long)E.k * N, 2, m, C.stream);
    if (fused(C, kFuseCombine) && (!b1 || b1 == b0 + half)) {
      combine_into(C, w.Y, 2, m, b0, half, b1 ? 2 : 1, w.KS, ks_stride, 0, out, half, nullptr);
      return;
    }
    xform(E, C.transform, w.Y, 2, 0, m, E.k, true, C.stream);
    if (b0 && b1 == b0 + half) {
      ks_combine(E, out, half, b0, half, w.KS, ks_stride, w.Y, (long)E.k * N, m, 2, 0, C.stream);
    } else {
      ks_combine(E, out, 0, b0, 0, w.KS, 0, w.Y, 0, m, 1, 0, C.stream);
      ks_combine(E, out + half, 0, b1, 0, w.KS + ks_stride, 0, w.Y + (long)E.k * N, 0, m, 1, 0, C.stream);
    }
  }
}

// HMult + relinearisation (ckks_mul_without_rescale, ckks.cpp:273-332),
// optionally followed by the rescale of ckks_mul (ckks.cpp:334-347).
// Transform-domain pipeline: tensor, one inverse transform of d2 for ModUp,
// the key products, inverse transforms of their B limbs only, and ModDown
// merged with the rescale (one forward transform per output limb).  The
// result is left in the transform domain (the reference leaves coefficients;
// the residues of every live limb are the same after a domain change).
static void hmult_core(Ctx& C, const Workspace& w, aoa_ct* out, aoa_ct* a, aoa_ct* b, const aoa_swk* evk,
                       bool do_rescale) {
  const Engine& E = *C.E;
  const long N = E.N;
  const int level = std::min(a->level, b->level);
  const int m = level + 1;
  const long half = (long)E.k * N;
  // operands to the transform domain, in place (poly_mul does the same, poly_t.cpp:201-220)
  const int tk = C.transform;
  to_domain(C, a, tk, a->level + 1);
  if (b != a) to_domain(C, b, tk, b->level + 1);
  uint64_t* D0 = w.D;
  uint64_t* D2 = w.D + 2 * half;
  if (tk == AOA_DGT) gi_tensor_op(E, a->d, half, b->d, half, D0, D0 + half, D2, m, C.stream);
  else tensor_op(E, a->d, half, b->d, half, D0, D0 + half, D2, m, C.stream);
  const uint64_t sa = a->scale, sb = b->scale;
  const int slots = a->slots;
  if (fused(C, kFuseSource)) {
    NttIo io;                                  // inverse of d2 read in place of a copy
    io.src = D2;
    io.src_poly_stride = m;
    ntt_batch_io(E, w.T, 1, 0, m, m, false, io, C.stream);
  } else {
    copy_limbs(C, w.T, D2, (long)m * N);
    xform(E, tk, w.T, 1, 0, m, m, false, C.stream);
  }
  keyswitch_core(C, w, w.T, D2, evk, level);
  keyswitch_finish(C, w, out->d, half, D0, D0 + half, level, do_rescale);
  out->level = do_rescale ? level - 1 : level;
  out->slots = slots;
  out->scale = scale_after_mult(E, sa, sb, level);
  out->domain = tk;
}

static void hmult_check(const Engine& E, const aoa_ct* a, const aoa_ct* b, const aoa_swk* evk) {
  if (a->level == 0 || b->level == 0)
    throw AoaError(AOA_ERR_LEVEL_EXHAUSTED, "The ciphertext level is 0. No more rescaling is possible.");
  if (a->slots != b->slots) throw AoaError(AOA_ERR_SLOT_MISMATCH, "Ciphertexts must have the same number of slots.");
  if (!evk || !evk->d) throw AoaError(AOA_ERR_NO_KEY, "missing relinearisation key");
  if (E.kl == 0) throw AoaError(AOA_ERR_BAD_PARAM, "key switching needs special primes (kl > 0)");
}

void hmult(Ctx& C, aoa_ct* out, aoa_ct* a, aoa_ct* b, const aoa_swk* evk, bool do_rescale) {
  hmult_check(*C.E, a, b, evk);
  hmult_core(C, get_ws(C), out, a, b, evk, do_rescale);
}

// Same pipeline on caller-provided scratch of workspace_words(E) words.
void hmult_with_scratch(Ctx& C, aoa_ct* out, aoa_ct* a, aoa_ct* b, const aoa_swk* evk, bool do_rescale,
                        uint64_t* scratch) {
  hmult_check(*C.E, a, b, evk);
  hmult_core(C, carve(*C.E, scratch), out, a, b, evk, do_rescale);
}

// Galois automorphism X -> X^g followed by the key switch with `key`
// (ckks_rotate_left/right, ckks.cpp:953-1009; ckks_conjugate, ckks.cpp:1011-1040).
// The automorphism is applied in the transform domain as a permutation of the
// evaluation points (the reference permutes coefficients with a sign).
void apply_galois(Ctx& C, aoa_ct* out, aoa_ct* in, long galois, const aoa_swk* key) {
  const Engine& E = *C.E;
  const long N = E.N;
  if (!key || !key->d) throw AoaError(AOA_ERR_NO_KEY, "missing switching key for this automorphism");
  if (E.kl == 0) throw AoaError(AOA_ERR_BAD_PARAM, "key switching needs special primes (kl > 0)");
  const int level = in->level, m = level + 1;
  const long half = (long)E.k * N;
  Workspace w = get_ws(C);
  uint64_t* X = w.D + 2 * half;
  const int slots = in->slots;
  const uint64_t scale = in->scale;
  const int tk = C.transform;
  if (tk == AOA_DGT) {
    // Galois maps do not permute the DGT's evaluation points: apply X -> X^g
    // to the coefficients (as the reference does, aoa-dgt src/tool/encoder.cu:
    // 338-470) and transform the results.
    to_domain(C, in, AOA_COEF, m);
    automorph_coef_op(E, w.R0, in->d, 0, galois, m, 1, C.stream);
    automorph_coef_op(E, w.T, in->d + half, 0, galois, m, 1, C.stream);
    copy_limbs(C, X, w.T, (long)m * N);
    xform(E, tk, X, 1, 0, m, m, true, C.stream);
    xform(E, tk, w.R0, 1, 0, m, m, true, C.stream);
  } else {
    to_domain(C, in, AOA_NTT, m);
    automorph_ntt_op(E, w.R0, in->d, 0, galois, m, 1, C.stream);
    automorph_ntt_op(E, X, in->d + half, 0, galois, m, 1, C.stream);
    if (fused(C, kFuseSource)) {
      NttIo io;                                // inverse read out of place
      io.src = X;
      io.src_poly_stride = m;
      ntt_batch_io(E, w.T, 1, 0, m, m, false, io, C.stream);
    } else {
      copy_limbs(C, w.T, X, (long)m * N);
      ntt_batch(E, w.T, 1, 0, m, m, false, C.stream);
    }
  }
  keyswitch_core(C, w, w.T, X, key, level);
  keyswitch_finish(C, w, out->d, half, w.R0, nullptr, level, false);
  out->level = level;
  out->slots = slots;
  out->scale = scale;
  out->domain = tk;
}

// Batched HMult (+ relinearise + rescale) of n <= kMaxBatch independent
// products at one level: every pipeline stage is one launch over the whole
// batch (transforms over n x limbs items, conversions over n x polys, the
// element-wise kernels over n ciphertexts), so small per-op stages no longer
// leave the GPU idle.  Batch workspace layout (N-word limbs):
//   D [3][n][k]  T [n][k]  UB [n][kl]  KS [2][n][k+kl]  U [2][n]  CL [2][n]  Y [2][n][k]
static size_t batch_words(const Engine& E, int n) {
  return (size_t)E.N * n * (8 * E.k + 3 * std::max(E.kl, 1) + 4);
}

static void hmult_batch_group(Ctx& C, cudaStream_t st, void*& ws, size_t& ws_bytes, int n, aoa_ct* const* out,
                              aoa_ct* const* a, aoa_ct* const* b, const aoa_swk* evk, bool do_rescale, int level) {
  const Engine& E = *C.E;
  const long N = E.N;
  const int m = level + 1, k = E.k, kl = E.kl;
  const long half = (long)k * N, ks = (long)(k + kl) * N;
  const size_t need = batch_words(E, n) * 8;
  if (ws_bytes < need) {
    if (ws) AOA_CUDA(cudaFreeAsync(ws, st));
    ws = nullptr;
    ws_bytes = 0;
    if (cudaMallocAsync(&ws, need, st) != cudaSuccess) {
      cudaGetLastError();
      throw AoaError(AOA_ERR_OOM, "batch workspace allocation failed");
    }
    ws_bytes = need;
  }
  uint64_t* p = (uint64_t*)ws;
  uint64_t* D = p;  p += 3L * n * half;
  uint64_t* T = p;  p += (long)n * half;
  uint64_t* UB = p; p += (long)n * kl * N;
  uint64_t* KS = p; p += 2L * n * ks;
  uint64_t* U = p;  p += 2L * n * N;
  uint64_t* CL = p; p += 2L * n * N;
  uint64_t* Y = p;
  CtPtrs ptr;
  uint64_t sa[kMaxBatch], sb[kMaxBatch];
  int slots[kMaxBatch];
  for (int z = 0; z < n; z++) {                 // operands are in the transform domain already
    ptr.a[z] = a[z]->d;
    ptr.b[z] = b[z]->d;
    sa[z] = a[z]->scale;
    sb[z] = b[z]->scale;
    slots[z] = a[z]->slots;
  }
  // the DGT context (aoa-dgt, ckks.cpp:275-360) runs the same pipeline on its
  // transform with Gaussian-integer products; the fused transform ends are NTT only
  const int tk = C.transform;
  uint64_t* D2 = D + 2L * n * half;
  if (tk == AOA_DGT) {
    gi_tensor_batch_op(E, ptr, half, D, n, m, st);
  } else {
    tensor_batch_op(E, ptr, half, D, n, m, st);
  }
  const int fuse = tk == AOA_NTT ? E.tune.fuse : 0;
  if (fuse & kFuseSource) {
    NttIo io;                                  // inverse of d2 read in place of a copy
    io.src = D2;
    io.src_poly_stride = k;
    ntt_batch_io(E, T, n, 0, m, k, false, io, st);
  } else {
    AOA_CUDA(cudaMemcpy2DAsync(T, half * 8, D2, half * 8, (size_t)m * N * 8, n, cudaMemcpyDeviceToDevice, st));
    xform(E, tk, T, n, 0, m, k, false, st);
  }
  modup(E, T, half, UB, (long)kl * N, n, level, st);
  if (tk == AOA_DGT) {
    xform(E, tk, UB, n, k, kl, kl, true, st);
    gi_keyswitch_mul_batch_op(E, D2, half, UB, (long)kl * N, evk->d, KS, ks, n, m, st);
  } else if (fuse & kFuseKeyProduct) {
    NttIo io;                                  // special-limb transform with the key products fused
    io.epi.mode = kEpiKeyProduct;
    io.epi.out = KS + (long)m * N;
    io.epi.out_stride = ks;
    io.epi.out_poly1 = (long)n * ks;
    io.epi.key = evk->d;
    io.epi.key_half = (long)E.nprimes * N;
    ntt_batch_io(E, UB, n, k, kl, kl, true, io, st);
    keyswitch_mul_batch_op(E, D2, half, nullptr, 0, evk->d, KS, ks, n, m, st, 0);
  } else {
    ntt_batch(E, UB, n, k, kl, kl, true, st);
    keyswitch_mul_batch_op(E, D2, half, UB, (long)kl * N, evk->d, KS, ks, n, m, st);
  }
  xform(E, tk, KS + (long)m * N, 2 * n, k, kl, k + kl, false, st);
  OutPtrs outp;
  for (int z = 0; z < n; z++) {
    outp.p[z] = out[z]->d;
    outp.p[n + z] = out[z]->d + half;
  }
  if (do_rescale) {
    ks_combine(E, U, N, D + (long)level * N, half, KS + (long)level * N, ks, nullptr, 0, 1, 2 * n, 0, st, level);
    xform(E, tk, U, 2 * n, level, 1, 1, false, st);
    rescale_corrections(E, KS + (long)m * N, ks, U, N, CL, N, Y, half, 2 * n, level, st);
    if (fuse & kFuseCombine) {
      combine_into(C, Y, 2 * n, level, D, half, 2 * n, KS, ks, level, nullptr, 0, &outp, st);
    } else {
      xform(E, tk, Y, 2 * n, 0, level, k, true, st);
      ks_combine_ptr(E, outp, D, half, KS, ks, Y, half, level, 2 * n, level, st);
    }
  } else {
    moddown_conv(E, KS + (long)m * N, ks, Y, half, 2 * n, m, st);
    if (fuse & kFuseCombine) {
      combine_into(C, Y, 2 * n, m, D, half, 2 * n, KS, ks, 0, nullptr, 0, &outp, st);
    } else {
      xform(E, tk, Y, 2 * n, 0, m, k, true, st);
      ks_combine_ptr(E, outp, D, half, KS, ks, Y, half, m, 2 * n, 0, st);
    }
  }
  for (int z = 0; z < n; z++) {
    out[z]->level = do_rescale ? level - 1 : level;
    out[z]->slots = slots[z];
    out[z]->scale = scale_after_mult(E, sa[z], sb[z], level);
    out[z]->domain = tk;
  }
}

// Runs `group(stream, workspace, bytes, count, outs, as, bs, level)` over groups of
// equal level (at most kMaxBatch ops each).  With the engine's two streams, a
// group of 8 or more runs as two halves on the context's two streams, and
// smaller groups go whole to the stream with less queued work (ops x limbs),
// so the groups of a mix of levels overlap on the device; each stream keeps
// its own stream-ordered workspace.  If an output of an op on one stream is an
// operand or an output of an op on the other, every group runs on one stream.
template <class F>
static void run_grouped(Ctx& C, int n, aoa_ct* const* out, aoa_ct* const* a, aoa_ct* const* b,
                        const std::function<int(int)>& lvl, F&& group) {
  const Engine& E = *C.E;
  std::vector<int> idx(n);
  for (int z = 0; z < n; z++) idx[z] = z;
  std::stable_sort(idx.begin(), idx.end(), [&](int x, int y) { return lvl(x) > lvl(y); });
  std::vector<aoa_ct*> go(n), ga(n), gb(n);
  for (int t = 0; t < n; t++) {
    go[t] = out[idx[t]];
    ga[t] = a[idx[t]];
    gb[t] = b ? b[idx[t]] : a[idx[t]];
  }
  struct Unit {
    int s, e, stream;
  };
  std::vector<Unit> groups, units;
  for (int s = 0; s < n;) {
    int e = s;
    while (e < n && lvl(idx[e]) == lvl(idx[s]) && e - s < kMaxBatch) e++;
    groups.push_back({s, e, 0});
    s = e;
  }
  bool use_aux = false;
  if (E.tune.batch_streams == 2) {
    double queued[2] = {0, 0};
    for (const Unit& g : groups) {
      const int cnt = g.e - g.s;
      const double cost = (double)cnt * (lvl(idx[g.s]) + 1);
      if (cnt >= 8) {
        units.push_back({g.s, g.s + cnt / 2, 0});
        units.push_back({g.s + cnt / 2, g.e, 1});
        queued[0] += cost / 2;
        queued[1] += cost / 2;
      } else {
        const int st = queued[1] < queued[0] ? 1 : 0;
        units.push_back({g.s, g.e, st});
        queued[st] += cost;
      }
    }
    for (const Unit& u : units) use_aux = use_aux || u.stream == 1;
  }
  if (use_aux) {                      // cross-stream hazards: outputs of one stream read or written by the other
    std::vector<const aoa_ct*> outs[2], ins[2];
    for (const Unit& u : units)
      for (int t = u.s; t < u.e; t++) {
        outs[u.stream].push_back(go[t]);
        ins[u.stream].push_back(ga[t]);
        ins[u.stream].push_back(gb[t]);
      }
    for (int x = 0; x < 2 && use_aux; x++)
      for (const aoa_ct* o : outs[x]) {
        for (const aoa_ct* i : ins[1 - x]) use_aux = use_aux && o != i;
        for (const aoa_ct* o2 : outs[1 - x]) use_aux = use_aux && o != o2;
        if (!use_aux) break;
      }
  }
  if (!use_aux) {
    for (const Unit& g : groups)
      group(C.stream, C.batch, C.batch_bytes, g.e - g.s, go.data() + g.s, ga.data() + g.s, gb.data() + g.s,
            lvl(idx[g.s]), idx.data() + g.s);
    return;
  }
  if (!C.aux) {
    AOA_CUDA(cudaStreamCreateWithFlags(&C.aux, cudaStreamNonBlocking));
    AOA_CUDA(cudaEventCreateWithFlags(&C.ev_fork, cudaEventDisableTiming));
    AOA_CUDA(cudaEventCreateWithFlags(&C.ev_join, cudaEventDisableTiming));
  }
  AOA_CUDA(cudaEventRecord(C.ev_fork, C.stream));
  AOA_CUDA(cudaStreamWaitEvent(C.aux, C.ev_fork, 0));
  for (const Unit& u : units) {
    const bool aux = u.stream == 1;
    group(aux ? C.aux : C.stream, aux ? C.batch2 : C.batch, aux ? C.batch2_bytes : C.batch_bytes, u.e - u.s,
          go.data() + u.s, ga.data() + u.s, gb.data() + u.s, lvl(idx[u.s]), idx.data() + u.s);
  }
  AOA_CUDA(cudaEventRecord(C.ev_join, C.aux));
  AOA_CUDA(cudaStreamWaitEvent(C.stream, C.ev_join, 0));
}

void hmult_batch(Ctx& C, int n, aoa_ct* const* out, aoa_ct* const* a, aoa_ct* const* b, const aoa_swk* evk,
                 bool do_rescale) {
  const Engine& E = *C.E;
  if (evk && evk->domain != C.transform)
    throw AoaError(AOA_ERR_BAD_PARAM, "the switching key is in another transform domain");
  if (n < 0) throw AoaError(AOA_ERR_BAD_PARAM, "negative batch size");
  if (n == 0) return;
  if (!out || !a || !b) throw AoaError(AOA_ERR_BAD_PARAM, "null batch arrays");
  if (!evk || !evk->d) throw AoaError(AOA_ERR_NO_KEY, "missing relinearisation key");
  if (E.kl == 0) throw AoaError(AOA_ERR_BAD_PARAM, "key switching needs special primes (kl > 0)");
  for (int z = 0; z < n; z++) {
    if (!out[z] || !a[z] || !b[z]) throw AoaError(AOA_ERR_BAD_PARAM, "null ciphertext in batch");
    if (a[z]->level == 0 || b[z]->level == 0)
      throw AoaError(AOA_ERR_LEVEL_EXHAUSTED, "The ciphertext level is 0. No more rescaling is possible.");
    if (a[z]->slots != b[z]->slots)
      throw AoaError(AOA_ERR_SLOT_MISMATCH, "Ciphertexts must have the same number of slots.");
  }
  for (int z = 0; z < n; z++) {                  // operands to the transform domain (poly_mul's rule)
    to_domain(C, a[z], C.transform, a[z]->level + 1);
    to_domain(C, b[z], C.transform, b[z]->level + 1);
  }
  // group by level (the operands' common limb count), chunks of kMaxBatch
  run_grouped(C, n, out, a, b, [&](int z) { return std::min(a[z]->level, b[z]->level); },
              [&](cudaStream_t st, void*& ws, size_t& wb, int g, aoa_ct* const* go, aoa_ct* const* ga,
                  aoa_ct* const* gb, int level, const int*) {
                hmult_batch_group(C, st, ws, wb, g, go, ga, gb, evk, do_rescale, level);
              });
}

// Batched Galois automorphism + key switch of n ciphertexts at one level with
// one key (apply_galois per op: ckks_rotate_left / ckks_conjugate,
// ckks.cpp:953-1040), every stage one launch over the batch.  Workspace
// (N-word limbs): R [2][n][k] (permuted c0 | permuted c1)  T [n][k]
// UB [n][kl]  KS [2][n][k+kl]  Y [2][n][k].
static size_t galois_words(const Engine& E, int n) {
  return (size_t)E.N * n * (3 * E.k + E.kl + 2 * (E.k + E.kl) + 2 * E.k);
}

static void galois_batch_group(Ctx& C, cudaStream_t st, void*& ws, size_t& ws_bytes, int n, aoa_ct* const* out,
                               aoa_ct* const* in, const long* galois, const aoa_swk* const* keys, int level) {
  const Engine& E = *C.E;
  const long N = E.N;
  const int m = level + 1, k = E.k, kl = E.kl;
  const long half = (long)k * N, ks = (long)(k + kl) * N;
  const size_t need = galois_words(E, n) * 8;
  if (ws_bytes < need) {
    if (ws) AOA_CUDA(cudaFreeAsync(ws, st));
    ws = nullptr;
    ws_bytes = 0;
    if (cudaMallocAsync(&ws, need, st) != cudaSuccess) {
      cudaGetLastError();
      throw AoaError(AOA_ERR_OOM, "batch workspace allocation failed");
    }
    ws_bytes = need;
  }
  uint64_t* p = (uint64_t*)ws;
  uint64_t* R = p;  p += 2L * n * half;
  uint64_t* T = p;  p += (long)n * half;
  uint64_t* UB = p; p += (long)n * kl * N;
  uint64_t* KS = p; p += 2L * n * ks;
  uint64_t* Y = p;
  uint64_t* X = R + (long)n * half;
  CtPtrs ptr;
  int slots[kMaxBatch];
  uint64_t scale[kMaxBatch];
  for (int z = 0; z < n; z++) {
    ptr.a[z] = in[z]->d;
    slots[z] = in[z]->slots;
    scale[z] = in[z]->scale;
  }
  GaloisList gl;
  bool one_key = true;
  for (int z = 0; z < n; z++) {
    gl.g[z] = galois[z];
    one_key = one_key && keys[z] == keys[0];
  }
  automorph_ntt_batch_op(E, ptr, half, R, n, gl, m, st);
  NttIo io;                                      // inverse of the permuted c1, out of place
  io.src = X;
  io.src_poly_stride = k;
  ntt_batch_io(E, T, n, 0, m, k, false, io, st);
  modup(E, T, half, UB, (long)kl * N, n, level, st);
  ntt_batch(E, UB, n, k, kl, kl, true, st);
  if (one_key) {                                 // each key word read once for the group
    keyswitch_mul_batch_op(E, X, half, UB, (long)kl * N, keys[0]->d, KS, ks, n, m, st);
  } else {
    KeyPtrs kp;
    for (int z = 0; z < n; z++) kp.k[z] = keys[z]->d;
    keyswitch_mul_keys_op(E, X, half, UB, (long)kl * N, kp, KS, ks, n, m, st);
  }
  ntt_batch(E, KS + (long)m * N, 2 * n, k, kl, k + kl, false, st);
  moddown_conv(E, KS + (long)m * N, ks, Y, half, 2 * n, m, st);
  ntt_batch(E, Y, 2 * n, 0, m, k, true, st);
  OutPtrs outp;
  for (int z = 0; z < n; z++) {
    outp.p[z] = out[z]->d;
    outp.p[n + z] = out[z]->d + half;
  }
  ks_combine_ptr(E, outp, R, half, KS, ks, Y, half, m, 2 * n, 0, st, n);   // c0 base for poly 0 only
  for (int z = 0; z < n; z++) {
    out[z]->level = level;
    out[z]->slots = slots[z];
    out[z]->scale = scale[z];
    out[z]->domain = AOA_NTT;
  }
}

// n automorphisms, op z by galois[z] with keys[z]: grouped by level only, so
// ops of different steps and keys share every launch of a group.
void galois_batch(Ctx& C, int n, aoa_ct* const* out, aoa_ct* const* in, const long* galois,
                  const aoa_swk* const* keys) {
  const Engine& E = *C.E;
  if (C.transform != AOA_NTT) throw AoaError(AOA_ERR_BAD_PARAM, "batched rotations run on the NTT transform only");
  if (n < 0) throw AoaError(AOA_ERR_BAD_PARAM, "negative batch size");
  if (n == 0) return;
  if (!out || !in || !galois || !keys) throw AoaError(AOA_ERR_BAD_PARAM, "null batch arrays");
  if (E.kl == 0) throw AoaError(AOA_ERR_BAD_PARAM, "key switching needs special primes (kl > 0)");
  for (int z = 0; z < n; z++) {
    if (!out[z] || !in[z]) throw AoaError(AOA_ERR_BAD_PARAM, "null ciphertext in batch");
    if (!keys[z] || !keys[z]->d) throw AoaError(AOA_ERR_NO_KEY, "missing switching key for this automorphism");
    if (keys[z]->domain != AOA_NTT)
      throw AoaError(AOA_ERR_BAD_PARAM, "the switching key is in another transform domain");
    if (!(galois[z] & 1)) throw AoaError(AOA_ERR_BAD_PARAM, "the Galois element must be odd");
  }
  for (int z = 0; z < n; z++) to_domain(C, in[z], AOA_NTT, in[z]->level + 1);
  run_grouped(C, n, out, in, nullptr, [&](int z) { return in[z]->level; },
              [&](cudaStream_t st, void*& ws, size_t& wb, int g, aoa_ct* const* go, aoa_ct* const* ga,
                  aoa_ct* const*, int level, const int* ids) {
                std::vector<long> gg(g);
                std::vector<const aoa_swk*> kk(g);
                for (int t = 0; t < g; t++) {
                  gg[t] = galois[ids[t]];
                  kk[t] = keys[ids[t]];
                }
                galois_batch_group(C, st, ws, wb, g, go, ga, gg.data(), kk.data(), level);
              });
}

static void galois_batch_uniform(Ctx& C, int n, aoa_ct* const* out, aoa_ct* const* in, long galois,
                                 const aoa_swk* key) {
  if (n < 0) throw AoaError(AOA_ERR_BAD_PARAM, "negative batch size");
  std::vector<long> g(n, galois);
  std::vector<const aoa_swk*> k(n, key);
  galois_batch(C, n, out, in, g.data(), k.data());
}

// The reference's per-call HMult + relinearise + rescale, step for step
// (ckks_mul, ckks.cpp:273-347 over poly_t.cpp's domain rules): every poly op
// covers the full base (k limbs, k + kl for the extended polys) whatever the
// level, operands are transformed on demand, d2 goes through a full QB inverse
// and forward transform, both key products through full QB inverse transforms,
// and d0 / d1 / d2 come back to coefficients before the additions.  Same
// residues as hmult(); kept as the plain per-call path the batched pipeline is
// compared against.
struct PlainWs {
  uint64_t *axbx1, *axbx2, *bxbx, *axax, *qb, *t0, *t1;
};

// the plain paths' workspace: four Q polys and three QB polys
static PlainWs plain_ws(Ctx& C) {
  const Engine& E = *C.E;
  const long half = (long)E.k * E.N, qb = (long)(E.k + E.kl) * E.N;
  if (!C.plain || C.plain_bytes < (size_t)(4 * half + 3 * qb) * 8) {
    if (C.plain) AOA_CUDA(cudaFreeAsync(C.plain, C.stream));
    C.plain = nullptr;
    if (cudaMallocAsync(&C.plain, (size_t)(4 * half + 3 * qb) * 8, C.stream) != cudaSuccess) {
      cudaGetLastError();
      throw AoaError(AOA_ERR_OOM, "plain-path workspace allocation failed");
    }
    C.plain_bytes = (size_t)(4 * half + 3 * qb) * 8;
  }
  uint64_t* p = (uint64_t*)C.plain;
  return PlainWs{p, p + half, p + 2 * half, p + 3 * half, p + 4 * half, p + 4 * half + qb, p + 4 * half + 2 * qb};
}

void hmult_plain(Ctx& C, aoa_ct* out, aoa_ct* a, aoa_ct* b, const aoa_swk* evk) {
  const Engine& E = *C.E;
  const long N = E.N;
  if (a->level == 0 || b->level == 0)
    throw AoaError(AOA_ERR_LEVEL_EXHAUSTED, "The ciphertext level is 0. No more rescaling is possible.");
  if (a->slots != b->slots) throw AoaError(AOA_ERR_SLOT_MISMATCH, "Ciphertexts must have the same number of slots.");
  if (!evk || !evk->d) throw AoaError(AOA_ERR_NO_KEY, "missing relinearisation key");
  if (C.transform != AOA_NTT || evk->domain != AOA_NTT)
    throw AoaError(AOA_ERR_BAD_PARAM, "the reference-structured path runs on the NTT transform only");
  if (a->domain == AOA_DGT) to_domain(C, a, AOA_COEF, a->level + 1);
  if (b->domain == AOA_DGT) to_domain(C, b, AOA_COEF, b->level + 1);
  const int k = E.k, nqb = E.k + E.kl;
  const int level = std::min(a->level, b->level);
  const long half = (long)k * N, qb = (long)nqb * N;
  const PlainWs s = plain_ws(C);
  cudaStream_t st = C.stream;
  int a_dom = a->domain, b_dom = b->domain;
  // poly_add_add(axbx1 = c1[1] + c1[0], axbx2 = c2[1] + c2[0]) in the operands' domain
  ew_binary_op(E, s.axbx1, 0, a->d + half, 0, a->d, 0, 0, 0, k, 1, st);
  ew_binary_op(E, s.axbx2, 0, b->d + half, 0, b->d, 0, 0, 0, k, 1, st);
  // poly_mul(axbx1, axbx1, axbx2): both to the transform domain, full base
  if (a_dom == AOA_COEF) ntt_batch(E, s.axbx1, 1, 0, k, k, true, st);
  if (b_dom == AOA_COEF) ntt_batch(E, s.axbx2, 1, 0, k, k, true, st);
  ew_binary_op(E, s.axbx1, 0, s.axbx1, 0, s.axbx2, 0, 2, 0, k, 1, st);
  // poly_mul(bxbx, c1[0], c2[0]) and poly_mul(axax, c1[1], c2[1]): operands transformed in place
  to_domain(C, a, AOA_NTT, k);
  if (b != a) to_domain(C, b, AOA_NTT, k);
  ew_binary_op(E, s.bxbx, 0, a->d, 0, b->d, 0, 2, 0, k, 1, st);
  ew_binary_op(E, s.axax, 0, a->d + half, 0, b->d + half, 0, 2, 0, k, 1, st);
  const uint64_t sa = a->scale, sb = b->scale;
  const int slots = a->slots;
  // poly_modup: copy the Q part into a QB poly, inverse transform over QB, convert
  copy_limbs(C, s.qb, s.axax, half);
  ntt_batch(E, s.qb, 1, 0, nqb, nqb, false, st);
  modup(E, s.qb, 0, s.qb + half, 0, 1, level, st);
  // poly_mul with evk.b / evk.a over QB (forward transform of the whole QB poly)
  ntt_batch(E, s.qb, 1, 0, nqb, nqb, true, st);
  ew_binary_op(E, s.t0, 0, s.qb, 0, evk->d, 0, 2, 0, nqb, 1, st);
  ew_binary_op(E, s.t1, 0, s.qb, 0, evk->d + qb, 0, 2, 0, nqb, 1, st);
  // poly_moddown x2: full QB inverse transforms, then B -> Q
  ntt_batch(E, s.t0, 2, 0, nqb, nqb, false, st);
  moddown(E, s.t0, s.t0 + half, 0, s.t0, 0, 1, level, st);
  moddown(E, s.t1, s.t1 + half, 0, s.t1, 0, 1, level, st);
  // poly_add_add(c0 = bxbx + ks0, c1 = axbx1 + ks1): mixed domains -> coefficients
  ntt_batch(E, s.bxbx, 1, 0, k, k, false, st);
  ntt_batch(E, s.axbx1, 1, 0, k, k, false, st);
  ew_binary_op(E, out->d, 0, s.bxbx, 0, s.t0, 0, 0, 0, k, 1, st);
  ew_binary_op(E, out->d + half, 0, s.axbx1, 0, s.t1, 0, 0, 0, k, 1, st);
  // poly_sub(c1 -= bxbx); poly_sub(c1 -= axax) with axax back to coefficients
  ew_binary_op(E, out->d + half, 0, out->d + half, 0, s.bxbx, 0, 1, 0, k, 1, st);
  ntt_batch(E, s.axax, 1, 0, k, k, false, st);
  ew_binary_op(E, out->d + half, 0, out->d + half, 0, s.axax, 0, 1, 0, k, 1, st);
  // ckks_rescale
  rescale(E, out->d, half, 2, level, st);
  out->level = level - 1;
  out->slots = slots;
  out->scale = scale_after_mult(E, sa, sb, level);
  out->domain = AOA_COEF;
}

// The reference's per-call rotation / conjugation sequence on this engine's
// kernels (ckks_rotate_left, ckks.cpp:982-1009, with rotate_slots_left,
// encoder.cu:325-350; ckks_conjugate, ckks.cpp:1011-1040): both input polys
// back to coefficients over the whole Q base, the coefficient permutation
// X -> X^g with its sign, ModUp of the permuted c1 into a QB poly, a forward
// transform of the whole QB poly, the two key products, inverse transforms
// of both whole QB products, two ModDowns, and c0' + ks0; the output is in
// coefficients.  The reference transforms its input in place; here the
// inverse reads the input out of place (the same work), so the input keeps
// its domain.  The plain per-call baseline of the uneven benchmark beside
// hmult_plain; apply_galois is the engine's own path.
void galois_plain(Ctx& C, aoa_ct* out, aoa_ct* in, long galois, const aoa_swk* key) {
  const Engine& E = *C.E;
  const long N = E.N;
  if (!key || !key->d) throw AoaError(AOA_ERR_NO_KEY, "missing switching key for this automorphism");
  if (E.kl == 0) throw AoaError(AOA_ERR_BAD_PARAM, "key switching needs special primes (kl > 0)");
  if (C.transform != AOA_NTT || key->domain != AOA_NTT)
    throw AoaError(AOA_ERR_BAD_PARAM, "the reference-structured path runs on the NTT transform only");
  const int k = E.k, nqb = E.k + E.kl;
  const int level = in->level, slots = in->slots;
  const uint64_t scale = in->scale;
  const long half = (long)k * N, qb = (long)nqb * N;
  const PlainWs s = plain_ws(C);
  cudaStream_t st = C.stream;
  // rotate_slots_left on c0 and c1: the input in coefficients (full base), then the map
  if (in->domain == AOA_DGT) throw AoaError(AOA_ERR_BAD_PARAM, "the reference-structured path runs on the NTT transform only");
  const uint64_t* coef = in->d;
  if (in->domain == AOA_NTT) {
    NttIo io;
    io.src = in->d;
    io.src_poly_stride = k;
    ntt_batch_io(E, s.t0, 2, 0, k, k, false, io, st);     // both polys into t0 / t0 + half
    coef = s.t0;
  }
  automorph_coef_op(E, s.bxbx, coef, 0, galois, k, 1, st);
  automorph_coef_op(E, s.axax, coef + half, 0, galois, k, 1, st);
  // poly_modup(d2axaxQB, axax, level)
  copy_limbs(C, s.qb, s.axax, half);
  modup(E, s.qb, 0, s.qb + half, 0, 1, level, st);
  // poly_mul with rtk.b / rtk.a over QB: the QB poly to the transform domain
  ntt_batch(E, s.qb, 1, 0, nqb, nqb, true, st);
  ew_binary_op(E, s.t0, 0, s.qb, 0, key->d, 0, 2, 0, nqb, 1, st);
  ew_binary_op(E, s.t1, 0, s.qb, 0, key->d + qb, 0, 2, 0, nqb, 1, st);
  // poly_moddown x2: full QB inverse transforms, then B -> Q
  ntt_batch(E, s.t0, 2, 0, nqb, nqb, false, st);
  moddown(E, s.t0, s.t0 + half, 0, s.t0, 0, 1, level, st);
  moddown(E, s.t1, s.t1 + half, 0, s.t1, 0, 1, level, st);
  // c2.c0 = rotated c0 + ks0; c2.c1 = ks1
  ew_binary_op(E, out->d, 0, s.bxbx, 0, s.t0, 0, 0, 0, k, 1, st);
  copy_limbs(C, out->d + half, s.t1, half);
  out->level = level;
  out->slots = slots;
  out->scale = scale;
  out->domain = AOA_COEF;
}

}  // namespace aoa

// ---------------------------------------------------------------------------
extern "C" {

int aoa_ct_create(aoa_ctx* c, aoa_ct** out) {
  if (!c || !out) return fail(AOA_ERR_BAD_PARAM, "null argument");
  return guarded([&] {
    const Engine& E = *c->c.E;
    aoa_ct* ct = new aoa_ct();
    cudaError_t e = cudaMallocAsync(&ct->d, (size_t)2 * E.k * E.N * 8, c->c.stream);
    if (e != cudaSuccess) {
      cudaGetLastError();
      delete ct;
      throw AoaError(AOA_ERR_OOM, "ciphertext allocation failed");
    }
    AOA_CUDA(cudaMemsetAsync(ct->d, 0, (size_t)2 * E.k * E.N * 8, c->c.stream));
    ct->level = E.k - 1;                                   // cipher_init (cipher_t.cpp:3-9)
    ct->scale = E.scale_bits > 0 && E.scale_bits < 64 ? (1ull << E.scale_bits) : 1;
    ct->slots = 0;
    ct->domain = AOA_COEF;
    *out = ct;
  });
}

int aoa_ct_destroy(aoa_ctx* c, aoa_ct* ct) {
  if (!ct) return AOA_OK;
  if (!c) return fail(AOA_ERR_BAD_PARAM, "null context");
  int st = guarded([&] { AOA_CUDA(cudaFreeAsync(ct->d, c->c.stream)); });
  delete ct;
  return st;
}

int aoa_ct_set(aoa_ct* ct, int level, int slots, uint64_t scale, int domain) {
  if (!ct || (domain != AOA_COEF && domain != AOA_NTT && domain != AOA_DGT)) return fail(AOA_ERR_BAD_PARAM, "bad argument");
  ct->level = level; ct->slots = slots; ct->scale = scale; ct->domain = domain;
  return AOA_OK;
}

int aoa_ct_get(const aoa_ct* ct, int* level, int* slots, uint64_t* scale, int* domain) {
  if (!ct) return fail(AOA_ERR_BAD_PARAM, "null ciphertext");
  if (level) *level = ct->level;
  if (slots) *slots = ct->slots;
  if (scale) *scale = ct->scale;
  if (domain) *domain = ct->domain;
  return AOA_OK;
}

int aoa_ct_data(aoa_ct* ct, uint64_t** d) {
  if (!ct || !d) return fail(AOA_ERR_BAD_PARAM, "null argument");
  *d = ct->d;
  return AOA_OK;
}

// host residues [2][nlimbs][N] (c0 then c1) in `domain`
int aoa_ct_upload(aoa_ctx* c, aoa_ct* ct, const uint64_t* host, int nlimbs, int domain) {
  if (!c || !ct || !host) return fail(AOA_ERR_BAD_PARAM, "null argument");
  return guarded([&] {
    const Engine& E = *c->c.E;
    if (nlimbs < 1 || nlimbs > E.k) throw AoaError(AOA_ERR_BAD_PARAM, "nlimbs out of range");
    if (domain != AOA_COEF && domain != AOA_NTT && domain != AOA_DGT) throw AoaError(AOA_ERR_BAD_PARAM, "bad domain");
    const size_t limb = (size_t)E.N * 8;
    for (int p = 0; p < 2; p++)
      AOA_CUDA(cudaMemcpyAsync(ct->d + (size_t)p * E.k * E.N, host + (size_t)p * nlimbs * E.N, nlimbs * limb,
                               cudaMemcpyHostToDevice, c->c.stream));
    ct->domain = domain;
    ct->level = nlimbs - 1;
  });
}

// download limbs 0..nlimbs-1 of both polys in `domain` (converts a copy)
static int download(aoa_ctx* c, const aoa_ct* ct, uint64_t* host, int nlimbs, int domain, bool wait);

int aoa_ct_download(aoa_ctx* c, const aoa_ct* ct, uint64_t* host, int nlimbs, int domain) {
  return download(c, ct, host, nlimbs, domain, true);
}

// the same, queued on the context's stream without waiting: `host` (pinned for
// an asynchronous copy) is valid after aoa_ctx_sync or a later synchronising call
int aoa_ct_download_async(aoa_ctx* c, const aoa_ct* ct, uint64_t* host, int nlimbs, int domain) {
  return download(c, ct, host, nlimbs, domain, false);
}

static int download(aoa_ctx* c, const aoa_ct* ct, uint64_t* host, int nlimbs, int domain, bool wait) {
  if (!c || !ct || !host) return fail(AOA_ERR_BAD_PARAM, "null argument");
  return guarded([&] {
    Ctx& C = c->c;
    const Engine& E = *C.E;
    if (nlimbs < 1 || nlimbs > E.k) throw AoaError(AOA_ERR_BAD_PARAM, "nlimbs out of range");
    if (domain != AOA_COEF && domain != AOA_NTT && domain != AOA_DGT) throw AoaError(AOA_ERR_BAD_PARAM, "bad domain");
    const size_t limb = (size_t)E.N * 8;
    const uint64_t* src = ct->d;
    uint64_t* tmp = nullptr;
    if (domain != ct->domain) {
      if (C.conv_bytes < 2 * E.k * limb) {
        if (C.conv) AOA_CUDA(cudaFreeAsync(C.conv, C.stream));
        C.conv = nullptr;
        AOA_CUDA(cudaMallocAsync(&C.conv, 2 * E.k * limb, C.stream));
        C.conv_bytes = 2 * E.k * limb;
      }
      tmp = (uint64_t*)C.conv;
      AOA_CUDA(cudaMemcpy2DAsync(tmp, E.k * limb, ct->d, E.k * limb, nlimbs * limb, 2, cudaMemcpyDeviceToDevice,
                                 C.stream));
      if (ct->domain != AOA_COEF) xform(E, ct->domain, tmp, 2, 0, nlimbs, E.k, false, C.stream);
      if (domain != AOA_COEF) xform(E, domain, tmp, 2, 0, nlimbs, E.k, true, C.stream);
      src = tmp;
    }
    for (int p = 0; p < 2; p++)
      AOA_CUDA(cudaMemcpyAsync(host + (size_t)p * nlimbs * E.N, src + (size_t)p * E.k * E.N, nlimbs * limb,
                               cudaMemcpyDeviceToHost, C.stream));
    if (wait) AOA_CUDA(cudaStreamSynchronize(C.stream));
  });
}

// Switching key from host residues b, a ([k+kl][N] each) in `domain`.
int aoa_swk_create(aoa_ctx* c, const uint64_t* host_b, const uint64_t* host_a, int domain, aoa_swk** out) {
  if (!c || !host_b || !host_a || !out) return fail(AOA_ERR_BAD_PARAM, "null argument");
  if (domain != AOA_COEF && domain != AOA_NTT && domain != AOA_DGT) return fail(AOA_ERR_BAD_PARAM, "bad domain");
  return guarded([&] {
    Ctx& C = c->c;
    const Engine& E = *C.E;
    const size_t half = (size_t)E.nprimes * E.N;
    aoa_swk* k = new aoa_swk();
    if (cudaMallocAsync(&k->d, 2 * half * 8, C.stream) != cudaSuccess) {
      cudaGetLastError();
      delete k;
      throw AoaError(AOA_ERR_OOM, "key allocation failed");
    }
    AOA_CUDA(cudaMemcpyAsync(k->d, host_b, half * 8, cudaMemcpyHostToDevice, C.stream));
    AOA_CUDA(cudaMemcpyAsync(k->d + half, host_a, half * 8, cudaMemcpyHostToDevice, C.stream));
    // a coefficient-domain key goes to the context's transform domain
    k->domain = domain == AOA_COEF ? C.transform : domain;
    if (domain == AOA_COEF) xform(E, k->domain, k->d, 2, 0, E.nprimes, E.nprimes, true, C.stream);
    AOA_CUDA(cudaStreamSynchronize(C.stream));
    *out = k;
  });
}

int aoa_swk_data(aoa_swk* k, uint64_t** device_ptr, int* domain) {
  if (!k || !device_ptr) return fail(AOA_ERR_BAD_PARAM, "null argument");
  *device_ptr = k->d;
  if (domain) *domain = k->domain;
  return AOA_OK;
}

int aoa_swk_destroy(aoa_ctx* c, aoa_swk* k) {
  if (!k) return AOA_OK;
  if (!c) return fail(AOA_ERR_BAD_PARAM, "null context");
  int st = guarded([&] { AOA_CUDA(cudaFreeAsync(k->d, c->c.stream)); });
  delete k;
  return st;
}

int aoa_hmult(aoa_ctx* c, aoa_ct* out, aoa_ct* a, aoa_ct* b, const aoa_swk* evk) {
  if (!c || !out || !a || !b) return fail(AOA_ERR_BAD_PARAM, "null argument");
  return guarded([&] { hmult(c->c, out, a, b, evk, false); });
}

int aoa_hmult_relin_rescale(aoa_ctx* c, aoa_ct* out, aoa_ct* a, aoa_ct* b, const aoa_swk* evk) {
  if (!c || !out || !a || !b) return fail(AOA_ERR_BAD_PARAM, "null argument");
  return guarded([&] { hmult(c->c, out, a, b, evk, true); });
}

int aoa_hmult_batch(aoa_ctx* c, int n, aoa_ct* const* out, aoa_ct* const* a, aoa_ct* const* b,
                    const aoa_swk* evk, int rescale) {
  if (!c) return fail(AOA_ERR_BAD_PARAM, "null context");
  return guarded([&] { hmult_batch(c->c, n, out, a, b, evk, rescale != 0); });
}

int aoa_hmult_plain(aoa_ctx* c, aoa_ct* out, aoa_ct* a, aoa_ct* b, const aoa_swk* evk) {
  if (!c || !out || !a || !b) return fail(AOA_ERR_BAD_PARAM, "null argument");
  return guarded([&] { hmult_plain(c->c, out, a, b, evk); });
}

int aoa_rescale(aoa_ctx* c, aoa_ct* ct) {
  if (!c || !ct) return fail(AOA_ERR_BAD_PARAM, "null argument");
  return guarded([&] {
    if (ct->level == 0)
      throw AoaError(AOA_ERR_LEVEL_EXHAUSTED, "The ciphertext level is 0. No more rescaling is possible.");
    to_domain(c->c, ct, AOA_COEF, ct->level + 1);
    rescale(*c->c.E, ct->d, (long)c->c.E->k * c->c.E->N, 2, ct->level, c->c.stream);
    ct->level--;
  });
}

// ckks_add / ckks_sub (ckks.cpp:240-271): level = min, scale and slots of a.
static int add_sub(aoa_ctx* c, aoa_ct* out, aoa_ct* a, aoa_ct* b, int op) {
  if (!c || !out || !a || !b) return fail(AOA_ERR_BAD_PARAM, "null argument");
  return guarded([&] {
    Ctx& C = c->c;
    const Engine& E = *C.E;
    if (a->slots != b->slots) throw AoaError(AOA_ERR_SLOT_MISMATCH, "Ciphertexts must have the same number of slots.");
    const int level = std::min(a->level, b->level);
    if (a->domain != b->domain) {       // mixed states: both to coefficients (poly_t.cpp:143-146)
      to_domain(C, a, AOA_COEF, a->level + 1);
      to_domain(C, b, AOA_COEF, b->level + 1);
    }
    const long half = (long)E.k * E.N;
    ew_binary_op(E, out->d, half, a->d, half, b->d, half, op, 0, level + 1, 2, C.stream);
    out->level = level;
    out->slots = a->slots;
    out->scale = a->scale;
    out->domain = a->domain;
  });
}

int aoa_add(aoa_ctx* c, aoa_ct* out, aoa_ct* a, aoa_ct* b) { return add_sub(c, out, a, b, 0); }
int aoa_sub(aoa_ctx* c, aoa_ct* out, aoa_ct* a, aoa_ct* b) { return add_sub(c, out, a, b, 1); }

// rotation by `steps` slots to the left with key rtk (ckks_rotate_left);
// negative steps rotate right (rotate_slots_right = left by N/2 - r).
int aoa_rotate(aoa_ctx* c, aoa_ct* out, aoa_ct* in, int steps, const aoa_swk* rtk) {
  if (!c || !out || !in) return fail(AOA_ERR_BAD_PARAM, "null argument");
  return guarded([&] {
    const Engine& E = *c->c.E;
    const long M = 2 * E.N;
    long r = steps % (E.N / 2);
    if (r < 0) r += E.N / 2;
    const long g = (long)h_powmod(5, (uint64_t)r, (uint64_t)M);
    apply_galois(c->c, out, in, g, rtk);
  });
}

// batched forms: every op of the batch rotates by the same step with the same key
int aoa_rotate_batch(aoa_ctx* c, int n, aoa_ct* const* out, aoa_ct* const* in, int steps, const aoa_swk* rtk) {
  if (!c) return fail(AOA_ERR_BAD_PARAM, "null argument");
  return guarded([&] {
    const Engine& E = *c->c.E;
    long r = steps % (E.N / 2);
    if (r < 0) r += E.N / 2;
    galois_batch_uniform(c->c, n, out, in, (long)h_powmod(5, (uint64_t)r, (uint64_t)(2 * E.N)), rtk);
  });
}

int aoa_rotate_batch_steps(aoa_ctx* c, int n, aoa_ct* const* out, aoa_ct* const* in, const int* steps,
                           const aoa_swk* const* rtks) {
  if (!c) return fail(AOA_ERR_BAD_PARAM, "null argument");
  return guarded([&] {
    const Engine& E = *c->c.E;
    if (n < 0) throw AoaError(AOA_ERR_BAD_PARAM, "negative batch size");
    if (n > 0 && !steps) throw AoaError(AOA_ERR_BAD_PARAM, "null batch arrays");
    std::vector<long> g(n);
    for (int z = 0; z < n; z++) {
      long r = steps[z] % (E.N / 2);
      if (r < 0) r += E.N / 2;
      g[z] = (long)h_powmod(5, (uint64_t)r, (uint64_t)(2 * E.N));
    }
    galois_batch(c->c, n, out, in, g.data(), rtks);
  });
}

int aoa_conjugate_batch(aoa_ctx* c, int n, aoa_ct* const* out, aoa_ct* const* in, const aoa_swk* cjk) {
  if (!c) return fail(AOA_ERR_BAD_PARAM, "null argument");
  return guarded([&] { galois_batch_uniform(c->c, n, out, in, 2 * c->c.E->N - 1, cjk); });
}

int aoa_conjugate(aoa_ctx* c, aoa_ct* out, aoa_ct* in, const aoa_swk* cjk) {
  if (!c || !out || !in) return fail(AOA_ERR_BAD_PARAM, "null argument");
  return guarded([&] { apply_galois(c->c, out, in, 2 * c->c.E->N - 1, cjk); });
}

int aoa_rotate_plain(aoa_ctx* c, aoa_ct* out, aoa_ct* in, int steps, const aoa_swk* rtk) {
  if (!c || !out || !in) return fail(AOA_ERR_BAD_PARAM, "null argument");
  return guarded([&] {
    const Engine& E = *c->c.E;
    long r = steps % (E.N / 2);
    if (r < 0) r += E.N / 2;
    galois_plain(c->c, out, in, (long)h_powmod(5, (uint64_t)r, (uint64_t)(2 * E.N)), rtk);
  });
}

int aoa_conjugate_plain(aoa_ctx* c, aoa_ct* out, aoa_ct* in, const aoa_swk* cjk) {
  if (!c || !out || !in) return fail(AOA_ERR_BAD_PARAM, "null argument");
  return guarded([&] { galois_plain(c->c, out, in, 2 * c->c.E->N - 1, cjk); });
}

// Standalone basis conversions on device buffers (coefficient domain):
// ModUp reads Q limbs 0..level of `in_q` ([k][N]) and writes kl limbs to `out_b`;
// ModDown reads a QB poly ([k + kl][N], B limbs at offset k) and writes limbs
// 0..level of `out_q`.
int aoa_modup(aoa_ctx* c, const uint64_t* in_q, uint64_t* out_b, int level) {
  if (!c || !in_q || !out_b) return fail(AOA_ERR_BAD_PARAM, "null argument");
  return guarded([&] { modup(*c->c.E, in_q, 0, out_b, 0, 1, level, c->c.stream); });
}

int aoa_moddown(aoa_ctx* c, const uint64_t* in_qb, uint64_t* out_q, int level) {
  if (!c || !in_qb || !out_q) return fail(AOA_ERR_BAD_PARAM, "null argument");
  return guarded([&] {
    const Engine& E = *c->c.E;
    moddown(E, in_qb, in_qb + (long)E.k * E.N, 0, out_q, 0, 1, level, c->c.stream);
  });
}

int aoa_rescale_polys(aoa_ctx* c, uint64_t* d, int npolys, int poly_stride, int level) {
  if (!c || !d) return fail(AOA_ERR_BAD_PARAM, "null argument");
  return guarded([&] { rescale(*c->c.E, d, (long)poly_stride * c->c.E->N, npolys, level, c->c.stream); });
}

}  // extern "C"
