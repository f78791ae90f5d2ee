// Plaintext and constant operations of the evaluator (aoa-ntt
// src/ckks/ckks.cpp:502-690, aoa-dgt src/ckks.cpp): multiply by an encoded
// plaintext, multiply / add a real constant, and rotate-and-sum over the
// slots (ckks_sumslots, ckks.cpp:484-500), the building blocks of the
// reference's inner products and of the logistic-regression steps its
// downstream user runs.  Scale bookkeeping follows the reference exactly.
#include "aoa_internal.h"

using namespace aoa;

namespace aoa {
void ct_to_domain(Ctx& C, aoa_ct* ct, int domain, int nlimbs);
void apply_galois(Ctx& C, aoa_ct* out, aoa_ct* in, long galois, const aoa_swk* key);
}  // namespace aoa

namespace {

constexpr int kMaxScalarLimbs = 256;
struct LimbScalars {
  uint64_t v[kMaxScalarLimbs];
};

// out = in (op) s[limb] on npolys polys; op 0: add to every word, 1: multiply,
// 2: add to word 0 of each limb only, 3: add to the first half of each limb
// (the real plane of a DGT limb).
__global__ void scalar_limb_op(uint64_t* out, const uint64_t* in, long poly_stride, LimbScalars s, int op,
                               const PrimeConst* __restrict__ pc, int log_n) {
  const long N = 1L << log_n;
  const long c = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= N) return;
  const int l = blockIdx.y;
  const long off = blockIdx.z * poly_stride + (long)l * N + c;
  const PrimeConst& P = pc[l];
  const uint64_t x = in[off], y = s.v[l];
  uint64_t r = x;
  if (op == 1) r = mul_mod(x, y, P);
  else if (op == 0 || (op == 2 && c == 0) || (op == 3 && c < N / 2)) r = add_mod(x, y, P.q);
  out[off] = r;
}

void scalar_op(Ctx& C, uint64_t* out, const uint64_t* in, long poly_stride, int npolys, int nlimbs,
               const LimbScalars& s, int op) {
  const Engine& E = *C.E;
  dim3 grid((unsigned)((E.N + 255) / 256), (unsigned)nlimbs, (unsigned)npolys);
  scalar_limb_op<<<grid, 256, 0, C.stream>>>(out, in, poly_stride, s, op, E.d_pc, E.log_n);
  note_launch();
  AOA_CHECK_LAUNCH();
}

uint64_t product_scale(const Engine& E, uint64_t sa, uint64_t sb, int level) {
  return (uint64_t)(((unsigned __int128)sa * sb) / E.primes[level]);
}

void do_rescale(Ctx& C, aoa_ct* ct) {
  if (ct->level == 0)
    throw AoaError(AOA_ERR_LEVEL_EXHAUSTED, "The ciphertext level is 0. No more rescaling is possible.");
  ct_to_domain(C, ct, AOA_COEF, ct->level + 1);
  rescale(*C.E, ct->d, (long)C.E->k * C.E->N, 2, ct->level, C.stream);
  ct->level--;
}

void copy_meta(aoa_ct* out, const aoa_ct* in) {
  out->level = in->level;
  out->slots = in->slots;
  out->scale = in->scale;
  out->domain = in->domain;
}

}  // namespace

extern "C" {

// ckks_mul(ctx, c2, c1, poly_t*) / ckks_mul_without_rescale (ckks.cpp:646-676)
// and, with the plaintext encoded at the ciphertext's scale, ckks_mul(ctx, c2,
// c1, complex*) (ckks.cpp:610-632): out = in * pt in the context's transform
// domain; scale = floor(in.scale * pt_scale / q_level); then rescaled when
// `rescale` is set.  d_pt: [k][N] plaintext (limbs 0..level used) in pt_domain.
int aoa_mul_plaintext(aoa_ctx* c, aoa_ct* out, aoa_ct* in, const uint64_t* d_pt, int pt_domain, uint64_t pt_scale,
                      int rescale) {
  if (!c || !out || !in || !d_pt) return fail(AOA_ERR_BAD_PARAM, "null argument");
  return guarded([&] {
    Ctx& C = c->c;
    const Engine& E = *C.E;
    if (pt_domain != AOA_COEF && pt_domain != AOA_NTT && pt_domain != AOA_DGT)
      throw AoaError(AOA_ERR_BAD_PARAM, "bad domain");
    if (rescale && in->level == 0)
      throw AoaError(AOA_ERR_LEVEL_EXHAUSTED, "The ciphertext level is 0. No more rescaling is possible.");
    const int tk = C.transform, m = in->level + 1;
    const long half = (long)E.k * E.N;
    ct_to_domain(C, in, tk, m);
    const uint64_t* pt = d_pt;
    if (pt_domain != tk) {
      if (C.enc_bytes < (size_t)m * E.N * 8) {
        if (C.enc) AOA_CUDA(cudaFreeAsync(C.enc, C.stream));
        C.enc = nullptr;
        C.enc_bytes = 0;
        if (cudaMallocAsync(&C.enc, (size_t)E.k * E.N * 8, C.stream) != cudaSuccess) {
          cudaGetLastError();
          throw AoaError(AOA_ERR_OOM, "plaintext buffer allocation failed");
        }
        C.enc_bytes = (size_t)E.k * E.N * 8;
      }
      uint64_t* t = (uint64_t*)C.enc;
      AOA_CUDA(cudaMemcpyAsync(t, d_pt, (size_t)m * E.N * 8, cudaMemcpyDeviceToDevice, C.stream));
      if (pt_domain != AOA_COEF) xform(E, pt_domain, t, 1, 0, m, m, false, C.stream);
      xform(E, tk, t, 1, 0, m, m, true, C.stream);
      pt = t;
    }
    if (tk == AOA_DGT) gi_mul_op(E, out->d, half, in->d, half, pt, 0, 0, m, 2, C.stream);
    else ew_binary_op(E, out->d, half, in->d, half, pt, 0, 2, 0, m, 2, C.stream);
    const uint64_t scale = product_scale(E, in->scale, pt_scale, in->level);
    copy_meta(out, in);
    out->domain = tk;
    out->scale = scale;
    if (rescale) do_rescale(C, out);
  });
}

// ckks_mul_without_rescale(ctx, c2, c1, double) (ckks.cpp:570-592) and
// ckks_mul(ctx, c2, c1, double) (ckks.cpp:540-546): out = in * x with
// x = lrint(|val| * scale), negated for val < 0; scale = floor(scale^2 / q_level).
int aoa_mul_const(aoa_ctx* c, aoa_ct* out, aoa_ct* in, double val, int rescale) {
  if (!c || !out || !in) return fail(AOA_ERR_BAD_PARAM, "null argument");
  return guarded([&] {
    Ctx& C = c->c;
    const Engine& E = *C.E;
    const int m = in->level + 1;
    if (m > kMaxScalarLimbs) throw AoaError(AOA_ERR_BAD_PARAM, "too many limbs for a constant operation");
    if (rescale && in->level == 0)
      throw AoaError(AOA_ERR_LEVEL_EXHAUSTED, "The ciphertext level is 0. No more rescaling is possible.");
    const uint64_t x = (uint64_t)llrint(fabs(val) * (double)in->scale);
    LimbScalars s;
    for (int l = 0; l < m; l++) {
      const uint64_t q = E.primes[l], r = x % q;
      s.v[l] = val < 0 ? (r ? q - r : 0) : r;
    }
    scalar_op(C, out->d, in->d, (long)E.k * E.N, 2, m, s, 1);
    const uint64_t scale = product_scale(E, in->scale, in->scale, in->level);
    copy_meta(out, in);
    out->scale = scale;
    if (rescale) do_rescale(C, out);
  });
}

// ckks_add(ctx, c2, c1, double) (ckks.cpp:512-530): c0 + cnst (c0 - cnst for
// val < 0) with cnst = (uint64) (|val| * scale), c1 copied.  Adding the
// constant polynomial adds cnst to every NTT value, to coefficient 0, or to
// the real plane of every DGT value.
int aoa_add_const(aoa_ctx* c, aoa_ct* out, aoa_ct* in, double val) {
  if (!c || !out || !in) return fail(AOA_ERR_BAD_PARAM, "null argument");
  return guarded([&] {
    Ctx& C = c->c;
    const Engine& E = *C.E;
    const int m = in->level + 1;
    if (m > kMaxScalarLimbs) throw AoaError(AOA_ERR_BAD_PARAM, "too many limbs for a constant operation");
    const uint64_t cnst = (uint64_t)(fabs(val) * (double)in->scale);
    LimbScalars s;
    for (int l = 0; l < m; l++) {
      const uint64_t q = E.primes[l], r = cnst % q;
      s.v[l] = val < 0 ? (r ? q - r : 0) : r;
    }
    const int op = in->domain == AOA_NTT ? 0 : in->domain == AOA_DGT ? 3 : 2;
    scalar_op(C, out->d, in->d, 0, 1, m, s, op);
    if (out != in)
      AOA_CUDA(cudaMemcpyAsync(out->d + (long)E.k * E.N, in->d + (long)E.k * E.N, (size_t)m * E.N * 8,
                               cudaMemcpyDeviceToDevice, C.stream));
    copy_meta(out, in);
  });
}

// ckks_sumslots (ckks.cpp:484-500): for i = slots/2, slots/4, ..., 1:
// out = out + rotate_left(out, i).  rtks[j] is the left-rotation key for 2^j
// (j = 0 .. nkeys-1).
int aoa_sumslots(aoa_ctx* c, aoa_ct* out, aoa_ct* in, const aoa_swk* const* rtks, int nkeys) {
  if (!c || !out || !in || (nkeys > 0 && !rtks)) return fail(AOA_ERR_BAD_PARAM, "null argument");
  return guarded([&] {
    Ctx& C = c->c;
    const Engine& E = *C.E;
    const size_t bytes = (size_t)2 * E.k * E.N * 8;
    if (out != in) {
      AOA_CUDA(cudaMemcpyAsync(out->d, in->d, bytes, cudaMemcpyDeviceToDevice, C.stream));
      copy_meta(out, in);
    }
    aoa_ct tmp;
    if (cudaMallocAsync(&tmp.d, bytes, C.stream) != cudaSuccess) {
      cudaGetLastError();
      throw AoaError(AOA_ERR_OOM, "sumslots buffer allocation failed");
    }
    try {
      for (int i = out->slots >> 1; i >= 1; i >>= 1) {
        int j = 0;
        while ((1 << j) < i) j++;
        if (j >= nkeys || !rtks[j]) throw AoaError(AOA_ERR_NO_KEY, "missing rotation key for step " + std::to_string(i));
        const long g = (long)[&] {                      // 5^i mod 2N
          uint64_t r = 1, b = 5, e = (uint64_t)i, M = 2 * (uint64_t)E.N;
          while (e) { if (e & 1) r = r * b % M; b = b * b % M; e >>= 1; }
          return r;
        }();
        apply_galois(C, &tmp, out, g, rtks[j]);
        ct_to_domain(C, out, tmp.domain, out->level + 1);
        ew_binary_op(E, out->d, (long)E.k * E.N, out->d, (long)E.k * E.N, tmp.d, (long)E.k * E.N, 0, 0,
                     out->level + 1, 2, C.stream);
      }
    } catch (...) {
      cudaFreeAsync(tmp.d, C.stream);
      throw;
    }
    AOA_CUDA(cudaFreeAsync(tmp.d, C.stream));
  });
}

}  // extern "C"
