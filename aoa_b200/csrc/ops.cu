// Elementwise residue kernels (ntt_vector_op / _int / dualop / seqop,
// aoa-ntt src/cuda/htrans/ntt.cu:479-667), the HMult tensor product, the
// key-switch products and the Galois automorphisms (aoa-ntt
// src/ckks/encoder.cu:300-427).
//
// Launch shape: grid (N / 256, limbs, polys), one thread per coefficient;
// the prime of limb l is prime0 + l.  Every limb is N contiguous words, so each
// warp reads and writes 256 contiguous bytes per operand.
#include "aoa_internal.h"

namespace aoa {

struct Limbs {            // npolys x nlimbs limbs of N words
  uint64_t* p;
  long poly_stride;       // words between polys
};
struct CLimbs {
  const uint64_t* p;
  long poly_stride;
};

__device__ __forceinline__ long coef_index() { return (long)blockIdx.x * blockDim.x + threadIdx.x; }

// The HMult element-wise kernels take kEwPer coefficients per thread (u-th at
// coef_u(u), each access still coalesced across the block), so a thread's
// per-limb constants and addresses serve several coefficients (N >= 1024).
constexpr int kEwPer = 4;
__device__ __forceinline__ long coef_u(int u) { return ((long)blockIdx.x * kEwPer + u) * blockDim.x + threadIdx.x; }

// c = a (op) b over limbs; op: 0 add, 1 sub, 2 mul (Montgomery pair), 3 neg(a)
__global__ void ew_binary(Limbs c, CLimbs a, CLimbs b, int op, int prime0, const PrimeConst* pc, int log_n) {
  const long N = 1L << log_n;
  const long off = (long)blockIdx.y * N + coef_index();
  const PrimeConst& P = pc[prime0 + blockIdx.y];
  const uint64_t x = a.p[blockIdx.z * a.poly_stride + off];
  uint64_t r;
  if (op == 3) {
    r = neg_mod(x, P.q);
  } else {
    const uint64_t y = b.p[blockIdx.z * b.poly_stride + off];
    r = op == 0 ? add_mod(x, y, P.q) : op == 1 ? sub_mod(x, y, P.q) : mul_mod(x, y, P);
  }
  c.p[blockIdx.z * c.poly_stride + off] = r;
}

// c = a (op) s with a per-limb scalar s[l] (already reduced mod its prime);
// op: 0 add, 1 sub, 2 mul
__global__ void ew_scalar(Limbs c, CLimbs a, const uint64_t* s, int op, int prime0, const PrimeConst* pc,
                          int log_n) {
  const long N = 1L << log_n;
  const long off = (long)blockIdx.y * N + coef_index();
  const PrimeConst& P = pc[prime0 + blockIdx.y];
  const uint64_t x = a.p[blockIdx.z * a.poly_stride + off], y = s[blockIdx.y];
  c.p[blockIdx.z * c.poly_stride + off] =
      op == 0 ? add_mod(x, y, P.q) : op == 1 ? sub_mod(x, y, P.q) : mul_mod(x, y, P);
}

// d = a * b + c  (ntt_vector_seqop)
__global__ void ew_muladd(Limbs d, CLimbs a, CLimbs b, CLimbs c, int prime0, const PrimeConst* pc, int log_n) {
  const long N = 1L << log_n;
  const long off = (long)blockIdx.y * N + coef_index();
  const PrimeConst& P = pc[prime0 + blockIdx.y];
  const uint64_t x = a.p[blockIdx.z * a.poly_stride + off];
  const uint64_t y = b.p[blockIdx.z * b.poly_stride + off];
  const uint64_t z = c.p[blockIdx.z * c.poly_stride + off];
  d.p[blockIdx.z * d.poly_stride + off] = add_mod(mul_mod(x, y, P), z, P.q);
}

// HMult tensor (ckks_mul_without_rescale, ckks.cpp:300-307), transform domain:
//   d0 = a0 b0,  d1 = a0 b1 + a1 b0,  d2 = a1 b1
// (the reference forms d1 as (a0+a1)(b0+b1) - d0 - d2: the same residues).
__device__ __forceinline__ void tensor3(uint64_t x0, uint64_t x1, uint64_t y0, uint64_t y1, const PrimeConst& P,
                                        uint64_t& d0, uint64_t& d1, uint64_t& d2) {
  const uint64_t q = P.q;
  if (P.bar_sh) {
    const uint64_t mu = P.bar_mu;
    const uint32_t s = (uint32_t)P.bar_sh;
    d0 = barrett_mul(x0, y0, q, mu, s);
    d1 = s <= 59 ? barrett_mul_add2(x0, y1, x1, y0, q, mu, s)        // q < 2^61: one reduction
                 : add_mod(barrett_mul(x0, y1, q, mu, s), barrett_mul(x1, y0, q, mu, s), q);
    d2 = barrett_mul(x1, y1, q, mu, s);
    return;
  }
  // Montgomery products carry a 2^-64 factor; one more REDC by R^2 clears it.
  const uint64_t qi = P.qinv_neg;
  const uint64_t m0 = mont_mul(x0, y0, q, qi);
  const uint64_t m1 = add_mod(mont_mul(x0, y1, q, qi), mont_mul(x1, y0, q, qi), q);
  const uint64_t m2 = mont_mul(x1, y1, q, qi);
  d0 = mont_mul(m0, P.r2, q, qi);
  d1 = mont_mul(m1, P.r2, q, qi);
  d2 = mont_mul(m2, P.r2, q, qi);
}

// operands of kEwPer coefficients, loaded before any store
__device__ __forceinline__ void tensor_ew(const uint64_t* a, long a_half, const uint64_t* b, long b_half,
                                          uint64_t* d0, uint64_t* d1, uint64_t* d2, const PrimeConst& P) {
  uint64_t x0[kEwPer], x1[kEwPer], y0[kEwPer], y1[kEwPer];
#pragma unroll
  for (int u = 0; u < kEwPer; u++) {
    const long c = coef_u(u);
    x0[u] = a[c];
    x1[u] = a[a_half + c];
    y0[u] = b[c];
    y1[u] = b[b_half + c];
  }
#pragma unroll
  for (int u = 0; u < kEwPer; u++) {
    const long c = coef_u(u);
    uint64_t r0, r1, r2;
    tensor3(x0[u], x1[u], y0[u], y1[u], P, r0, r1, r2);
    d0[c] = r0;
    d1[c] = r1;
    d2[c] = r2;
  }
}

__global__ void hmult_tensor(const uint64_t* a, const uint64_t* b, long a_half, long b_half, uint64_t* d0,
                             uint64_t* d1, uint64_t* d2, const PrimeConst* pc, int log_n) {
  const long limb = (long)blockIdx.y << log_n;
  const PrimeConst P = pc[blockIdx.y];
  tensor_ew(a + limb, a_half, b + limb, b_half, d0 + limb, d1 + limb, d2 + limb, P);
}

// Key-switch products over the QB limbs of the extended d2 (transform domain):
//   k0 = x * key_b,  k1 = x * key_a
// x limb l < nq lives at xq + l*N (prime l), limb nq + j at xb + j*N (prime K + j);
// the key is [b | a], each (k + kl) limbs in the reference's QB layout.
__global__ void keyswitch_mul(const uint64_t* xq, const uint64_t* xb, const uint64_t* key, long key_half,
                              uint64_t* k0, uint64_t* k1, int nq, int K, const PrimeConst* pc, int log_n) {
  const long N = 1L << log_n;
  const int l = blockIdx.y;
  const int prime = l < nq ? l : K + (l - nq);
  const uint64_t* x = l < nq ? xq + (long)l * N : xb + (long)(l - nq) * N;
  const uint64_t* kbp = key + (long)prime * N;
  const PrimeConst P = pc[prime];
  uint64_t xv[kEwPer], kb[kEwPer], ka[kEwPer];
#pragma unroll
  for (int u = 0; u < kEwPer; u++) {
    const long c = coef_u(u);
    xv[u] = x[c];
    kb[u] = kbp[c];
    ka[u] = kbp[key_half + c];
  }
#pragma unroll
  for (int u = 0; u < kEwPer; u++) {
    const long c = coef_u(u);
    k0[(long)l * N + c] = mul_mod(xv[u], kb[u], P);
    k1[(long)l * N + c] = mul_mod(xv[u], ka[u], P);
  }
}

// Coefficient-domain automorphism X -> X^g (g odd, mod 2N) with the
// negacyclic sign (execute_rotation, encoder.cu:300-322).
__global__ void automorph_coef(uint64_t* out, const uint64_t* in, long poly_stride, long galois,
                               const PrimeConst* pc, int log_n) {
  const long N = 1L << log_n;
  const long c = coef_index();
  const long off = blockIdx.z * poly_stride + (long)blockIdx.y * N;
  long t = (c * galois) & (2 * N - 1);
  uint64_t v = in[off + c];
  if (t >= N) { t -= N; v = neg_mod(v, pc[blockIdx.y].q); }
  out[off + t] = v;
}

// Transform-domain automorphism: a permutation of the evaluation points
// psi^(2 br(p) + 1) -> psi^((2 br(p) + 1) g).  Output position p reads the
// input position holding the evaluation at psi^((2 br(p)+1) g).
__global__ void automorph_ntt(uint64_t* out, const uint64_t* in, long poly_stride, long galois, int log_n) {
  const long N = 1L << log_n;
  const long p = coef_index();
  const long off = blockIdx.z * poly_stride + (long)blockIdx.y * N;
  const uint32_t br = __brev((uint32_t)p) >> (32 - log_n);
  const long e = ((2L * br + 1) * galois) & (2 * N - 1);   // odd exponent mod 2N
  const long src_br = (e - 1) >> 1;
  const long src = __brev((uint32_t)src_br) >> (32 - log_n);
  out[off + p] = in[off + src];
}

// ---- batched variants (one launch for a batch of ciphertexts) ---------------------

// NTT-domain automorphism of both polys of ciphertext z = blockIdx.z / 2
// (poly blockIdx.z % 2, stride half) into out: poly 0 of every op first
// (op stride half), then poly 1 (block offset n*half).
__global__ void automorph_ntt_batch(CtPtrs ptr, long half, uint64_t* out, int n, GaloisList gl, int log_n) {
  const long N = 1L << log_n;
  const long p = coef_index();
  const int z = blockIdx.z >> 1, poly = blockIdx.z & 1;
  const uint32_t br = __brev((uint32_t)p) >> (32 - log_n);
  const long e = ((2L * br + 1) * gl.g[z]) & (2 * N - 1);
  const long src = __brev((uint32_t)((e - 1) >> 1)) >> (32 - log_n);
  const long limb = (long)blockIdx.y * N;
  out[(long)poly * n * half + (long)z * half + limb + p] = ptr.a[z][(long)poly * half + limb + src];
}

// tensor for op z = blockIdx.z: a = ptr.a[z], b = ptr.b[z] ([c0 | c1], stride half);
// outputs to the blocks D0 = D, D1 = D + n*half, D2 = D + 2n*half, op stride half.
__global__ void hmult_tensor_batch(CtPtrs ptr, long half, uint64_t* D, int n, const PrimeConst* pc, int log_n) {
  const int z = blockIdx.z;
  const long limb = (long)blockIdx.y << log_n;
  const PrimeConst P = pc[blockIdx.y];
  const long nh = (long)n * half;
  uint64_t* d = D + (long)z * half + limb;
  tensor_ew(ptr.a[z] + limb, half, ptr.b[z] + limb, half, d, d + nh, d + 2 * nh, P);
}

// key products for op z: x limbs (Q part at xq + z*xq_stride, B part at
// xb + z*xb_stride) times the key; k0 of op z at k + z*k_stride, k1 at
// k + (n + z)*k_stride.
// One thread per (limb, kEwPer coefficients) loops over the n ops, so that
// each key word is read from memory once per launch.
__global__ void keyswitch_mul_batch(const uint64_t* xq, long xq_stride, const uint64_t* xb, long xb_stride,
                                    const uint64_t* key, long key_half, uint64_t* k, long k_stride, int n, int nq,
                                    int K, const PrimeConst* pc, int log_n) {
  const long N = 1L << log_n;
  const int l = blockIdx.y;
  const int prime = l < nq ? l : K + (l - nq);
  const uint64_t* x = l < nq ? xq + (long)l * N : xb + (long)(l - nq) * N;
  const long xs = l < nq ? xq_stride : xb_stride;
  const PrimeConst P = pc[prime];
  const uint64_t* kbp = key + (long)prime * N;
  uint64_t kb[kEwPer], ka[kEwPer];
#pragma unroll
  for (int u = 0; u < kEwPer; u++) {
    const long c = coef_u(u);
    kb[u] = kbp[c];
    ka[u] = kbp[key_half + c];
  }
  uint64_t* o = k + (long)l * N;
  for (int z = 0; z < n; z++) {
    uint64_t v[kEwPer];
#pragma unroll
    for (int u = 0; u < kEwPer; u++) v[u] = x[z * xs + coef_u(u)];
#pragma unroll
    for (int u = 0; u < kEwPer; u++) {
      const long c = coef_u(u);
      o[z * k_stride + c] = mul_mod(v[u], kb[u], P);
      o[(n + z) * k_stride + c] = mul_mod(v[u], ka[u], P);
    }
  }
}

// key products with a key per op: op z's x limbs times keys.k[z] (the same
// layout as keyswitch_mul_batch; each op's key words are read for that op)
__global__ void keyswitch_mul_keys(const uint64_t* xq, long xq_stride, const uint64_t* xb, long xb_stride,
                                   KeyPtrs keys, long key_half, uint64_t* k, long k_stride, int n, int nq, int K,
                                   const PrimeConst* pc, int log_n) {
  const long N = 1L << log_n;
  const int l = blockIdx.y;
  const int prime = l < nq ? l : K + (l - nq);
  const uint64_t* x = l < nq ? xq + (long)l * N : xb + (long)(l - nq) * N;
  const long xs = l < nq ? xq_stride : xb_stride;
  const PrimeConst P = pc[prime];
  uint64_t* o = k + (long)l * N;
  for (int z = 0; z < n; z++) {
    const uint64_t* kbp = keys.k[z] + (long)prime * N;
    uint64_t v[kEwPer], kb[kEwPer], ka[kEwPer];
#pragma unroll
    for (int u = 0; u < kEwPer; u++) {
      const long c = coef_u(u);
      v[u] = x[z * xs + c];
      kb[u] = kbp[c];
      ka[u] = kbp[key_half + c];
    }
#pragma unroll
    for (int u = 0; u < kEwPer; u++) {
      const long c = coef_u(u);
      o[z * k_stride + c] = mul_mod(v[u], kb[u], P);
      o[(n + z) * k_stride + c] = mul_mod(v[u], ka[u], P);
    }
  }
}

// ---- host wrappers -----------------------------------------------------------

static dim3 ew_grid(const Engine& E, int nlimbs, int npolys) { return dim3(E.N / 256, nlimbs, npolys); }
static dim3 ew4_grid(const Engine& E, int nlimbs, int npolys) { return dim3(E.N / (256 * kEwPer), nlimbs, npolys); }

void ew_binary_op(const Engine& E, uint64_t* c, long cs, const uint64_t* a, long as, const uint64_t* b, long bs,
                  int op, int prime0, int nlimbs, int npolys, cudaStream_t st) {
  if (nlimbs <= 0 || npolys <= 0) return;
  ew_binary<<<ew_grid(E, nlimbs, npolys), 256, 0, st>>>(Limbs{c, cs}, CLimbs{a, as}, CLimbs{b, bs}, op, prime0,
                                                        E.d_pc, E.log_n); note_launch();
  AOA_CHECK_LAUNCH();
}

void ew_scalar_op(const Engine& E, uint64_t* c, long cs, const uint64_t* a, long as, const uint64_t* d_scalars,
                  int op, int prime0, int nlimbs, int npolys, cudaStream_t st) {
  if (nlimbs <= 0 || npolys <= 0) return;
  ew_scalar<<<ew_grid(E, nlimbs, npolys), 256, 0, st>>>(Limbs{c, cs}, CLimbs{a, as}, d_scalars, op, prime0,
                                                        E.d_pc, E.log_n); note_launch();
  AOA_CHECK_LAUNCH();
}

void ew_muladd_op(const Engine& E, uint64_t* d, long ds, const uint64_t* a, long as, const uint64_t* b, long bs,
                  const uint64_t* c, long cs, int prime0, int nlimbs, int npolys, cudaStream_t st) {
  if (nlimbs <= 0 || npolys <= 0) return;
  ew_muladd<<<ew_grid(E, nlimbs, npolys), 256, 0, st>>>(Limbs{d, ds}, CLimbs{a, as}, CLimbs{b, bs},
                                                        CLimbs{c, cs}, prime0, E.d_pc, E.log_n); note_launch();
  AOA_CHECK_LAUNCH();
}

void tensor_op(const Engine& E, const uint64_t* a, long a_half, const uint64_t* b, long b_half, uint64_t* d0,
               uint64_t* d1, uint64_t* d2, int nlimbs, cudaStream_t st) {
  hmult_tensor<<<ew4_grid(E, nlimbs, 1), 256, 0, st>>>(a, b, a_half, b_half, d0, d1, d2, E.d_pc, E.log_n); note_launch();
  AOA_CHECK_LAUNCH();
}

void tensor_batch_op(const Engine& E, const CtPtrs& ptr, long half, uint64_t* D, int n, int nlimbs, cudaStream_t st) {
  hmult_tensor_batch<<<ew4_grid(E, nlimbs, n), 256, 0, st>>>(ptr, half, D, n, E.d_pc, E.log_n);
  note_launch();
  AOA_CHECK_LAUNCH();
}

void keyswitch_mul_batch_op(const Engine& E, const uint64_t* xq, long xq_stride, const uint64_t* xb, long xb_stride,
                            const uint64_t* key, uint64_t* k, long k_stride, int n, int nq, cudaStream_t st, int nb) {
  const long half = (long)E.nprimes * E.N;
  if (nb < 0) nb = E.kl;
  keyswitch_mul_batch<<<ew4_grid(E, nq + nb, 1), 256, 0, st>>>(xq, xq_stride, xb, xb_stride, key, half, k, k_stride,
                                                               n, nq, E.k, E.d_pc, E.log_n);
  note_launch();
  AOA_CHECK_LAUNCH();
}

void keyswitch_mul_op(const Engine& E, const uint64_t* xq, const uint64_t* xb, const uint64_t* key, uint64_t* k0,
                      uint64_t* k1, int nq, cudaStream_t st, int nb) {
  const long half = (long)E.nprimes * E.N;
  if (nb < 0) nb = E.kl;
  keyswitch_mul<<<ew4_grid(E, nq + nb, 1), 256, 0, st>>>(xq, xb, key, half, k0, k1, nq, E.k, E.d_pc, E.log_n); note_launch();
  AOA_CHECK_LAUNCH();
}

void automorph_coef_op(const Engine& E, uint64_t* out, const uint64_t* in, long poly_stride, long galois,
                       int nlimbs, int npolys, cudaStream_t st) {
  automorph_coef<<<ew_grid(E, nlimbs, npolys), 256, 0, st>>>(out, in, poly_stride, galois, E.d_pc, E.log_n); note_launch();
  AOA_CHECK_LAUNCH();
}

void automorph_ntt_batch_op(const Engine& E, const CtPtrs& ptr, long half, uint64_t* out, int n,
                            const GaloisList& galois, int nlimbs, cudaStream_t st) {
  automorph_ntt_batch<<<ew_grid(E, nlimbs, 2 * n), 256, 0, st>>>(ptr, half, out, n, galois, E.log_n);
  note_launch();
  AOA_CHECK_LAUNCH();
}

void keyswitch_mul_keys_op(const Engine& E, const uint64_t* xq, long xq_stride, const uint64_t* xb, long xb_stride,
                           const KeyPtrs& keys, uint64_t* k, long k_stride, int n, int nq, cudaStream_t st) {
  const long half = (long)E.nprimes * E.N;
  keyswitch_mul_keys<<<ew4_grid(E, nq + E.kl, 1), 256, 0, st>>>(xq, xq_stride, xb, xb_stride, keys, half, k, k_stride,
                                                                 n, nq, E.k, E.d_pc, E.log_n);
  note_launch();
  AOA_CHECK_LAUNCH();
}

void automorph_ntt_op(const Engine& E, uint64_t* out, const uint64_t* in, long poly_stride, long galois,
                      int nlimbs, int npolys, cudaStream_t st) {
  automorph_ntt<<<ew_grid(E, nlimbs, npolys), 256, 0, st>>>(out, in, poly_stride, galois, E.log_n); note_launch();
  AOA_CHECK_LAUNCH();
}

}  // namespace aoa
