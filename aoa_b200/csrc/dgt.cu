// The DGT variant of the transform (aoa-dgt src/cuda/dgt.cu): a degree-N
// polynomial folded into N/2 Gaussian integers a_j + i a_{j+N/2}, twisted by
// r^n (r^(N/2) = i in GF(p)[i]) and transformed by a length-N/2 cyclic DFT
// with Z_p twiddles, output in bit-reversed order.  Position P holds the
// folded polynomial evaluated at r w^bitrev(P), w = g^((p-1)/(N/2)), which is
// what the reference's hierarchical (N/2 >= 1024) and single-block kernels
// both compute.
//
// B200 layout: a GI limb is stored planar, the N/2 real parts then the N/2
// imaginary parts.  That is exactly the coefficient array of the unfolded
// polynomial, so folding and unfolding cost nothing and every
// coefficient-wise kernel (basis conversion, rescale, automorphisms) runs on
// GI limbs unchanged.  Because the DFT twiddles are in Z_p, the transform
// acts on the two planes independently: one twist pass (GI product by r^n)
// followed by the engine's cyclic limb transform on 2 planes per limb.
#include <vector>

#include "aoa_internal.h"

using namespace aoa;

namespace {

long bitrev_l(long x, int bits) {
  long r = 0;
  for (int i = 0; i < bits; i++) r |= ((x >> i) & 1L) << (bits - 1 - i);
  return r;
}

template <class T>
T* upload(const Engine& E, const std::vector<T>& h) {
  T* d = nullptr;
  AOA_CUDA(cudaMalloc(&d, std::max<size_t>(1, h.size()) * sizeof(T)));
  E.allocations.push_back(d);
  if (!h.empty()) AOA_CUDA(cudaMemcpy(d, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice));
  return d;
}

struct GIh { uint64_t re, im; };

GIh gi_mul_h(GIh a, GIh b, uint64_t q) {
  const uint64_t ac = h_mulmod(a.re, b.re, q), bd = h_mulmod(a.im, b.im, q);
  const uint64_t ad = h_mulmod(a.re, b.im, q), bc = h_mulmod(a.im, b.re, q);
  return {ac >= bd ? ac - bd : ac + (q - bd), (ad + bc) % q};
}

// A root r of i with r^(N/2) = i from the generator: with u of order 2N and
// iota = u^(N/2) (a square root of -1 in Z_p), GF(p)[i] = Z_p x Z_p through
// x + iy -> (x + iota y, x - iota y); r is the preimage of (u, u^-1).
GIh derived_root(uint64_t q, uint64_t g, long N) {
  const uint64_t u = h_powmod(g, (q - 1) / (2 * (uint64_t)N), q);
  const uint64_t ui = h_invmod(u, q);
  const uint64_t iota = h_powmod(u, (uint64_t)N / 2, q);
  const uint64_t inv2 = h_invmod(2, q);
  const uint64_t x = h_mulmod((u + ui) % q, inv2, q);
  const uint64_t y = h_mulmod(h_mulmod(u >= ui ? u - ui : u + (q - ui), inv2, q), h_invmod(iota, q), q);
  return {x, y};
}

// Twist (forward) or untwist (inverse) of GI limbs in place: limb l of poly p
// at data + p*poly_stride + l*N, planes [re | im] of H = N/2 words; entry n
// of the prime's table is r^(+-n) = c + di, applied as the three-product
// (a + ib)(c + id) = (k1 - k3) + i (k1 + k2), k1 = c (a + b), k2 = a (d - c),
// k3 = b (c + d) (a + b < 2q, which a Shoup product takes).  For primes below
// 2^kLazyPrimeBits the products use the three-product quotient of the limb
// transforms (each in [0, 4q); the shorter remainder where q = 1 mod 2^32);
// with lazy_out (a forward twist whose limb transform takes inputs below 16q)
// the results stay in [0, 8q), otherwise they are reduced to [0, q).
template <bool Q1>
__device__ __forceinline__ void gi_twist_lazy(uint64_t* x, int n, int H, const uint64_t* w, uint64_t a, uint64_t b,
                                              uint64_t q, bool lazy_out) {
  auto mul = [&](uint64_t y, uint64_t wv, uint64_t wp) {
    if constexpr (Q1) return shoup_lazy_mad3_q1(y, wv, wp, q);
    else return shoup_lazy_mad3(y, wv, wp, 0 - q);
  };
  const uint64_t q2 = q << 1, q4 = q << 2;
  uint64_t k1 = mul(a + b, w[0], w[H]);
  uint64_t k2 = mul(a, w[2 * H], w[3 * H]);
  uint64_t k3 = mul(b, w[4 * H], w[5 * H]);
  if (lazy_out) {
    x[n] = k1 - k3 + q4;
    x[H + n] = k1 + k2;
    return;
  }
  k1 = k1 >= q2 ? k1 - q2 : k1;
  k1 = k1 >= q ? k1 - q : k1;
  k2 = k2 >= q2 ? k2 - q2 : k2;
  k2 = k2 >= q ? k2 - q : k2;
  k3 = k3 >= q2 ? k3 - q2 : k3;
  k3 = k3 >= q ? k3 - q : k3;
  x[n] = sub_mod(k1, k3, q);
  x[H + n] = add_mod(k1, k2, q);
}

__global__ void gi_twist(uint64_t* data, long poly_stride, int npolys, int first_prime, const uint64_t* __restrict__ tab,
                         int H, const PrimeConst* __restrict__ pc, bool lazy_out) {
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= H) return;
  const int item = blockIdx.y, limb = item / npolys, p = item % npolys;
  const int prime = first_prime + limb;
  uint64_t* x = data + (long)p * poly_stride + (long)limb * 2 * H;
  const uint64_t q = pc[prime].q;
  const uint64_t* w = tab + (long)prime * 6 * H + n;
  const uint64_t a = x[n], b = x[H + n];
  if (q < (1ull << kLazyPrimeBits)) {      // the prime is the same for the whole block
    if ((q & 0xffffffffull) == 1) gi_twist_lazy<true>(x, n, H, w, a, b, q, lazy_out);
    else gi_twist_lazy<false>(x, n, H, w, a, b, q, lazy_out);
    return;
  }
  const uint64_t k1 = shoup(a + b, w[0], w[H], q);
  const uint64_t k2 = shoup(a, w[2 * H], w[3 * H], q);
  const uint64_t k3 = shoup(b, w[4 * H], w[5 * H], q);
  x[n] = sub_mod(k1, k3, q);
  x[H + n] = add_mod(k1, k2, q);
}

// Karatsuba GI product of canonical operands (GIMul, aoa-dgt src/cuda/dgt.cu:530-553).
__device__ __forceinline__ void gi_mul_dev(uint64_t ar, uint64_t ai, uint64_t br, uint64_t bi, uint64_t& cr,
                                           uint64_t& ci, const PrimeConst& P) {
  const uint64_t q = P.q;
  const uint64_t s1 = mul_mod(ar, br, P), s2 = mul_mod(ai, bi, P);
  const uint64_t s3 = mul_mod(add_mod(ar, ai, q), add_mod(br, bi, q), P);
  cr = sub_mod(s1, s2, q);
  ci = sub_mod(s3, add_mod(s1, s2, q), q);
}

// c = a * b element-wise on GI limbs (mul_dgt<GaussianInteger>, dgt.cu:1327-1341).
__global__ void gi_mul(uint64_t* c, long cs, const uint64_t* a, long as, const uint64_t* b, long bs, int prime0,
                       int npolys, int H, const PrimeConst* __restrict__ pc) {
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= H) return;
  const int item = blockIdx.y, limb = item / npolys, p = item % npolys;
  const long off = (long)limb * 2 * H + n;
  const PrimeConst& P = pc[prime0 + limb];
  const uint64_t* x = a + p * as + off;
  const uint64_t* y = b + p * bs + off;
  uint64_t cr, ci;
  gi_mul_dev(x[0], x[H], y[0], y[H], cr, ci, P);
  uint64_t* z = c + p * cs + off;
  z[0] = cr;
  z[H] = ci;
}

// HMult tensor on GI limbs (dr2_dgt, dgt.cu:1252-1283, with the middle term
// as (a0 + a1)(b0 + b1) - d0 - d2 as ckks_mul_without_rescale forms it,
// aoa-dgt src/ckks.cpp:299-306).
__device__ __forceinline__ void gi_tensor_at(const uint64_t* a, long a_half, const uint64_t* b, long b_half,
                                             uint64_t* d0, uint64_t* d1, uint64_t* d2, int H,
                                             const PrimeConst* __restrict__ pc, int n, int limb) {
  const long off = (long)limb * 2 * H + n;
  const PrimeConst& P = pc[limb];
  const uint64_t q = P.q;
  const uint64_t a0r = a[off], a0i = a[off + H], a1r = a[a_half + off], a1i = a[a_half + off + H];
  const uint64_t b0r = b[off], b0i = b[off + H], b1r = b[b_half + off], b1i = b[b_half + off + H];
  uint64_t e0r, e0i, e2r, e2i, sr, si;
  gi_mul_dev(a0r, a0i, b0r, b0i, e0r, e0i, P);
  gi_mul_dev(a1r, a1i, b1r, b1i, e2r, e2i, P);
  gi_mul_dev(add_mod(a0r, a1r, q), add_mod(a0i, a1i, q), add_mod(b0r, b1r, q), add_mod(b0i, b1i, q), sr, si, P);
  d0[off] = e0r; d0[off + H] = e0i;
  d2[off] = e2r; d2[off + H] = e2i;
  d1[off] = sub_mod(sr, add_mod(e0r, e2r, q), q);
  d1[off + H] = sub_mod(si, add_mod(e0i, e2i, q), q);
}

__global__ void gi_tensor(const uint64_t* a, long a_half, const uint64_t* b, long b_half, uint64_t* d0, uint64_t* d1,
                          uint64_t* d2, int H, const PrimeConst* __restrict__ pc) {
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= H) return;
  gi_tensor_at(a, a_half, b, b_half, d0, d1, d2, H, pc, n, blockIdx.y);
}

// the tensor of op z = blockIdx.z of a batch: operands ptr.a[z] / ptr.b[z]
// ([c0 | c1], stride half), outputs D0 = D, D1 = D + n half, D2 = D + 2n half
// at op stride half
__global__ void gi_tensor_batch(CtPtrs ptr, long half, uint64_t* D, int nops, int H, const PrimeConst* __restrict__ pc) {
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= H) return;
  const int z = blockIdx.z;
  uint64_t* d = D + (long)z * half;
  const long nh = (long)nops * half;
  gi_tensor_at(ptr.a[z], half, ptr.b[z], half, d, d + nh, d + 2 * nh, H, pc, n, blockIdx.y);
}

// Key-switch products on GI limbs: k0 = x * key_b, k1 = x * key_a over the QB
// limbs of the extended input (Q limbs < nq at xq, the B limbs at xb).
__device__ __forceinline__ void gi_keyswitch_at(const uint64_t* xq, const uint64_t* xb, const uint64_t* key,
                                                long key_half, uint64_t* k0, uint64_t* k1, int nq, int K, int H,
                                                const PrimeConst* __restrict__ pc, int n, int l) {
  const int prime = l < nq ? l : K + (l - nq);
  const long N = 2L * H;
  const uint64_t* x = (l < nq ? xq + (long)l * N : xb + (long)(l - nq) * N) + n;
  const uint64_t* kb = key + (long)prime * N + n;
  const uint64_t* ka = key + key_half + (long)prime * N + n;
  const PrimeConst& P = pc[prime];
  uint64_t r, i;
  gi_mul_dev(x[0], x[H], kb[0], kb[H], r, i, P);
  k0[(long)l * N + n] = r;
  k0[(long)l * N + n + H] = i;
  gi_mul_dev(x[0], x[H], ka[0], ka[H], r, i, P);
  k1[(long)l * N + n] = r;
  k1[(long)l * N + n + H] = i;
}

__global__ void gi_keyswitch_mul(const uint64_t* xq, const uint64_t* xb, const uint64_t* key, long key_half,
                                 uint64_t* k0, uint64_t* k1, int nq, int K, int H, const PrimeConst* __restrict__ pc) {
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= H) return;
  gi_keyswitch_at(xq, xb, key, key_half, k0, k1, nq, K, H, pc, n, blockIdx.y);
}

// the key products of op z = blockIdx.z: x at xq + z xq_stride (Q limbs) and
// xb + z xb_stride (B limbs), k0 at k + z k_stride, k1 at k + (n + z) k_stride
__global__ void gi_keyswitch_mul_batch(const uint64_t* xq, long xq_stride, const uint64_t* xb, long xb_stride,
                                       const uint64_t* key, long key_half, uint64_t* k, long k_stride, int nops,
                                       int nq, int K, int H, const PrimeConst* __restrict__ pc) {
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= H) return;
  const int z = blockIdx.z;
  gi_keyswitch_at(xq + z * xq_stride, xb + z * xb_stride, key, key_half, k + z * k_stride, k + (nops + z) * k_stride,
                  nq, K, H, pc, n, blockIdx.y);
}

// Reference GaussianInteger layout <-> planar GI limbs.
__global__ void gi_layout(uint64_t* dst, const uint64_t* src, int H, bool to_planar) {
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= H) return;
  const long base = (long)blockIdx.y * 2 * H;
  if (to_planar) {
    dst[base + n] = src[base + 2 * n];
    dst[base + H + n] = src[base + 2 * n + 1];
  } else {
    dst[base + 2 * n] = src[base + n];
    dst[base + 2 * n + 1] = src[base + H + n];
  }
}

NttTables dgt_tables(const Engine& E) {
  NttTables T;
  T.tw = E.d_dtw; T.itw = E.d_ditw; T.pc = E.d_dpc;
  T.log_n = E.log_n - 1; T.prime_shift = 1; T.kind = std::max(E.ntt_kind, 0);
  T.split = E.tune.dgt_split;
  if (E.ntt_kind < 0) T.prime_kind = E.prime_kind.data();
  return T;
}

dim3 gi_grid(const Engine& E, int items) { return dim3((unsigned)((E.N / 2 + 255) / 256), (unsigned)items); }

}  // namespace

namespace aoa {

// Tables of the DGT of folded length H = N/2 for every engine prime
// (DGTEngine::init, aoa-dgt src/cuda/dgt.cu:1696-1945, recast for the merged
// cyclic transform).  roots: 2 per prime or null.
void dgt_init(Engine& E, const uint64_t* roots) {
  const long H = E.N / 2;
  const int lh = E.log_n - 1;
  const int np = E.nprimes;
  std::vector<ShoupW> tw((size_t)np * H), itw((size_t)np * H);
  std::vector<PrimeConst> pc(E.h_pc);
  E.dgt_roots.assign((size_t)2 * np, 0);
  bool bad = false;
#pragma omp parallel for schedule(dynamic)
  for (int p = 0; p < np; p++) {
    const uint64_t q = E.primes[p];
    // cyclic merged table: T[m + j] = w^((H / 2m) bitrev_m(j)) = psi^(bitrev_H(m + j) - H / 2m)
    const uint64_t psi = h_powmod(E.gens[p], (q - 1) / (2 * (uint64_t)H), q);
    std::vector<uint64_t> pw(2 * H);
    pw[0] = 1;
    for (long i = 1; i < 2 * H; i++) pw[i] = h_mulmod(pw[i - 1], psi, q);
    tw[(size_t)p * H] = ShoupW{1, h_shoup_companion(1, q)};
    itw[(size_t)p * H] = tw[(size_t)p * H];
    for (long idx = 1; idx < H; idx++) {
      long m = 1;
      while (2 * m <= idx) m <<= 1;
      const long e = bitrev_l(idx, lh) - H / (2 * m);
      const uint64_t w = pw[e], wi = e ? q - pw[H - e] : 1;   // psi^H = -1, so psi^-e = -psi^(H-e)
      tw[(size_t)p * H + idx] = ShoupW{w, h_shoup_companion(w, q)};
      itw[(size_t)p * H + idx] = ShoupW{wi, h_shoup_companion(wi, q)};
    }
    PrimeConst& c = pc[p];
    c.ninv = h_invmod((uint64_t)H % q, q);
    c.ninv_sh = h_shoup_companion(c.ninv, q);
    c.ninv_w1 = h_mulmod(c.ninv, itw[(size_t)p * H + 1].w, q);
    c.ninv_w1_sh = h_shoup_companion(c.ninv_w1, q);
    // twist root and its inverse
    GIh r = roots ? GIh{roots[2 * p] % q, roots[2 * p + 1] % q} : derived_root(q, E.gens[p], E.N);
    GIh chk = {1, 0}, base = r;
    for (uint64_t e = (uint64_t)H; e; e >>= 1) {        // r^H must be i
      if (e & 1) chk = gi_mul_h(chk, base, q);
      base = gi_mul_h(base, base, q);
    }
    if (chk.re != 0 || chk.im != 1) { bad = true; continue; }
    E.dgt_roots[2 * p] = r.re;
    E.dgt_roots[2 * p + 1] = r.im;
  }
  if (bad) throw AoaError(AOA_ERR_BAD_PARAM, "dgt_roots: a root r does not satisfy r^(N/2) = i");
  E.d_dtw = upload(E, tw);
  E.d_ditw = upload(E, itw);
  E.d_dpc = upload(E, pc);
}

// The twist tables, on the first DGT of the engine (12 words per prime and
// Gaussian integer: 190 MB for 61 primes at N = 2^16).
static void dgt_twist_tables(const Engine& E) {
  std::lock_guard<std::mutex> lock(E.dgt_twist_mu);
  if (E.d_twist) return;
  const long H = E.N / 2;
  const int np = E.nprimes;
  std::vector<uint64_t> tf((size_t)np * 6 * H), uf((size_t)np * 6 * H);
#pragma omp parallel for schedule(dynamic)
  for (int p = 0; p < np; p++) {
    const uint64_t q = E.primes[p];
    const GIh r = {E.dgt_roots[2 * p], E.dgt_roots[2 * p + 1]};
    const uint64_t norm = (uint64_t)(((unsigned __int128)r.re * r.re + (unsigned __int128)r.im * r.im) % q);
    const uint64_t ni = h_invmod(norm, q);
    const GIh ri = {h_mulmod(r.re, ni, q), h_mulmod(r.im ? q - r.im : 0, ni, q)};
    auto put = [&](std::vector<uint64_t>& t, long n, GIh v) {
      uint64_t* base = t.data() + (size_t)p * 6 * H + n;
      const uint64_t c = v.re, dc = (v.im + q - v.re) % q, cd = (v.re + v.im) % q;
      base[0] = c;
      base[H] = h_shoup_companion(c, q);
      base[2 * H] = dc;
      base[3 * H] = h_shoup_companion(dc, q);
      base[4 * H] = cd;
      base[5 * H] = h_shoup_companion(cd, q);
    };
    GIh a = {1, 0}, b = {1, 0};
    for (long n = 0; n < H; n++) {
      put(tf, n, a);
      put(uf, n, b);
      a = gi_mul_h(a, r, q);
      b = gi_mul_h(b, ri, q);
    }
  }
  uint64_t* t = upload(E, tf);
  uint64_t* u = upload(E, uf);
  E.d_untwist = u;
  E.d_twist = t;
}

// DGT / inverse DGT of limbs 0..nlimbs-1 (primes first_prime..) of npolys GI
// polys, poly_stride limbs apart (execute_dgt, aoa-dgt src/cuda/dgt.cu:1055-1096).
void dgt_batch(const Engine& E, uint64_t* data, int npolys, int first_prime, int nlimbs, long poly_stride,
               bool forward, cudaStream_t st) {
  if (npolys <= 0 || nlimbs <= 0) return;
  if (first_prime < 0 || first_prime + nlimbs > E.nprimes)
    throw AoaError(AOA_ERR_BAD_PARAM, "dgt: prime range out of bounds");
  const int H = (int)(E.N / 2);
  const NttTables T = dgt_tables(E);
  dgt_twist_tables(E);
  if (forward) {
    // the limb transforms of rings of 2^11 and more take forward inputs below
    // 16q on their lazy limbs (the smaller ones run canonical butterflies)
    gi_twist<<<gi_grid(E, nlimbs * npolys), 256, 0, st>>>(data, poly_stride * E.N, npolys, first_prime, E.d_twist,
                                                            H, E.d_pc, T.log_n >= 10);
    note_launch();
    AOA_CHECK_LAUNCH();
    ntt_batch_tables(E, T, data, npolys, first_prime, 2 * nlimbs, 2 * poly_stride, true, st);
  } else {
    ntt_batch_tables(E, T, data, npolys, first_prime, 2 * nlimbs, 2 * poly_stride, false, st);
    gi_twist<<<gi_grid(E, nlimbs * npolys), 256, 0, st>>>(data, poly_stride * E.N, npolys, first_prime,
                                                            E.d_untwist, H, E.d_pc, false);
    note_launch();
    AOA_CHECK_LAUNCH();
  }
}

void gi_mul_op(const Engine& E, uint64_t* c, long cs, const uint64_t* a, long as, const uint64_t* b, long bs,
               int prime0, int nlimbs, int npolys, cudaStream_t st) {
  if (nlimbs <= 0 || npolys <= 0) return;
  gi_mul<<<gi_grid(E, nlimbs * npolys), 256, 0, st>>>(c, cs, a, as, b, bs, prime0, npolys, (int)(E.N / 2), E.d_pc);
  note_launch();
  AOA_CHECK_LAUNCH();
}

void gi_tensor_op(const Engine& E, const uint64_t* a, long a_half, const uint64_t* b, long b_half, uint64_t* d0,
                  uint64_t* d1, uint64_t* d2, int nlimbs, cudaStream_t st) {
  gi_tensor<<<gi_grid(E, nlimbs), 256, 0, st>>>(a, a_half, b, b_half, d0, d1, d2, (int)(E.N / 2), E.d_pc);
  note_launch();
  AOA_CHECK_LAUNCH();
}

void gi_tensor_batch_op(const Engine& E, const CtPtrs& ptr, long half, uint64_t* D, int n, int nlimbs,
                        cudaStream_t st) {
  const dim3 g = gi_grid(E, nlimbs);
  gi_tensor_batch<<<dim3(g.x, g.y, n), 256, 0, st>>>(ptr, half, D, n, (int)(E.N / 2), E.d_pc);
  note_launch();
  AOA_CHECK_LAUNCH();
}

void gi_keyswitch_mul_batch_op(const Engine& E, const uint64_t* xq, long xq_stride, const uint64_t* xb,
                               long xb_stride, const uint64_t* key, uint64_t* k, long k_stride, int n, int nq,
                               cudaStream_t st) {
  const dim3 g = gi_grid(E, nq + E.kl);
  gi_keyswitch_mul_batch<<<dim3(g.x, g.y, n), 256, 0, st>>>(xq, xq_stride, xb, xb_stride, key,
                                                              (long)(E.k + E.kl) * E.N, k, k_stride, n, nq, E.k,
                                                              (int)(E.N / 2), E.d_pc);
  note_launch();
  AOA_CHECK_LAUNCH();
}

void gi_keyswitch_mul_op(const Engine& E, const uint64_t* xq, const uint64_t* xb, const uint64_t* key, uint64_t* k0,
                         uint64_t* k1, int nq, cudaStream_t st) {
  gi_keyswitch_mul<<<gi_grid(E, nq + E.kl), 256, 0, st>>>(xq, xb, key, (long)(E.k + E.kl) * E.N, k0, k1, nq, E.k,
                                                          (int)(E.N / 2), E.d_pc);
  note_launch();
  AOA_CHECK_LAUNCH();
}

}  // namespace aoa

extern "C" {

// execute_dgt FORWARD / INVERSE (aoa-dgt src/cuda/dgt.cu:1055-1096) on planar
// GI limbs laid out [npolys][poly_stride][N].
int aoa_dgt_fwd(aoa_ctx* c, uint64_t* d, int npolys, int first_prime, int nlimbs, int poly_stride) {
  if (!c || !d) return fail(AOA_ERR_BAD_PARAM, "null argument");
  return guarded([&] {
    if (poly_stride < nlimbs) throw AoaError(AOA_ERR_BAD_PARAM, "poly_stride < nlimbs");
    dgt_batch(*c->c.E, d, npolys, first_prime, nlimbs, poly_stride, true, c->c.stream);
  });
}

int aoa_dgt_inv(aoa_ctx* c, uint64_t* d, int npolys, int first_prime, int nlimbs, int poly_stride) {
  if (!c || !d) return fail(AOA_ERR_BAD_PARAM, "null argument");
  return guarded([&] {
    if (poly_stride < nlimbs) throw AoaError(AOA_ERR_BAD_PARAM, "poly_stride < nlimbs");
    dgt_batch(*c->c.E, d, npolys, first_prime, nlimbs, poly_stride, false, c->c.stream);
  });
}

// mul_dgt<GaussianInteger> (dgt.cu:1327-1341): c = a * b on nlimbs planar GI
// limbs (primes first_prime..), transform domain.
int aoa_gi_mul(aoa_ctx* c, uint64_t* d_c, const uint64_t* d_a, const uint64_t* d_b, int first_prime, int nlimbs) {
  if (!c || !d_c || !d_a || !d_b) return fail(AOA_ERR_BAD_PARAM, "null argument");
  return guarded([&] {
    const Engine& E = *c->c.E;
    if (first_prime < 0 || nlimbs < 0 || first_prime + nlimbs > E.nprimes)
      throw AoaError(AOA_ERR_BAD_PARAM, "prime range out of bounds");
    gi_mul_op(E, d_c, 0, d_a, 0, d_b, 0, first_prime, nlimbs, 1, c->c.stream);
  });
}

// The reference's GaussianInteger arrays ({re, im} pairs, [nlimbs][N/2]) to
// planar GI limbs and back.  dst and src must not overlap.
int aoa_gi_to_planar(aoa_ctx* c, uint64_t* d_dst, const uint64_t* d_src, int nlimbs) {
  if (!c || !d_dst || !d_src) return fail(AOA_ERR_BAD_PARAM, "null argument");
  return guarded([&] {
    const Engine& E = *c->c.E;
    if (nlimbs <= 0) return;
    gi_layout<<<gi_grid(E, nlimbs), 256, 0, c->c.stream>>>(d_dst, d_src, (int)(E.N / 2), true);
    note_launch();
    AOA_CHECK_LAUNCH();
  });
}

int aoa_gi_from_planar(aoa_ctx* c, uint64_t* d_dst, const uint64_t* d_src, int nlimbs) {
  if (!c || !d_dst || !d_src) return fail(AOA_ERR_BAD_PARAM, "null argument");
  return guarded([&] {
    const Engine& E = *c->c.E;
    if (nlimbs <= 0) return;
    gi_layout<<<gi_grid(E, nlimbs), 256, 0, c->c.stream>>>(d_dst, d_src, (int)(E.N / 2), false);
    note_launch();
    AOA_CHECK_LAUNCH();
  });
}

// The DGT twist roots the engine uses (2 per prime: re, im).
int aoa_engine_dgt_roots(const aoa_engine* e, uint64_t* out) {
  if (!e || !out) return fail(AOA_ERR_BAD_PARAM, "null argument");
  std::copy(e->e.dgt_roots.begin(), e->e.dgt_roots.end(), out);
  return AOA_OK;
}

// Transform used by this context's evaluations (ckks_mul & co.): AOA_NTT (the
// aoa-ntt library) or AOA_DGT (the aoa-dgt library).
int aoa_ctx_set_transform(aoa_ctx* c, int domain) {
  if (!c || (domain != AOA_NTT && domain != AOA_DGT)) return fail(AOA_ERR_BAD_PARAM, "bad transform");
  return guarded([&] {
    if (domain == AOA_DGT) dgt_twist_tables(*c->c.E);    // allocated now, not inside later evaluations
    c->c.transform = domain;
  });
}

}  // extern "C"
