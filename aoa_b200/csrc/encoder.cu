// CKKS encode / decode and encrypt / decrypt.
//
// Encode (aoa-ntt src/ckks/encoder.cu:143-221): the slot vector goes through
// the inverse "special" FFT of length `slots` (fftSpecialInv, encoder.cu:75-124),
// is bit-reversed, divided by `slots`, multiplied by the scale, truncated to
// int64 and reduced into every limb at coefficient positions sid*gap (real
// part) and N/2 + sid*gap (imaginary part), gap = (N/2)/slots.  Decode
// (encoder.cu:234-298) reads limb 0 of the coefficient-domain message at the
// same positions, centres and divides by the scale, and runs the forward
// special FFT (fftSpecial, encoder.cu:33-73).  The DGT library's encoder
// (aoa-dgt src/tool/encoder.cu:148-336) writes the same coefficients through
// its folded layout.
//
// The reference runs both FFTs on the host.  Here they run on the device in
// FP64 with every product and sum rounded on its own (__dmul_rn, __dadd_rn,
// __dsub_rn: no fused multiply-add), in the reference's butterfly order, on
// the same host-computed table of roots, so the doubles are the reference's
// bit for bit.  Stages whose butterfly span exceeds one CTA's tile run as one
// launch per stage over the whole vector; the rest run in shared memory.
//
// Encrypt / decrypt (aoa-ntt src/ckks/ckks.cpp:87-105, 179-192): randomness
// enters as inputs (signed u, e1, e2 per coefficient), so results are
// deterministic and comparable with the reference given the same draws.
#include "aoa_internal.h"

using namespace aoa;

namespace aoa {
size_t workspace_words(const Engine& E);
void ct_to_domain(Ctx& C, aoa_ct* ct, int domain, int nlimbs);
}  // namespace aoa

namespace {

constexpr int kFftTile = 2048;            // complex doubles per CTA (32 KiB of shared memory)

__device__ __forceinline__ double2 c_add(double2 a, double2 b) {
  return make_double2(__dadd_rn(a.x, b.x), __dadd_rn(a.y, b.y));
}
__device__ __forceinline__ double2 c_sub(double2 a, double2 b) {
  return make_double2(__dsub_rn(a.x, b.x), __dsub_rn(a.y, b.y));
}
// (a.re b.re - a.im b.im, a.re b.im + a.im b.re), each product rounded
__device__ __forceinline__ double2 c_mul(double2 a, double2 b) {
  return make_double2(__dsub_rn(__dmul_rn(a.x, b.x), __dmul_rn(a.y, b.y)),
                      __dadd_rn(__dmul_rn(a.x, b.y), __dmul_rn(a.y, b.x)));
}

__device__ __forceinline__ unsigned bitrev_bits(unsigned x, int bits) {
  return bits ? __brev(x) >> (32 - bits) : 0u;
}

// Inverse-FFT butterfly at (a, b = a + lenh) with in-group index j
// (fftSpecialInv: u = x + y, v = (x - y) * ksi[(lenq - rot[j] % lenq) * M / lenq]).
__device__ __forceinline__ void inv_bf(double2& x, double2& y, unsigned j, unsigned len, const double2* ksi,
                                       const uint32_t* rot, unsigned M) {
  const unsigned lenq = len << 2;
  const unsigned idx = (lenq - (rot[j] & (lenq - 1))) * (M / lenq);
  const double2 u = c_add(x, y);
  const double2 v = c_mul(c_sub(x, y), ksi[idx]);
  x = u;
  y = v;
}

// Forward-FFT butterfly (fftSpecial: v = y * ksi[(rot[j] % lenq) * M / lenq];
// x, y = x + v, x - v).
__device__ __forceinline__ void fwd_bf(double2& x, double2& y, unsigned j, unsigned len, const double2* ksi,
                                       const uint32_t* rot, unsigned M) {
  const unsigned lenq = len << 2;
  const unsigned idx = (rot[j] & (lenq - 1)) * (M / lenq);
  const double2 v = c_mul(y, ksi[idx]);
  const double2 u = x;
  x = c_add(u, v);
  y = c_sub(u, v);
}

// One stage of span `len` over the whole vector: thread t handles butterfly t.
template <bool INV>
__global__ void fft_stage(double2* v, unsigned size, unsigned len, const double2* __restrict__ ksi,
                          const uint32_t* __restrict__ rot, unsigned M) {
  const unsigned t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= size / 2) return;
  const unsigned lenh = len >> 1;
  const unsigned j = t % lenh;
  const unsigned a = (t / lenh) * len + j;
  double2 x = v[a], y = v[a + lenh];
  if (INV) inv_bf(x, y, j, len, ksi, rot, M);
  else fwd_bf(x, y, j, len, ksi, rot, M);
  v[a] = x;
  v[a + lenh] = y;
}

// Inverse stages len = tile .. 2 on one tile of `tile` consecutive entries.
__global__ void fft_inv_tile(double2* v, unsigned tile, const double2* __restrict__ ksi,
                             const uint32_t* __restrict__ rot, unsigned M) {
  extern __shared__ double2 sv[];
  double2* g = v + (size_t)blockIdx.x * tile;
  for (unsigned i = threadIdx.x; i < tile; i += blockDim.x) sv[i] = g[i];
  __syncthreads();
  for (unsigned len = tile; len >= 2; len >>= 1) {
    const unsigned lenh = len >> 1;
    for (unsigned t = threadIdx.x; t < tile / 2; t += blockDim.x) {
      const unsigned j = t % lenh;
      const unsigned a = (t / lenh) * len + j;
      inv_bf(sv[a], sv[a + lenh], j, len, ksi, rot, M);
    }
    __syncthreads();
  }
  for (unsigned i = threadIdx.x; i < tile; i += blockDim.x) g[i] = sv[i];
}

// ADJUSTSCALE (encoder.cu:131): centred residue of limb 0 divided by the scale.
__device__ __forceinline__ double adjust_scale(uint64_t x, uint64_t p, double factor) {
  return x <= (p >> 1) ? __ddiv_rn((double)x, factor) : __ddiv_rn(__dsub_rn((double)x, (double)p), factor);
}

// Decode front end: the bit-reversed, centred and scaled slot values of one
// tile, then forward stages len = 2 .. tile in shared memory.
__global__ void fft_fwd_tile_from_message(double2* v, const uint64_t* __restrict__ m0, uint64_t p, double factor,
                                          int log_size, unsigned tile, unsigned gap, unsigned half_n,
                                          const double2* __restrict__ ksi, const uint32_t* __restrict__ rot,
                                          unsigned M) {
  extern __shared__ double2 sv[];
  const unsigned base = blockIdx.x * tile;
  for (unsigned i = threadIdx.x; i < tile; i += blockDim.x) {
    const unsigned sid = bitrev_bits(base + i, log_size);
    sv[i] = make_double2(adjust_scale(m0[(size_t)sid * gap], p, factor),
                         adjust_scale(m0[(size_t)sid * gap + half_n], p, factor));
  }
  __syncthreads();
  for (unsigned len = 2; len <= tile; len <<= 1) {
    const unsigned lenh = len >> 1;
    for (unsigned t = threadIdx.x; t < tile / 2; t += blockDim.x) {
      const unsigned j = t % lenh;
      const unsigned a = (t / lenh) * len + j;
      fwd_bf(sv[a], sv[a + lenh], j, len, ksi, rot, M);
    }
    __syncthreads();
  }
  for (unsigned i = threadIdx.x; i < tile; i += blockDim.x) v[base + i] = sv[i];
}

// ADJUSTNEG (encoder.cu:130): x >= 0 ? x mod p : p - (-x mod p), the second
// form giving p itself for a negative multiple of p, as the reference does.
__device__ __forceinline__ uint64_t adjust_neg(int64_t x, const PrimeConst& P) {
  if (x >= 0) return shoup((uint64_t)x, 1, P.one_sh, P.q);
  return P.q - shoup((uint64_t)0 - (uint64_t)x, 1, P.one_sh, P.q);
}

// Encode back end: every coefficient of limbs 0..nlimbs-1 (zeros off the slot
// positions), from the inverse-FFT output in bit-reversed order.
__global__ void encode_residues(uint64_t* out, const double2* __restrict__ v, const PrimeConst* __restrict__ pc,
                                unsigned N, int log_size, unsigned gap, double size_d, double scale_d) {
  const unsigned t = blockIdx.x * blockDim.x + threadIdx.x;
  const int lid = blockIdx.y;
  if (t >= N) return;
  const unsigned half = N >> 1;
  const unsigned pos = t < half ? t : t - half;
  uint64_t r = 0;
  if (pos % gap == 0) {
    const unsigned sid = pos / gap;
    const double2 z = v[bitrev_bits(sid, log_size)];
    const double c = __ddiv_rn(t < half ? z.x : z.y, size_d);
    r = adjust_neg((int64_t)__dmul_rn(c, scale_d), pc[lid]);
  }
  out[(size_t)lid * N + t] = r;
}

// Encrypt front end: U = u, E1 = e1 + m, E2 = e2 in limbs 0..k-1 (coefficients).
__global__ void encrypt_prep(uint64_t* U, uint64_t* E1, uint64_t* E2, const uint64_t* __restrict__ m,
                             const int64_t* __restrict__ u, const int64_t* __restrict__ e1,
                             const int64_t* __restrict__ e2, const PrimeConst* __restrict__ pc, unsigned N) {
  const unsigned t = blockIdx.x * blockDim.x + threadIdx.x;
  const int l = blockIdx.y;
  if (t >= N) return;
  const uint64_t q = pc[l].q;
  auto res = [q](int64_t x) { return x >= 0 ? (uint64_t)x : q - (uint64_t)(-x); };
  const size_t i = (size_t)l * N + t;
  U[i] = res(u[t]);
  E1[i] = add_mod(res(e1[t]), m[i], q);
  E2[i] = res(e2[t]);
}

void* ctx_enc_buffer(Ctx& C, size_t bytes) {
  if (C.enc_bytes < bytes) {
    if (C.enc) AOA_CUDA(cudaFreeAsync(C.enc, C.stream));
    C.enc = nullptr;
    C.enc_bytes = 0;
    if (cudaMallocAsync(&C.enc, bytes, C.stream) != cudaSuccess) {
      cudaGetLastError();
      throw AoaError(AOA_ERR_OOM, "encoder buffer allocation failed");
    }
    C.enc_bytes = bytes;
  }
  return C.enc;
}

int log2_exact(long x) {
  int l = 0;
  while ((1L << l) < x) ++l;
  return (1L << l) == x ? l : -1;
}

bool valid_domain(int d) { return d == AOA_COEF || d == AOA_NTT || d == AOA_DGT; }

}  // namespace

extern "C" {

// ckks_encode (encoder.cu:166-221): `filled` complex values (re, im pairs in
// host memory), `empty` zero slots after them; writes limbs 0..nlimbs-1 of
// d_out ([nlimbs][N]) in `domain`.
int aoa_encode(aoa_ctx* c, const double* host_vals, int filled, int empty, uint64_t scale, int nlimbs, int domain,
               uint64_t* d_out) {
  if (!c || !d_out || (filled > 0 && !host_vals)) return fail(AOA_ERR_BAD_PARAM, "null argument");
  return guarded([&] {
    Ctx& C = c->c;
    const Engine& E = *C.E;
    const long slots = (long)filled + empty;
    const int log_size = log2_exact(slots);
    if (filled < 0 || empty < 0 || slots < 1 || log_size < 0 || slots > E.N / 2)
      throw AoaError(AOA_ERR_BAD_PARAM, "slots must be a power of two in [1, N/2]");
    if (scale == 0) throw AoaError(AOA_ERR_BAD_PARAM, "scale must be positive");
    if (nlimbs < 1 || nlimbs > E.k) throw AoaError(AOA_ERR_BAD_PARAM, "nlimbs out of range");
    if (!valid_domain(domain)) throw AoaError(AOA_ERR_BAD_PARAM, "bad domain");
    double2* v = (double2*)ctx_enc_buffer(C, (size_t)E.N * 8 + 16);
    if (filled)
      AOA_CUDA(cudaMemcpyAsync(v, host_vals, (size_t)filled * 16, cudaMemcpyHostToDevice, C.stream));
    if (empty) AOA_CUDA(cudaMemsetAsync(v + filled, 0, (size_t)empty * 16, C.stream));
    const unsigned M = (unsigned)(2 * E.N);
    const unsigned tile = (unsigned)std::min<long>(slots, kFftTile);
    for (long len = slots; len > (long)tile; len >>= 1) {
      fft_stage<true><<<(unsigned)((slots / 2 + 255) / 256), 256, 0, C.stream>>>(v, (unsigned)slots, (unsigned)len,
                                                                                  E.d_ksi, E.d_rot, M);
      AOA_CHECK_LAUNCH();
      note_launch();
    }
    if (tile >= 2) {
      fft_inv_tile<<<(unsigned)(slots / tile), std::min(tile / 2, 1024u), tile * sizeof(double2), C.stream>>>(
          v, tile, E.d_ksi, E.d_rot, M);
      AOA_CHECK_LAUNCH();
      note_launch();
    }
    dim3 grid((unsigned)((E.N + 255) / 256), (unsigned)nlimbs);
    encode_residues<<<grid, 256, 0, C.stream>>>(d_out, v, E.d_pc, (unsigned)E.N, log_size,
                                                 (unsigned)(E.N / 2 / slots), (double)slots, (double)scale);
    AOA_CHECK_LAUNCH();
    note_launch();
    if (domain != AOA_COEF) xform(E, domain, d_out, 1, 0, nlimbs, nlimbs, true, C.stream);
  });
}

// ckks_decode (encoder.cu:259-298): `slots` complex values (re, im pairs) into
// host memory from limb 0 of d_m (given in `domain`).  Synchronises.
int aoa_decode(aoa_ctx* c, const uint64_t* d_m, int domain, int slots, uint64_t scale, double* host_vals) {
  if (!c || !d_m || !host_vals) return fail(AOA_ERR_BAD_PARAM, "null argument");
  return guarded([&] {
    Ctx& C = c->c;
    const Engine& E = *C.E;
    const int log_size = log2_exact(slots);
    if (slots < 1 || log_size < 0 || slots > E.N / 2)
      throw AoaError(AOA_ERR_BAD_PARAM, "slots must be a power of two in [1, N/2]");
    if (scale == 0) throw AoaError(AOA_ERR_BAD_PARAM, "scale must be positive");
    if (!valid_domain(domain)) throw AoaError(AOA_ERR_BAD_PARAM, "bad domain");
    uint8_t* buf = (uint8_t*)ctx_enc_buffer(C, (size_t)E.N * 16 + 16);
    double2* v = (double2*)buf;                           // N/2 complex
    const uint64_t* m0 = d_m;
    if (domain != AOA_COEF) {                             // COMMONEngine::execute(INVERSE) on limb 0
      uint64_t* limb = (uint64_t*)(buf + (size_t)E.N * 8);
      AOA_CUDA(cudaMemcpyAsync(limb, d_m, (size_t)E.N * 8, cudaMemcpyDeviceToDevice, C.stream));
      xform(E, domain, limb, 1, 0, 1, 1, false, C.stream);
      m0 = limb;
    }
    const unsigned M = (unsigned)(2 * E.N);
    const unsigned tile = (unsigned)std::min<int>(slots, kFftTile);
    fft_fwd_tile_from_message<<<(unsigned)(slots / tile), std::max(1u, std::min(tile / 2, 1024u)),
                                tile * sizeof(double2), C.stream>>>(
        v, m0, E.primes[0], (double)scale, log_size, tile, (unsigned)(E.N / 2 / slots), (unsigned)(E.N / 2), E.d_ksi,
        E.d_rot, M);
    AOA_CHECK_LAUNCH();
    note_launch();
    for (long len = 2L * tile; len <= slots; len <<= 1) {
      fft_stage<false><<<(unsigned)((slots / 2 + 255) / 256), 256, 0, C.stream>>>(v, (unsigned)slots, (unsigned)len,
                                                                                   E.d_ksi, E.d_rot, M);
      AOA_CHECK_LAUNCH();
      note_launch();
    }
    AOA_CUDA(cudaMemcpyAsync(host_vals, v, (size_t)slots * 16, cudaMemcpyDeviceToHost, C.stream));
    AOA_CUDA(cudaStreamSynchronize(C.stream));
  });
}

// ckks_encrypt_poly (ckks.cpp:87-105): out = (u pk.b + e1 + m, u pk.a + e2) in
// the NTT domain at level k-1.  d_m: [k][N] message in `m_domain`; d_u, d_e1,
// d_e2: N signed coefficients each (|x| < every prime).  pk is a
// ciphertext-shaped (b, a) pair over the k Q primes; it is brought to the NTT
// domain in place, as the reference's poly_mul_add does.
int aoa_encrypt(aoa_ctx* c, aoa_ct* out, const uint64_t* d_m, int m_domain, aoa_ct* pk, const int64_t* d_u,
                const int64_t* d_e1, const int64_t* d_e2, int slots, uint64_t scale) {
  if (!c || !out || !d_m || !pk || !d_u || !d_e1 || !d_e2) return fail(AOA_ERR_BAD_PARAM, "null argument");
  return guarded([&] {
    Ctx& C = c->c;
    const Engine& E = *C.E;
    if (!valid_domain(m_domain)) throw AoaError(AOA_ERR_BAD_PARAM, "bad domain");
    if (pk->level != E.k - 1) throw AoaError(AOA_ERR_BAD_PARAM, "the public key must cover every Q prime");
    const size_t limb = (size_t)E.N;
    const size_t need = 3 * E.k * limb * 8;
    if (C.scratch_bytes < need) {
      if (C.scratch) AOA_CUDA(cudaFreeAsync(C.scratch, C.stream));
      C.scratch = nullptr;
      C.scratch_bytes = 0;
      const size_t ws = std::max(need, workspace_words(E) * 8);
      if (cudaMallocAsync(&C.scratch, ws, C.stream) != cudaSuccess) {
        cudaGetLastError();
        throw AoaError(AOA_ERR_OOM, "workspace allocation failed");
      }
      C.scratch_bytes = ws;
    }
    uint64_t* U = (uint64_t*)C.scratch;
    uint64_t* E1 = U + E.k * limb;
    uint64_t* E2 = E1 + E.k * limb;
    const uint64_t* m = d_m;
    if (m_domain != AOA_COEF) {           // poly_add of mixed states works in coefficients
      AOA_CUDA(cudaMemcpyAsync(E2, d_m, E.k * limb * 8, cudaMemcpyDeviceToDevice, C.stream));
      xform(E, m_domain, E2, 1, 0, E.k, E.k, false, C.stream);
      m = E2;
    }
    dim3 grid((unsigned)((E.N + 255) / 256), (unsigned)E.k);
    encrypt_prep<<<grid, 256, 0, C.stream>>>(U, E1, E2, m, d_u, d_e1, d_e2, E.d_pc, (unsigned)E.N);
    AOA_CHECK_LAUNCH();
    note_launch();
    ntt_batch(E, U, 3, 0, E.k, E.k, true, C.stream);      // U, E1, E2: 3 polys of k limbs
    ct_to_domain(C, pk, AOA_NTT, E.k);
    const long half = (long)E.k * E.N;
    // c0 = U b + E1, c1 = U a + E2 (two polys, one launch)
    ew_muladd_op(E, out->d, half, U, 0, pk->d, half, E1, half, 0, E.k, 2, C.stream);
    out->level = E.k - 1;
    out->slots = slots;
    out->scale = scale;
    out->domain = AOA_NTT;
  });
}

// ckks_decrypt_poly (ckks.cpp:179-192): m = c1 s + c0 over limbs 0..level, in
// coefficients, into d_m_out ([level+1][N]).  d_s: [k][N] secret in
// `s_domain`.  The ciphertext is brought to the NTT domain in place (as the
// reference's poly_mul_add does).
int aoa_decrypt(aoa_ctx* c, aoa_ct* ct, const uint64_t* d_s, int s_domain, uint64_t* d_m_out) {
  if (!c || !ct || !d_s || !d_m_out) return fail(AOA_ERR_BAD_PARAM, "null argument");
  return guarded([&] {
    Ctx& C = c->c;
    const Engine& E = *C.E;
    if (!valid_domain(s_domain)) throw AoaError(AOA_ERR_BAD_PARAM, "bad domain");
    const int nl = ct->level + 1;
    const uint64_t* s = d_s;
    if (s_domain != AOA_NTT) {
      uint64_t* tmp = (uint64_t*)ctx_enc_buffer(C, (size_t)E.k * E.N * 8);
      AOA_CUDA(cudaMemcpyAsync(tmp, d_s, (size_t)nl * E.N * 8, cudaMemcpyDeviceToDevice, C.stream));
      if (s_domain == AOA_DGT) xform(E, AOA_DGT, tmp, 1, 0, nl, nl, false, C.stream);
      ntt_batch(E, tmp, 1, 0, nl, nl, true, C.stream);
      s = tmp;
    }
    ct_to_domain(C, ct, AOA_NTT, nl);
    const long half = (long)E.k * E.N;
    ew_muladd_op(E, d_m_out, 0, ct->d + half, 0, s, 0, ct->d, 0, 0, nl, 1, C.stream);
    ntt_batch(E, d_m_out, 1, 0, nl, nl, false, C.stream);
  });
}

}  // extern "C"
