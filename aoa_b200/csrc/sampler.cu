// Device samplers (the reference's Sampler, aoa-ntt src/cuda/sampler.cu:
// 13-230: sample_uniform, sample_DG, sample_Z0, sample_hw), on a documented
// counter-based generator so that every draw is reproducible from
// (seed, stream, index) on any device or on the host:
//   Philox4x32-10 (Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as
//   easy as 1, 2, 3", SC 2011): 10 rounds over a 128-bit counter with a
//   64-bit key; round: (hi0, lo0) = M0 * c0, (hi1, lo1) = M1 * c2,
//   c = (hi1 ^ c1 ^ k0, lo1, hi0 ^ c3 ^ k1, lo0); key += (W0, W1).
// Counter of draw i in stream s: (i mod 2^32, i >> 32, s mod 2^32, s >> 32);
// key = seed.  Outputs:
//   uniform   residue of limb l at coefficient i = (x3 x2 x1 x0 as a 128-bit
//             integer) mod q, counter index l * N + i (bias < 2^-64; the
//             reference reduces one 64-bit Sobol draw, biased up to q / 2^64)
//   gaussian  Box-Muller on the draw's two 64-bit halves (53-bit uniforms),
//             rounded to the nearest integer (sample_DG rounds a normal draw)
//   ternary   exactly hw entries +-1 at the positions of the hw smallest keys
//             (draw word 0, then the index: no ties), sign from draw bit
//             32; the rest 0 (sample_hw: hw = 64; sample_Z0: hw = N/2)
#include "aoa_internal.h"

using namespace aoa;

namespace {

constexpr uint32_t kPhiloxM0 = 0xD2511F53u, kPhiloxM1 = 0xCD9E8D57u;
constexpr uint32_t kPhiloxW0 = 0x9E3779B9u, kPhiloxW1 = 0xBB67AE85u;

__device__ __forceinline__ uint4 philox(uint64_t index, uint64_t stream, uint64_t seed) {
  uint32_t c0 = (uint32_t)index, c1 = (uint32_t)(index >> 32), c2 = (uint32_t)stream, c3 = (uint32_t)(stream >> 32);
  uint32_t k0 = (uint32_t)seed, k1 = (uint32_t)(seed >> 32);
#pragma unroll
  for (int r = 0; r < 10; r++) {
    const uint32_t lo0 = kPhiloxM0 * c0, hi0 = __umulhi(kPhiloxM0, c0);
    const uint32_t lo1 = kPhiloxM1 * c2, hi1 = __umulhi(kPhiloxM1, c2);
    const uint32_t n0 = hi1 ^ c1 ^ k0, n2 = hi0 ^ c3 ^ k1;
    c0 = n0; c1 = lo1; c2 = n2; c3 = lo0;
    k0 += kPhiloxW0;
    k1 += kPhiloxW1;
  }
  return make_uint4(c0, c1, c2, c3);
}

__global__ void sample_uniform_kernel(uint64_t* out, long N, int nlimbs, int first_prime, const PrimeConst* pc,
                                      uint64_t seed, uint64_t stream) {
  const long total = N * nlimbs;
  for (long t = (long)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (long)gridDim.x * blockDim.x) {
    const uint4 r = philox((uint64_t)t, stream, seed);
    const uint64_t lo = ((uint64_t)r.y << 32) | r.x, hi = ((uint64_t)r.w << 32) | r.z;
    out[t] = reduce128(lo, hi, pc[first_prime + t / N]);
  }
}

__global__ void sample_gaussian_kernel(int64_t* out, long n, double sigma, uint64_t seed, uint64_t stream) {
  for (long t = (long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long)gridDim.x * blockDim.x) {
    const uint4 r = philox((uint64_t)t, stream, seed);
    const uint64_t a = ((uint64_t)r.y << 32) | r.x, b = ((uint64_t)r.w << 32) | r.z;
    const double u1 = ((double)(a >> 11) + 1.0) * 0x1.0p-53;        // (0, 1]
    const double u2 = (double)(b >> 11) * 0x1.0p-53;                // [0, 1)
    const double z = sqrt(-2.0 * log(u1)) * cospi(2.0 * u2);
    out[t] = (int64_t)llrint(z * sigma);
  }
}

// One CTA: radix select of the hw smallest 64-bit keys (random word 0 in the
// high 32 bits, the index in the low bits, so all keys differ), 8 bits per pass.
constexpr int kSelThreads = 1024;

__global__ void __launch_bounds__(kSelThreads) sample_ternary_kernel(int64_t* out, long n, long hw, uint64_t seed,
                                                                      uint64_t stream) {
  __shared__ unsigned hist[256];
  __shared__ uint64_t prefix_s, mask_s;
  __shared__ long need_s;
  auto key_of = [&](long i) { return ((uint64_t)philox((uint64_t)i, stream, seed).x << 32) | (uint64_t)i; };
  if (threadIdx.x == 0) {
    prefix_s = 0;
    mask_s = 0;
    need_s = hw;                       // keys still to take below the current prefix
  }
  __syncthreads();
  for (int shift = 56; shift >= 0; shift -= 8) {
    for (int b = threadIdx.x; b < 256; b += blockDim.x) hist[b] = 0;
    __syncthreads();
    const uint64_t prefix = prefix_s, mask = mask_s;
    for (long i = threadIdx.x; i < n; i += blockDim.x) {
      const uint64_t k = key_of(i);
      if ((k & mask) == prefix) atomicAdd(&hist[(k >> shift) & 255], 1u);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      long need = need_s;
      int b = 0;
      for (; b < 255 && (long)hist[b] < need; b++) need -= hist[b];
      prefix_s = prefix | ((uint64_t)b << shift);
      mask_s = mask | ((uint64_t)255 << shift);
      need_s = need;
    }
    __syncthreads();
  }
  // prefix_s is now the hw-th smallest key (keys are distinct)
  const uint64_t kth = prefix_s;
  for (long i = threadIdx.x; i < n; i += blockDim.x) {
    const uint4 r = philox((uint64_t)i, stream, seed);
    const uint64_t k = ((uint64_t)r.x << 32) | (uint64_t)i;
    out[i] = (hw > 0 && k <= kth) ? ((r.y & 1) ? -1 : 1) : 0;
  }
}

__global__ void signed_to_residues_kernel(const int64_t* in, uint64_t* out, long N, int nlimbs, int first_prime,
                                          const PrimeConst* pc) {
  const long total = N * nlimbs;
  for (long t = (long)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (long)gridDim.x * blockDim.x) {
    const uint64_t q = pc[first_prime + t / N].q;
    const int64_t v = in[t % N];
    const uint64_t m = (uint64_t)(v < 0 ? -v : v) % q;
    out[t] = v < 0 ? (m ? q - m : 0) : m;
  }
}

}  // namespace

extern "C" {

// small signed integers (a secret, noise) -> [nlimbs][N] canonical residues
// under primes first_prime .. (the cast of sample_hw / sample_DG)
int aoa_signed_to_residues(aoa_ctx* c, const int64_t* d_in, uint64_t* d_out, int first_prime, int nlimbs) {
  if (!c || !d_in || !d_out) return fail(AOA_ERR_BAD_PARAM, "null argument");
  return guarded([&] {
    const Engine& E = *c->c.E;
    if (first_prime < 0 || nlimbs < 1 || first_prime + nlimbs > E.nprimes)
      throw AoaError(AOA_ERR_BAD_PARAM, "prime range out of bounds");
    signed_to_residues_kernel<<<2 * E.num_sms, 256, 0, c->c.stream>>>(d_in, d_out, E.N, nlimbs, first_prime, E.d_pc);
    note_launch();
    AOA_CHECK_LAUNCH();
  });
}

int aoa_sample_uniform(aoa_ctx* c, uint64_t* d_out, int first_prime, int nlimbs, uint64_t seed, uint64_t stream) {
  if (!c || !d_out) return fail(AOA_ERR_BAD_PARAM, "null argument");
  return guarded([&] {
    const Engine& E = *c->c.E;
    if (first_prime < 0 || nlimbs < 1 || first_prime + nlimbs > E.nprimes)
      throw AoaError(AOA_ERR_BAD_PARAM, "prime range out of bounds");
    sample_uniform_kernel<<<4 * E.num_sms, 256, 0, c->c.stream>>>(d_out, E.N, nlimbs, first_prime, E.d_pc, seed,
                                                                   stream);
    note_launch();
    AOA_CHECK_LAUNCH();
  });
}

int aoa_sample_gaussian(aoa_ctx* c, int64_t* d_out, long n, double sigma, uint64_t seed, uint64_t stream) {
  if (!c || !d_out || n < 0 || !(sigma >= 0)) return fail(AOA_ERR_BAD_PARAM, "bad argument");
  return guarded([&] {
    if (n == 0) return;
    sample_gaussian_kernel<<<2 * c->c.E->num_sms, 256, 0, c->c.stream>>>(d_out, n, sigma, seed, stream);
    note_launch();
    AOA_CHECK_LAUNCH();
  });
}

int aoa_sample_ternary(aoa_ctx* c, int64_t* d_out, long n, long hw, uint64_t seed, uint64_t stream) {
  if (!c || !d_out || n < 0 || hw < 0 || hw > n || n > (1L << 31)) return fail(AOA_ERR_BAD_PARAM, "bad argument");
  return guarded([&] {
    if (n == 0) return;
    sample_ternary_kernel<<<1, kSelThreads, 0, c->c.stream>>>(d_out, n, hw, seed, stream);
    note_launch();
    AOA_CHECK_LAUNCH();
  });
}

}  // extern "C"
