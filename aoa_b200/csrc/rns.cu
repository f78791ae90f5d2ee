// RNS basis conversion (ModUp / ModDown), rescale and the key-switch epilogues.
// The conversion runs on the int8 tensor cores (basis_convert_tc) when both
// bases have at most 32 primes, else on the CUDA cores (basis_convert).
//
// Both conversions are small dense modular matrix products per coefficient:
//   ModUp   (fast_conv_Q_to_B_opt, aoa-ntt src/cuda/manager.cu:180-223)
//     B_j = sum_{i<=l} [x_i (Q_l/q_i)^-1]_{q_i} * [(Q_l/q_i)]_{b_j}   mod b_j
//   ModDown (fast_conv_B_to_Q, manager.cu:312-341)
//     out_i = (x_i - conv_i) * B^-1 mod q_i,
//     conv_i = sum_j [x_j (B/b_j)^-1]_{b_j} * [(B/b_j)]_{q_i}          mod q_i
// The reference reduces after every term (mulmod + addmod per term); here the
// products accumulate exactly in 128 bits and each output is reduced once
// (the 128-bit bound is checked per engine in rns_init).  The exact residues
// are identical.  One thread owns one coefficient and keeps 16 accumulators in
// registers; a CTA covers 128 coefficients x 32 outputs, the constant matrix
// slice sits in shared memory and is read as a warp broadcast.
//
// Epilogues (what a conversion writes, per output limb i under prime p_i):
//   kRaw        out = conv_i                                  (ModUp; ModDown's conv)
//   kModDown    out = (x_i - conv_i) * B^-1                   (ModDown, coefficients)
//   kRescaleTop out = u_l - conv_l * B^-1                      (c_l: limb l of d + ModDown(x),
//                                                               u_l = d_l + x_l B^-1 in coefficients)
//   kRescaleY   out = conv_i * B^-1 + [c_l]_{q_i}              (merged ModDown + rescale)
//   kRescaleFused  both in one pass when all outputs 0..l fit one launch: the
//               thread owning output l shares c_l through shared memory
#include "aoa_internal.h"
#include "async.cuh"

namespace aoa {

constexpr int kConvOut = 32;     // outputs per launch: kConvHalves groups of kConvAcc
constexpr int kConvAcc = 16;     // register accumulators per thread
constexpr int kConvHalves = kConvOut / kConvAcc;
constexpr int kConvCoefs = 128;  // coefficients per CTA
constexpr int kConvThreads = kConvCoefs * kConvHalves;

enum { kRaw = 0, kModDown = 1, kRescaleTop = 2, kRescaleY = 3, kRescaleFused = 4 };

// in:  nin limbs at `in` (stride N), under primes in_prime0 + i
// out: limbs j in [j_begin, j_end) at `out` + (j - out_shift)*N, under primes out_prime0 + j
// zc[i]  : Shoup constant applied to input limb i before the product
// mat    : [nin][mat_ld] matrix, entry (i, j) = multiplier of z_i for output j
struct ConvArgs {
  const uint64_t* in;
  uint64_t* out;
  const uint64_t* x;        // kModDown: x limbs (limb j at x + (j - x_shift)*N)
  const uint64_t* d;        // kRescaleTop / kRescaleFused: u_l;  kRescaleY: c_l (one limb per poly)
  long in_poly_stride, out_poly_stride, x_poly_stride, d_poly_stride;   // in words
  int nin, mat_ld;
  int in_prime0, out_prime0;
  int out_shift, x_shift;
  const ShoupW* zc;
  const uint64_t* mat;
  const ShoupW* binv;       // B^-1 mod q_j (Shoup form), indexed by output j
  const PrimeConst* pc;
  int log_n;
  int mode;
  const uint8_t* tc_b;      // tensor-core image of `mat` (null: CUDA-core kernel only)
  unsigned* err;            // device error word
  int npolys;
  int spin;                 // polls of a bounded wait for this kernel's own copies and MMAs (engine knob)
};

// Epilogue of the non-fused modes for output jj with the reduced sum r.
__device__ __forceinline__ void conv_store(const ConvArgs& a, int jj, uint64_t r, uint64_t dv, uint64_t* out, long c,
                                           long N, long poly) {
  const PrimeConst& P = a.pc[a.out_prime0 + jj];
  if (a.mode == kModDown) {
    const uint64_t x = a.x[poly * a.x_poly_stride + (long)(jj - a.x_shift) * N + c];
    r = shoup(sub_mod(x, r, P.q), a.binv[jj], P.q);
  } else if (a.mode == kRescaleTop) {
    r = sub_mod(dv, shoup(r, a.binv[jj], P.q), P.q);
  } else if (a.mode == kRescaleY) {
    r = add_mod(shoup(r, a.binv[jj], P.q), shoup(dv, 1, P.one_sh, P.q), P.q);
  }
  out[(long)(jj - a.out_shift) * N] = r;
}

__global__ void __launch_bounds__(kConvThreads, 2)
basis_convert(ConvArgs a, int j_first, int j_end) {
  extern __shared__ uint64_t smat[];    // [nin][kConvOut]
  const int nout = min(kConvOut, j_end - j_first);
  for (int e = threadIdx.x; e < a.nin * kConvOut; e += blockDim.x) {
    const int i = e / kConvOut, j = e % kConvOut;
    smat[e] = j < nout ? a.mat[(long)i * a.mat_ld + j_first + j] : 0;
  }
  __syncthreads();
  const long N = 1L << a.log_n;
  const int half = threadIdx.x / kConvCoefs;          // which kConvAcc outputs of this launch
  const long c = (long)blockIdx.x * kConvCoefs + (threadIdx.x % kConvCoefs);
  const uint64_t* in = a.in + blockIdx.y * a.in_poly_stride + c;
  uint64_t lo[kConvAcc], hi[kConvAcc];
#pragma unroll
  for (int j = 0; j < kConvAcc; j++) lo[j] = hi[j] = 0;
  uint64_t x_next = in[0];
  for (int i = 0; i < a.nin; i++) {
    const uint64_t xi = x_next;
    if (i + 1 < a.nin) x_next = in[(long)(i + 1) * N];     // prefetch the next input limb
    const uint64_t qi = a.pc[a.in_prime0 + i].q;
    const uint64_t z = shoup(xi, a.zc[i], qi);
    const uint64_t* row = smat + i * kConvOut + half * kConvAcc;
#pragma unroll
    for (int j = 0; j < kConvAcc; j++) mac128(lo[j], hi[j], z, row[j]);
  }
  uint64_t* out = a.out + blockIdx.y * a.out_poly_stride + c;
  uint64_t dv = 0;
  if (a.mode >= kRescaleTop) dv = a.d[blockIdx.y * a.d_poly_stride + c];
  if (a.mode == kRescaleFused) {
    // outputs 0..l with l = j_end - 1 < kConvOut: c_l first, shared through smem
    __shared__ uint64_t s_cl[kConvCoefs];
    const int l = j_end - 1;
    if (half == l / kConvAcc) {
#pragma unroll
      for (int jl = 0; jl < kConvAcc; jl++)
        if (jl == l % kConvAcc) {
          const PrimeConst& P = a.pc[a.out_prime0 + l];
          const uint64_t r = reduce128(lo[jl], hi[jl], P);
          s_cl[threadIdx.x % kConvCoefs] = sub_mod(dv, shoup(r, a.binv[l], P.q), P.q);
        }
    }
    __syncthreads();
    const uint64_t cl = s_cl[threadIdx.x % kConvCoefs];
#pragma unroll
    for (int jl = 0; jl < kConvAcc; jl++) {
      const int j = half * kConvAcc + jl;
      if (j < l) {
        const PrimeConst& P = a.pc[a.out_prime0 + j];
        const uint64_t r = reduce128(lo[jl], hi[jl], P);
        out[(long)(j - a.out_shift) * N] = add_mod(shoup(r, a.binv[j], P.q), shoup(cl, 1, P.one_sh, P.q), P.q);
      }
    }
    return;
  }
#pragma unroll
  for (int jl = 0; jl < kConvAcc; jl++) {
    const int j = half * kConvAcc + jl;
    if (j < nout) {
      const int jj = j_first + j;
      conv_store(a, jj, reduce128(lo[jl], hi[jl], a.pc[a.out_prime0 + jj]), dv, out, c, N, blockIdx.y);
    }
  }
}

// ---- tensor-core variant ------------------------------------------------------------
// The conversion as one int8 GEMM per 128-coefficient tile on the 5th-generation
// tensor cores.  With the scaled inputs z_i split into their 8 bytes z_i[a],
// sum_i z_i h_ij = sum_i sum_a z_i[a] (h_ij 2^(8a)), and modulo the output
// prime p_j the factor h_ij 2^(8a) can be replaced by its residue
// g_ija = h_ij 2^(8a) mod p_j.  Splitting g_ija into bytes g_ija[b]:
//   sum_i z_i h_ij = sum_b 2^(8b) T_jb  (mod p_j),
//   T_jb = sum_i sum_a z_i[a] g_ija[b] < 8 * 32 * 255^2 < 2^24  (at most 32 inputs).
// That is C = A B with
//   A[row][8i + a] = z_i[a]            (the bytes of z_i: just z_i stored as u64)
//   B[8i + a][8j + b] = g_ija[b]       (a precomputed image per table)
// so one tcgen05.mma kind::i8 (M = 128, N = 256, K = 32 per instruction,
// u8 x u8 -> s32 in tensor memory) computes the 8 byte sums of all 32
// outputs per K step (4 inputs).  The epilogue reads each thread's 8 columns
// of an output from tensor memory (tcgen05.ld), forms sum_b 2^(8b) T_jb <
// 2^81 and reduces it once.
// Shared memory (no swizzle, K-major "core matrices" of 8 rows x 16 bytes):
//   A: [16 k-chunks][128 rows][16 B]   = 32 KiB, descriptor LBO 2048, SBO 128
//   B: [16 k-chunks][256 rows][16 B]   = 64 KiB, descriptor LBO 4096, SBO 128
constexpr int kTcRowsLog = 7;
constexpr int kTcRows = 1 << kTcRowsLog;
constexpr int kTcThreads = 512;
constexpr int kTcN = 256;
constexpr size_t kTcA = 16 * kTcRows * 16;
constexpr size_t kTcB = 16 * kTcN * 16;
constexpr size_t kTcSmem = kTcA + kTcB + 1024;
constexpr uint32_t kTcCols = 256;

__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((saddr >> 4) & 0x3FFF) | ((uint64_t)((lbo >> 4) & 0x3FFF) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFF) << 32) | (1ull << 46);   // version 1, no swizzle
}

// instruction descriptor: s32 accumulator, u8 x u8, both K-major, M = 128, N = 256
constexpr uint32_t kTcIdesc = (2u << 4) | (uint32_t(256 >> 3) << 17) | (uint32_t(128 >> 4) << 24);

__device__ __forceinline__ void tc_mma(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}"
      ::"r"(d_tmem), "l"(adesc), "l"(bdesc), "r"(kTcIdesc), "r"(accumulate), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
}

__device__ __forceinline__ void tc_commit(uint64_t* mb) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(mb))
               : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

__device__ __forceinline__ void tc_ld16(uint32_t taddr, uint32_t (&v)[16]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15}, [%16];"
      : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
        "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

// sum_b T_b 2^(8b) (b < 8, T_b < 2^24) reduced mod P.  W_0 = sum_t T_t 2^(8t)
// and W_1 = sum_t T_(4+t) 2^(8t) (< 2^49 each) come from 32 x 32 -> 64-bit
// multiply-adds; x = W_0 + W_1 2^32 < 2^81 has a high word below 2^17, so
// one Barrett step (s >= 32) reduces it.
// an output prime's constants, staged in shared memory once per CTA
struct TcOut {
  uint64_t q, mu, sh, one_sh;
};

// Q1: every input and output prime of the launch is q = 1 mod 2^32 below
// 2^60 (the engine's butterfly kind kButterflyLazyQ1): the quotient times q
// in the reductions and Shoup products takes one 32-bit multiply (mul_q1).
template <bool Q1>
__device__ __forceinline__ uint64_t tc_combine(const uint32_t* v, const TcOut& c, const PrimeConst* P) {
  uint64_t W0 = v[0], W1 = v[4];
  asm("mad.wide.u32 %0, %1, 256, %0;" : "+l"(W0) : "r"(v[1]));
  asm("mad.wide.u32 %0, %1, 256, %0;" : "+l"(W1) : "r"(v[5]));
  asm("mad.wide.u32 %0, %1, 65536, %0;" : "+l"(W0) : "r"(v[2]));
  asm("mad.wide.u32 %0, %1, 65536, %0;" : "+l"(W1) : "r"(v[6]));
  asm("mad.wide.u32 %0, %1, 16777216, %0;" : "+l"(W0) : "r"(v[3]));
  asm("mad.wide.u32 %0, %1, 16777216, %0;" : "+l"(W1) : "r"(v[7]));
  uint32_t r1, r2;
  asm("add.cc.u32 %0, %2, %3;\n\t"
      "addc.u32 %1, %4, 0;"
      : "=r"(r1), "=r"(r2)
      : "r"((uint32_t)(W0 >> 32)), "r"((uint32_t)W1), "r"((uint32_t)(W1 >> 32)));
  const uint64_t lo = ((uint64_t)r1 << 32) | (uint32_t)W0;
  if (c.sh) return Q1 ? barrett_wide_q1(lo, r2, c.q, c.mu, (uint32_t)c.sh) : barrett_wide(lo, r2, c.q, c.mu, (uint32_t)c.sh);
  return reduce128(lo, r2, *P);
}

// exact Shoup product of the conversion kernel's epilogue
template <bool Q1>
__device__ __forceinline__ uint64_t tc_shoup(uint64_t a, uint64_t w, uint64_t wp, uint64_t q) {
  return Q1 ? shoup_q1(a, w, wp, q) : shoup(a, w, wp, q);
}

// an input scaled by its CRT constant, z = [x w]_q in [0, q): for Q1 primes
// the transforms' three-product quotient with the short remainder ([0, 4q))
// and two conditional subtractions
template <bool Q1>
__device__ __forceinline__ uint64_t tc_scale(uint64_t x, ShoupW w, uint64_t q) {
  if constexpr (Q1) {
    uint64_t r = shoup_lazy_mad3_q1(x, w.w, w.wp, q);
    r = r >= 2 * q ? r - 2 * q : r;
    return r >= q ? r - q : r;
  } else {
    return shoup(x, w, q);
  }
}

// x mod q_out for x < p (another prime): one subtraction when p < 2 q_out
template <bool Q1>
__device__ __forceinline__ uint64_t tc_cross(uint64_t x, uint64_t p, const TcOut& c) {
  if (p < 2 * c.q) return x >= c.q ? x - c.q : x;
  return tc_shoup<Q1>(x, 1, c.one_sh, c.q);
}

// Persistent: CTA b handles tiles b, b + grid, ...  Per tile: the inputs (loaded
// into registers during the previous tile's MMA and epilogue) are scaled and
// written to A, one thread issues the MMAs and commits them to an mbarrier,
// and all 16 warps read tensor memory: warp w owns lanes 32 (w % 4) .. + 31
// (tile rows) and every fourth output starting at w / 4.
constexpr int kTcPairs = 32 / 2 / (kTcThreads / kTcRows);   // input pairs per thread (nin <= 32)

template <int MODE, bool Q1>
__global__ void __launch_bounds__(kTcThreads, 1)
basis_convert_tc(ConvArgs a, int j_first, int j_end) {
  extern __shared__ __align__(1024) uint8_t tcs[];
  __shared__ __align__(8) uint64_t mbar[2];                // [0] image loaded, [1] MMA done
  __shared__ uint32_t tmem_slot;
  __shared__ ShoupW s_zc[32];                              // input scalings
  __shared__ uint64_t s_qin[32];                           // input primes
  __shared__ TcOut s_out[32];                              // output primes' constants
  uint8_t* As = tcs;
  uint8_t* Bs = tcs + kTcA;
  const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
  const long N = 1L << a.log_n;
  const int tile_shift = a.log_n - kTcRowsLog;             // tiles per poly = N / kTcRows = 2^tile_shift
  const long ntiles = (long)a.npolys << tile_shift;
  const int npairs = (a.nin + 1) / 2;
  // zero A (inputs beyond nin stay zero), barriers, tensor memory, the table image
  for (int e = threadIdx.x; e < (int)(kTcA / 16); e += blockDim.x) ((uint4*)As)[e] = make_uint4(0, 0, 0, 0);
  if (threadIdx.x == 0) {
    mbar_init(&mbar[0], 1);
    mbar_init(&mbar[1], 1);
    mbar_init_fence();
  }
  if (threadIdx.x < 32) {
    const int i = threadIdx.x;
    if (i < a.nin) {
      s_zc[i] = a.zc[i];
      s_qin[i] = a.pc[a.in_prime0 + i].q;
    }
    if (i < j_end) {
      const PrimeConst& P = a.pc[a.out_prime0 + i];
      s_out[i] = TcOut{P.q, P.bar_mu, P.bar_sh, P.one_sh};
    }
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_slot)),
                 "r"(kTcCols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  fence_proxy_async();
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = tmem_slot;
  if (threadIdx.x == 0) {
    mbar_expect_tx(&mbar[0], (unsigned)kTcB);
    for (int c = 0; c < (int)(kTcB / 16384); c++)
      bulk_g2s(smem_u32(Bs + c * 16384), a.tc_b + c * 16384, 16384, &mbar[0]);
  }
  // this thread's A rows / input pairs, and its prefetched inputs
  const int ar = threadIdx.x % kTcRows, ap = threadIdx.x / kTcRows;
  uint64_t xa[kTcPairs], xb[kTcPairs];
  // the rescale modes' own-limb word of this thread's epilogue row, fetched
  // with the inputs so that its latency is hidden too
  uint64_t dv_next = 0;
  const int erow = (warp % 4) * 32 + lane;
  auto load_inputs = [&](long tile) {
    const long poly = tile >> tile_shift, c0 = (tile & ((1L << tile_shift) - 1)) * kTcRows;
    const uint64_t* in = a.in + poly * a.in_poly_stride + c0 + ar;
#pragma unroll
    for (int m = 0; m < kTcPairs; m++) {
      const int p = ap + m * (kTcThreads / kTcRows);
      xa[m] = p < npairs ? in[(long)(2 * p) * N] : 0;
      xb[m] = 2 * p + 1 < a.nin ? in[(long)(2 * p + 1) * N] : 0;
    }
    if (MODE >= kRescaleTop) dv_next = a.d[poly * a.d_poly_stride + c0 + erow];
  };
  if (blockIdx.x < ntiles) load_inputs(blockIdx.x);
  bool ok = __syncthreads_and(mbar_wait(&mbar[0], 0, a.spin));
  bool in_flight = false;                                  // an MMA group not yet waited for
  const uint32_t a_base = smem_u32(As), b_base = smem_u32(Bs);
  const int ksteps = (a.nin + 3) / 4;                      // 4 inputs (32 bytes) per MMA K step
  uint32_t phase = 0;
  for (long tile = blockIdx.x; tile < ntiles && ok; tile += gridDim.x) {
    const long poly = tile >> tile_shift;
    const long c0 = (tile & ((1L << tile_shift) - 1)) * kTcRows;
    // A: row ar, inputs 2p and 2p + 1 as one 16-byte store at chunk p
#pragma unroll
    for (int m = 0; m < kTcPairs; m++) {
      const int p = ap + m * (kTcThreads / kTcRows);
      if (p < npairs) {
        const int i0 = 2 * p, i1 = 2 * p + 1;
        const uint64_t z0 = tc_scale<Q1>(xa[m], s_zc[i0], s_qin[i0]);
        const uint64_t z1 = i1 < a.nin ? tc_scale<Q1>(xb[m], s_zc[i1], s_qin[i1]) : 0;
        *(uint4*)(As + (size_t)p * (kTcRows * 16) + ar * 16) =
            make_uint4((uint32_t)z0, (uint32_t)(z0 >> 32), (uint32_t)z1, (uint32_t)(z1 >> 32));
      }
    }
    fence_proxy_async();                                   // generic smem writes -> tensor-core reads
    __syncthreads();
    if (threadIdx.x == 0) {
      tc_fence_after();
      for (int st = 0; st < ksteps; st++) {
        const uint64_t ad = umma_desc(a_base + st * 2 * (kTcRows * 16), kTcRows * 16, 128);
        const uint64_t bd = umma_desc(b_base + st * 2 * (kTcN * 16), kTcN * 16, 128);
        tc_mma(tmem, ad, bd, st > 0);
      }
      tc_commit(&mbar[1]);
    }
    in_flight = true;
    const uint64_t dv_cur = dv_next;                       // this tile's word, loaded with its inputs
    if (tile + gridDim.x < ntiles) load_inputs(tile + gridDim.x);   // overlaps the MMAs and the epilogue
    ok = !__syncthreads_or(!mbar_wait(&mbar[1], phase, a.spin));
    if (!ok) break;
    in_flight = false;
    phase ^= 1;
    tc_fence_after();
    // warp w reads tensor-memory lanes 32 (w % 4) .. + 31 (tile rows) and a
    // contiguous run of outputs: quarter w / 4 of them, two per load
    const int g = warp % 4, par = warp / 4;
    const long c = c0 + g * 32 + lane;
    const uint32_t t_lane = tmem + ((uint32_t)(g * 32) << 16);
    uint64_t* out = a.out + poly * a.out_poly_stride + c;
    const uint64_t dv = dv_cur;
    uint32_t v[16];
    if (MODE == kRescaleFused) {
      const int l = j_end - 1;                 // outputs 0..l-1 from c_l (j_first = 0)
      tc_ld16(t_lane + (l & ~1) * 8, v);
      const TcOut cpl = s_out[l];
      const PrimeConst* Pl = a.pc + a.out_prime0 + l;
      // the rescale modes read the table with B^-1 folded in: sums are conv * B^-1
      const uint64_t sl = (l & 1) ? tc_combine<Q1>(v + 8, cpl, Pl) : tc_combine<Q1>(v, cpl, Pl);
      const uint64_t cl = sub_mod(dv, sl, cpl.q);
      const int per = (((l + 3) / 4) + 1) & ~1;
      const int jb = par * per, je = min(l, jb + per);
      for (int j = jb; j < je; j += 2) {
        tc_ld16(t_lane + j * 8, v);
#pragma unroll
        for (int u = 0; u < 2; u++) {
          if (j + u < je) {
            const TcOut cp = s_out[j + u];
            out[(long)(j + u - a.out_shift) * N] =
                add_mod(tc_combine<Q1>(v + 8 * u, cp, a.pc + a.out_prime0 + j + u), tc_cross<Q1>(cl, cpl.q, cp),
                        cp.q);
          }
        }
      }
    } else {
      const int nout = j_end - j_first;
      const int per = (((nout + 3) / 4) + 1) & ~1;
      const int jb = j_first + par * per, je = min(j_end, jb + per);
      for (int jj = jb & ~1; jj < je; jj += 2) {
        tc_ld16(t_lane + jj * 8, v);
#pragma unroll
        for (int u = 0; u < 2; u++) {
          const int o = jj + u;
          if (o >= jb && o < je) {
            const TcOut cp = s_out[o];
            uint64_t r = tc_combine<Q1>(v + 8 * u, cp, a.pc + a.out_prime0 + o);
            if (MODE == kModDown) {
              const uint64_t x = a.x[poly * a.x_poly_stride + (long)(o - a.x_shift) * N + c];
              r = tc_shoup<Q1>(sub_mod(x, r, cp.q), a.binv[o].w, a.binv[o].wp, cp.q);
            } else if (MODE == kRescaleTop) {
              r = sub_mod(dv, r, cp.q);                            // folded table: r = conv * B^-1
            } else if (MODE == kRescaleY) {
              r = add_mod(r, tc_shoup<Q1>(dv, 1, cp.one_sh, cp.q), cp.q); // folded table: r = conv * B^-1
            }
            out[(long)(o - a.out_shift) * N] = r;
          }
        }
      }
    }
    tc_fence_before();
    __syncthreads();
  }
  if (!ok && threadIdx.x == 0) {
    atomicOr(a.err, kErrWaitTimeout);
    // let copies and MMAs in flight finish (bounded) before the memory is released
    mbar_wait(&mbar[0], 0);
    if (in_flight) mbar_wait(&mbar[1], phase);
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTcCols));
}

static void run_convert(const Engine& E, const ConvArgs& a, int npolys, int j_begin, int j_end, cudaStream_t st) {
  const long N = E.N;
  if (N % kConvCoefs) throw AoaError(AOA_ERR_BAD_PARAM, "basis conversion: N too small");
  const size_t smem = (size_t)a.nin * kConvOut * sizeof(uint64_t);
  if (smem > 200 * 1024) throw AoaError(AOA_ERR_BAD_PARAM, "basis conversion: too many input limbs");
  dim3 grid(N / kConvCoefs, npolys);
  if (a.tc_b && E.tune.conv_tensor_cores && a.nin <= 32 && j_end <= 32 && N % kTcRows == 0) {
    ConvArgs t = a;
    t.err = E.d_err;
    t.spin = E.tune.spin_limit;
    t.npolys = npolys;
    const long tiles = (N / kTcRows) * npolys;
    const unsigned grid_tc = (unsigned)std::min<long>(tiles, E.num_sms);
    bool q1 = true;                               // every input and output prime q = 1 mod 2^32 below 2^60
    for (int i = 0; i < a.nin; i++) q1 = q1 && E.prime_kind[a.in_prime0 + i] == kButterflyLazyQ1;
    for (int j = 0; j < j_end; j++) q1 = q1 && E.prime_kind[a.out_prime0 + j] == kButterflyLazyQ1;
#define AOA_TC(M)                                                                                   \
  if (q1) basis_convert_tc<M, true><<<grid_tc, kTcThreads, kTcSmem, st>>>(t, j_begin, j_end);     \
  else basis_convert_tc<M, false><<<grid_tc, kTcThreads, kTcSmem, st>>>(t, j_begin, j_end);
    switch (a.mode) {
      case kRaw: AOA_TC(kRaw) break;
      case kModDown: AOA_TC(kModDown) break;
      case kRescaleTop: AOA_TC(kRescaleTop) break;
      case kRescaleY: AOA_TC(kRescaleY) break;
      default: AOA_TC(kRescaleFused) break;
    }
#undef AOA_TC
    note_launch();
    AOA_CHECK_LAUNCH();
    return;
  }
  for (int j0 = j_begin; j0 < j_end; j0 += kConvOut) {
    basis_convert<<<grid, kConvThreads, smem, st>>>(a, j0, j_end);
    note_launch();
  }
  AOA_CHECK_LAUNCH();
}

// Once per engine (per device): opt in to the dynamic shared memory the
// conversion kernel needs, and check the 128-bit accumulation bound.
void rns_init(Engine& E) {
  AOA_CUDA(cudaFuncSetAttribute(basis_convert, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
#define AOA_TC_SMEM(M)                                                                                       \
  AOA_CUDA(cudaFuncSetAttribute(basis_convert_tc<M, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTcSmem)); \
  AOA_CUDA(cudaFuncSetAttribute(basis_convert_tc<M, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTcSmem));
  AOA_TC_SMEM(kRaw) AOA_TC_SMEM(kModDown) AOA_TC_SMEM(kRescaleTop) AOA_TC_SMEM(kRescaleY) AOA_TC_SMEM(kRescaleFused)
#undef AOA_TC_SMEM
  auto bits = [](uint64_t x) { int b = 0; while (x) { b++; x >>= 1; } return b; };
  uint64_t mq = 0, mb = 0;
  for (int i = 0; i < E.k; i++) mq = std::max(mq, E.primes[i]);
  for (int j = 0; j < E.kl; j++) mb = std::max(mb, E.primes[E.k + j]);
  const int terms = std::max(E.k, E.kl);
  if (E.kl && bits(mq) + bits(mb) + bits((uint64_t)terms) > 128)
    throw AoaError(AOA_ERR_BAD_PARAM, "basis conversion: prime sizes overflow the 128-bit accumulator");
}

// ModUp: Q limbs 0..level of `in` (coefficient domain) -> kl B limbs of `out_b`.
void modup(const Engine& E, const uint64_t* in, long in_stride, uint64_t* out_b, long out_stride,
           int npolys, int level, cudaStream_t st) {
  if (E.kl == 0) return;
  if (level < 0 || level >= E.k) throw AoaError(AOA_ERR_BAD_PARAM, "modup: bad level");
  ConvArgs a{};
  a.in = in; a.out = out_b;
  a.in_poly_stride = in_stride; a.out_poly_stride = out_stride;
  a.nin = level + 1; a.mat_ld = E.kl;
  a.in_prime0 = 0; a.out_prime0 = E.k;
  a.zc = E.rns.modup_inv + (long)level * E.k;
  a.mat = E.rns.modup_hat + (long)level * E.k * E.kl;
  a.tc_b = E.rns.tc_modup ? E.rns.tc_modup + (size_t)level * kTcB : nullptr;
  a.pc = E.d_pc; a.log_n = E.log_n; a.mode = kRaw;
  run_convert(E, a, npolys, 0, E.kl, st);
}

static ConvArgs moddown_args(const Engine& E, const uint64_t* in_b, long in_stride, uint64_t* out, long out_stride) {
  ConvArgs a{};
  a.in = in_b; a.out = out;
  a.in_poly_stride = in_stride; a.out_poly_stride = out_stride;
  a.nin = E.kl; a.mat_ld = E.k;
  a.in_prime0 = E.k; a.out_prime0 = 0;
  a.zc = E.rns.moddown_inv;
  a.mat = E.rns.moddown_hat;
  a.tc_b = E.rns.tc_moddown;
  a.binv = E.rns.moddown_binv; a.pc = E.d_pc; a.log_n = E.log_n;
  return a;
}

// ModDown: `in` holds Q limbs 0..level at in_q and kl B limbs at in_b
// (coefficient domain) -> limbs 0..level of `out`.
void moddown(const Engine& E, const uint64_t* in_q, const uint64_t* in_b, long in_stride, uint64_t* out,
             long out_stride, int npolys, int level, cudaStream_t st) {
  if (level < 0 || level >= E.k) throw AoaError(AOA_ERR_BAD_PARAM, "moddown: bad level");
  ConvArgs a = moddown_args(E, in_b, in_stride, out, out_stride);
  a.x = in_q; a.x_poly_stride = in_stride; a.mode = kModDown;
  run_convert(E, a, npolys, 0, level + 1, st);
}

// conv_i (coefficient domain) of ModDown for outputs 0..nout-1, written to out.
void moddown_conv(const Engine& E, const uint64_t* in_b, long in_stride, uint64_t* out, long out_stride,
                  int npolys, int nout, cudaStream_t st) {
  ConvArgs a = moddown_args(E, in_b, in_stride, out, out_stride);
  a.mode = kRaw;
  run_convert(E, a, npolys, 0, nout, st);
}

// Merged ModDown + rescale corrections: given the key products' B limbs (in_b,
// coefficients) and u_l = limb l of (d + k B^-1) in coefficients, writes
// y_i = conv_i B^-1 + [c_l]_{q_i} for i < level, c_l = u_l - conv_l B^-1.
// One launch when level < 32, else c_l first (into cl_tmp) and then the y_i.
void rescale_corrections(const Engine& E, const uint64_t* in_b, long in_stride, const uint64_t* u_l,
                         long u_stride, uint64_t* cl_tmp, long cl_stride, uint64_t* y, long y_stride, int npolys,
                         int level, cudaStream_t st) {
  ConvArgs a = moddown_args(E, in_b, in_stride, y, y_stride);
  a.tc_b = E.rns.tc_moddown_binv;                // the tensor-core kernel's rescale modes fold B^-1 in
  if (level < kConvOut) {
    a.mode = kRescaleFused;
    a.d = u_l; a.d_poly_stride = u_stride;
    run_convert(E, a, npolys, 0, level + 1, st);
    return;
  }
  ConvArgs t = moddown_args(E, in_b, in_stride, cl_tmp, cl_stride);
  t.tc_b = E.rns.tc_moddown_binv;
  t.mode = kRescaleTop;
  t.d = u_l; t.d_poly_stride = u_stride;
  t.out_shift = level;
  run_convert(E, t, npolys, level, level + 1, st);
  a.mode = kRescaleY;
  a.d = cl_tmp; a.d_poly_stride = cl_stride;
  run_convert(E, a, npolys, 0, level, st);
}

// Rescale by q_level (ckks_rescale, manager.cu:90-118): for i < level,
// c_i <- (c_i - [c_level]_{q_i}) * q_level^-1 mod q_i, floor semantics, on
// npolys polys (stride poly_stride) in place, coefficient domain.
__global__ void rescale_kernel(uint64_t* d, long poly_stride, int level, const ShoupW* inv,
                               const PrimeConst* pc, int log_n) {
  const long N = 1L << log_n;
  const long c = (long)blockIdx.x * blockDim.x + threadIdx.x;
  const int i = blockIdx.y;
  uint64_t* p = d + blockIdx.z * poly_stride;
  const PrimeConst& P = pc[i];
  const uint64_t top = shoup(p[(long)level * N + c], 1, P.one_sh, P.q);   // [c_level]_{q_i}
  p[(long)i * N + c] = shoup(sub_mod(p[(long)i * N + c], top, P.q), inv[i], P.q);
}

void rescale(const Engine& E, uint64_t* d, long poly_stride, int npolys, int level, cudaStream_t st) {
  if (level < 1 || level >= E.k) throw AoaError(AOA_ERR_LEVEL_EXHAUSTED, "rescale: level must be >= 1");
  dim3 grid(E.N / 256, level, npolys);
  rescale_kernel<<<grid, 256, 0, st>>>(d, poly_stride, level, E.rns.resc_inv + (long)level * E.k, E.d_pc,
                                       E.log_n);
  note_launch();
  AOA_CHECK_LAUNCH();
}

// Transform-domain key-switch epilogue, limbs i < nlimbs of npolys polys:
//   rescale_level > 0: out_i = (base_i + k_i B^-1 - y_i) * q_l^-1   (merged ModDown + rescale)
//   else:              out_i = base_i + (k_i - y_i) * B^-1           (ModDown)
// base and y may be null (treated as 0); limb b of the launch is limb prime0 + b
// (prime prime0 + b).  Strides are per poly, in words.
// kCombPer coefficients per thread (the u-th at ((blockIdx.x kCombPer + u)
// blockDim + threadIdx), coalesced), so the per-limb constants and addresses
// serve several outputs.
constexpr int kCombPer = 4;

__device__ __forceinline__ uint64_t ks_combine_one(uint64_t bv, uint64_t kv, uint64_t yv, ShoupW binv,
                                                   const ShoupW* resc, ShoupW rs, uint64_t q) {
  if (resc) return shoup(sub_mod(add_mod(bv, shoup(kv, binv, q), q), yv, q), rs, q);
  return add_mod(bv, shoup(sub_mod(kv, yv, q), binv, q), q);
}

__global__ void ks_combine_kernel(uint64_t* out, long out_stride, const uint64_t* base, long base_stride,
                                  const uint64_t* k, long k_stride, const uint64_t* y, long y_stride,
                                  const ShoupW* binv, const ShoupW* resc, const PrimeConst* pc, int prime0,
                                  int log_n) {
  const long N = 1L << log_n;
  const int i = prime0 + blockIdx.y, p = blockIdx.z;
  const long limb = (long)blockIdx.y * N;
  const uint64_t q = pc[i].q;
  const ShoupW bi = binv[i], rs = resc ? resc[i] : ShoupW{0, 0};
  const uint64_t* kp = k + p * k_stride + limb;
  const uint64_t* yp = y ? y + p * y_stride + limb : nullptr;
  const uint64_t* bp = base ? base + p * base_stride + limb : nullptr;
  uint64_t* op = out + p * out_stride + limb;
  uint64_t kv[kCombPer], yv[kCombPer], bv[kCombPer];
#pragma unroll
  for (int u = 0; u < kCombPer; u++) {
    const long c = ((long)blockIdx.x * kCombPer + u) * blockDim.x + threadIdx.x;
    kv[u] = kp[c];
    yv[u] = yp ? yp[c] : 0;
    bv[u] = bp ? bp[c] : 0;
  }
#pragma unroll
  for (int u = 0; u < kCombPer; u++) {
    const long c = ((long)blockIdx.x * kCombPer + u) * blockDim.x + threadIdx.x;
    op[c] = ks_combine_one(bv[u], kv[u], yv[u], bi, resc, rs, q);
  }
}

// Same epilogue writing poly p to outp.p[p] (a list of output polys).
__global__ void ks_combine_ptr_kernel(OutPtrs outp, const uint64_t* base, long base_stride, int base_polys,
                                      const uint64_t* k, long k_stride, const uint64_t* y, long y_stride,
                                      const ShoupW* binv, const ShoupW* resc, const PrimeConst* pc, int log_n) {
  const long N = 1L << log_n;
  const int i = blockIdx.y, p = blockIdx.z;
  const long limb = (long)i * N;
  const uint64_t q = pc[i].q;
  const ShoupW bi = binv[i], rs = resc ? resc[i] : ShoupW{0, 0};
  const uint64_t* kp = k + p * k_stride + limb;
  const uint64_t* yp = y + p * y_stride + limb;
  const uint64_t* bp = base && p < base_polys ? base + p * base_stride + limb : nullptr;
  uint64_t* op = outp.p[p] + limb;
  uint64_t kv[kCombPer], yv[kCombPer], bv[kCombPer];
#pragma unroll
  for (int u = 0; u < kCombPer; u++) {
    const long c = ((long)blockIdx.x * kCombPer + u) * blockDim.x + threadIdx.x;
    kv[u] = kp[c];
    yv[u] = yp[c];
    bv[u] = bp ? bp[c] : 0;
  }
#pragma unroll
  for (int u = 0; u < kCombPer; u++) {
    const long c = ((long)blockIdx.x * kCombPer + u) * blockDim.x + threadIdx.x;
    op[c] = ks_combine_one(bv[u], kv[u], yv[u], bi, resc, rs, q);
  }
}

void ks_combine_ptr(const Engine& E, const OutPtrs& outp, const uint64_t* base, long base_stride, const uint64_t* k,
                    long k_stride, const uint64_t* y, long y_stride, int nlimbs, int npolys, int rescale_level,
                    cudaStream_t st, int base_polys) {
  if (nlimbs <= 0) return;
  dim3 grid(E.N / (256 * kCombPer), nlimbs, npolys);
  const ShoupW* resc = rescale_level > 0 ? E.rns.resc_inv + (long)rescale_level * E.k : nullptr;
  ks_combine_ptr_kernel<<<grid, 256, 0, st>>>(outp, base, base_stride, base_polys < 0 ? npolys : base_polys, k,
                                              k_stride, y, y_stride, E.rns.moddown_binv, resc, E.d_pc, E.log_n);
  note_launch();
  AOA_CHECK_LAUNCH();
}

void ks_combine(const Engine& E, uint64_t* out, long out_stride, const uint64_t* base, long base_stride,
                const uint64_t* k, long k_stride, const uint64_t* y, long y_stride, int nlimbs, int npolys,
                int rescale_level, cudaStream_t st, int prime0) {
  if (nlimbs <= 0) return;
  dim3 grid(E.N / (256 * kCombPer), nlimbs, npolys);
  const ShoupW* resc = rescale_level > 0 ? E.rns.resc_inv + (long)rescale_level * E.k : nullptr;
  ks_combine_kernel<<<grid, 256, 0, st>>>(out, out_stride, base, base_stride, k, k_stride, y, y_stride,
                                          E.rns.moddown_binv, resc, E.d_pc, prime0, E.log_n);
  note_launch();
  AOA_CHECK_LAUNCH();
}

}  // namespace aoa
