// Negacyclic NTT / INTT over 64-bit RNS limbs, sm_100a.
//
// Transform contract (bit-exact with the reference): for a limb x under prime q
// with psi = g^((q-1)/2N), g the prime's smallest primitive root, the forward
// transform leaves at position p the value x(psi^(2*bitrev_N(p)+1)) — the order
// produced by the reference's hierarchical hntt_tr<Nb>/hntt_tr<Na> pair
// (aoa-ntt src/cuda/htrans/ntt.cu:35-50, 321-363; tables ntt.cu:685-1023,
// common.cu:314-357).  The inverse is its exact inverse (hintt/hintt_tr,
// ntt.cu:51-65, 373-460).
//
// Algorithm (not the reference's): the merged negacyclic Cooley-Tukey NTT
// (twist folded into bit-reversed psi powers, no separate twist pass) and its
// Gentleman-Sande inverse with N^-1 folded into the last stage.  The N-point
// limb is viewed as an R x C row-major matrix; the forward runs the high
// log2(R) stages as R-point transforms down the columns (column pass), then
// the low log2(C) stages along contiguous rows (row pass); the inverse runs the
// row pass first.  Each pass is one kernel: a thread holds 2^ceil(s/2)
// elements of an S = 2^s point sub-transform, does the high-digit stages in
// registers, exchanges once through (swizzled) shared memory and does the
// low-digit stages in registers.  Global loads and stores are coalesced in both
// passes.  Passes run in place; the host launches them over chunks of whole
// polys of at most the engine's chunk size (default 1 GiB: the passes are bound
// by integer arithmetic, so fewer launch tails pay more than keeping the
// column-pass output in L2 for the row pass).
#include <cuda.h>   // CUtensorMap and its enums (types only; the encoder is fetched through the runtime)

#include "aoa_internal.h"
#include "async.cuh"

namespace aoa {

template <int LOG_S>
struct Sub {
  static constexpr int S = 1 << LOG_S;
  static constexpr int HI = (LOG_S + 1) / 2;   // high digit width (first exchange half)
  static constexpr int LO = LOG_S / 2;         // low digit width (second exchange half)
  static constexpr int T = 1 << LO;            // threads per sub-transform
  static constexpr int E = 1 << HI;            // elements per thread
  static constexpr int G = 1 << (HI - LO);     // low-digit groups per thread (1 or 2)
  static constexpr int L = 1 << LO;            // elements per low-digit group
  // sub-transforms per CTA: <= 256 threads, <= 32 KiB shared memory, <= 32
  static constexpr int PER_CTA_A = 256 / T < 4096 / S ? 256 / T : 4096 / S;
  static constexpr int PER_CTA = PER_CTA_A < 32 ? PER_CTA_A : 32;
};

// ---- butterflies ------------------------------------------------------------
// The canonical kind keeps every value in [0, q) (any q < 2^63); the lazy
// kinds (primes < 2^60) let values grow between reductions (Harvey's lazy
// butterflies; bounds below), kButterflyLazyQ1 with the shorter Shoup
// remainder of primes q = 1 mod 2^32.  The last stage of each transform
// reduces to [0, q).

template <int KIND>
struct Bf;

template <>
struct Bf<kButterflyCanonical> {
  static __device__ __forceinline__ void ct(uint64_t& x, uint64_t& y, ShoupW w, uint64_t q, bool) {
    uint64_t U = x, V = shoup(y, w, q);
    x = add_mod(U, V, q);
    y = sub_mod(U, V, q);
  }
  static __device__ __forceinline__ void gs(uint64_t& x, uint64_t& y, ShoupW w, uint64_t q) {
    uint64_t U = x, V = y;
    x = add_mod(U, V, q);
    y = shoup(sub_mod(U, V, q), w, q);
  }
  // final inverse stage with N^-1 folded in
  static __device__ __forceinline__ void gs_last(uint64_t& x, uint64_t& y, ShoupW n0, ShoupW n1, uint64_t q) {
    uint64_t U = x, V = y;
    x = shoup(add_mod(U, V, q), n0, q);
    y = shoup(sub_mod(U, V, q), n1, q);
  }
  static __device__ __forceinline__ uint64_t fwd_out(uint64_t x, uint64_t) { return x; }
};

// Lazy butterflies (every prime below 2^60).  The Shoup products take their
// quotient from the three high 32 x 32-bit partial products
// (shoup_lazy_mad3): one wide multiply fewer than the exact quotient on the
// integer multiply pipe, which bounds these kernels, for products in [0, 4q)
// instead of [0, 2q) (measured 1255 -> 1412 GB/s for the forward transform of
// 256 x 30 limbs at 2^16; the exact quotient written the same way measured
// no faster than the compiler's lowering).  Forward values stay below 16q
// (< 2^64): a reducing stage (even stage index within its pass) maps [0, 16q)
// to [0, 12q) (U reduced by 8q), the stage after it maps [0, 12q) to
// [0, 16q).  Inverse values stay in [0, 4q), reduced at every stage.
template <int KIND>
struct Bf {
  static __device__ __forceinline__ uint64_t mulw(uint64_t y, ShoupW w, uint64_t q) {   // [0, 4q)
    if constexpr (KIND == kButterflyLazyQ1) return shoup_lazy_mad3_q1(y, w.w, w.wp, q);
    else return shoup_lazy_mad3(y, w.w, w.wp, 0 - q);
  }
  // x - b if x >= b else x, for x < 2^63 + b, b < 2^63 (sign of the difference)
  static __device__ __forceinline__ uint64_t csub(uint64_t x, uint64_t b) {
    const int64_t d = (int64_t)(x - b);
    return d < 0 ? x : (uint64_t)d;
  }
  // red (a compile-time constant after unrolling): reducing stage
  static __device__ __forceinline__ void ct(uint64_t& x, uint64_t& y, ShoupW w, uint64_t q, bool red) {
    const uint64_t q4 = q << 2;
    uint64_t U = x;                             // [0, 16q) if red, else [0, 12q)
    if (red) U = csub(U, q << 3);               // [0, 8q)
    const uint64_t V = mulw(y, w, q);           // [0, 4q)
    x = U + V;                                  // [0, 12q) if red, else [0, 16q)
    y = U - V + q4;                             // likewise
  }
  // inputs and outputs in [0, 4q)
  static __device__ __forceinline__ void gs(uint64_t& x, uint64_t& y, ShoupW w, uint64_t q) {
    const uint64_t q4 = q << 2;
    const uint64_t U = x, V = y;
    x = csub(U + V, q4);
    y = mulw(U - V + q4, w, q);
  }
  // final inverse stage with N^-1 folded in: outputs in [0, q)
  static __device__ __forceinline__ void gs_last(uint64_t& x, uint64_t& y, ShoupW n0, ShoupW n1, uint64_t q) {
    const uint64_t U = x, V = y;
    const uint64_t a = mulw(U + V, n0, q);
    const uint64_t b = mulw(U - V + (q << 2), n1, q);
    x = csub(csub(a, q << 1), q);
    y = csub(csub(b, q << 1), q);
  }
  static __device__ __forceinline__ uint64_t fwd_out(uint64_t x, uint64_t q) {   // [0, 16q) -> [0, q)
    x = csub(x, q << 3);
    x = csub(x, q << 2);
    x = csub(x, q << 1);
    return csub(x, q);
  }
};

// ---- explicit shared-memory accessors --------------------------------------------
// (ld.shared / st.shared: keeps every on-chip access on the short-latency path)


__device__ __forceinline__ uint64_t lds64(uint32_t a) {
  uint64_t v;
  asm volatile("ld.shared.u64 %0, [%1];" : "=l"(v) : "r"(a));
  return v;
}
__device__ __forceinline__ void sts64(uint32_t a, uint64_t v) {
  asm volatile("st.shared.u64 [%0], %1;" ::"r"(a), "l"(v));
}
__device__ __forceinline__ ShoupW ldsw(uint32_t a) {
  ShoupW w;
  asm volatile("ld.shared.v2.u64 {%0, %1}, [%2];" : "=l"(w.w), "=l"(w.wp) : "r"(a));
  return w;
}

// ---- forward (Cooley-Tukey, merged twist) ---------------------------------
// twiddle index for local half-span 2^j and local group g: K * S/2^(j+1) + g;
// here K = 1 and the twiddles 0..S-1 of the prime sit in shared memory at tw.

template <int LOG_S, int LAZY>
__device__ __forceinline__ void fwd_high_s(uint64_t (&v)[Sub<LOG_S>::E], uint32_t tw, uint64_t q) {
  using D = Sub<LOG_S>;
#pragma unroll
  for (int i = D::HI - 1; i >= 0; i--) {
    const int span = 1 << i;
#pragma unroll
    for (int h = 0; h < D::E; h++) {
      if (h & span) continue;
      const ShoupW w = ldsw(tw + 16 * ((1 << (D::HI - 1 - i)) + (h >> (i + 1))));
      Bf<LAZY>::ct(v[h], v[h + span], w, q, ((D::HI - 1 - i) & 1) == 0);
    }
  }
}

// Low-digit twiddle of level lvl = LOG_S - 1 - i for digit hi and group s:
// natural table order 2^lvl + hi 2^(lvl - HI) + s, or, with PERM, the order
// 2^lvl + s 2^HI + hi, in which the lanes of one s read consecutive entries
// (conflict-free when a warp's lanes hold different hi).
template <int LOG_S, bool PERM>
__device__ __forceinline__ int low_tw_index(int i, uint32_t hi, int s) {
  using D = Sub<LOG_S>;
  return PERM ? (1 << (LOG_S - 1 - i)) + (s << D::HI) + (int)hi
              : (1 << (LOG_S - 1 - i)) + ((int)hi << (D::LO - 1 - i)) + s;
}

// position of natural twiddle entry e in the PERM order
template <int LOG_S>
__device__ __forceinline__ int low_tw_perm(int e) {
  using D = Sub<LOG_S>;
  if (e < (1 << D::HI)) return e;
  const int lvl = 31 - __clz(e), sh = lvl - D::HI, off = e - (1 << lvl);
  return (1 << lvl) + ((off & ((1 << sh) - 1)) << D::HI) + (off >> sh);
}

template <int LOG_S, int LAZY, bool PERM = false>
__device__ __forceinline__ void fwd_low_s(uint64_t (&u)[Sub<LOG_S>::L], uint32_t tw, uint32_t hi, uint64_t q) {
  using D = Sub<LOG_S>;
#pragma unroll
  for (int i = D::LO - 1; i >= 0; i--) {
    const int span = 1 << i;
#pragma unroll
    for (int l = 0; l < D::L; l++) {
      if (l & span) continue;
      const ShoupW w = ldsw(tw + 16 * low_tw_index<LOG_S, PERM>(i, hi, l >> (i + 1)));
      Bf<LAZY>::ct(u[l], u[l + span], w, q, ((D::HI + D::LO - 1 - i) & 1) == 0);
    }
  }
}

// ---- inverse (Gentleman-Sande) -------------------------------------------

template <int LOG_S, int LAZY, bool PERM = false>
__device__ __forceinline__ void inv_low_s(uint64_t (&u)[Sub<LOG_S>::L], uint32_t itw, uint32_t hi, uint64_t q) {
  using D = Sub<LOG_S>;
#pragma unroll
  for (int i = 0; i < D::LO; i++) {
    const int span = 1 << i;
#pragma unroll
    for (int l = 0; l < D::L; l++) {
      if (l & span) continue;
      const ShoupW w = ldsw(itw + 16 * low_tw_index<LOG_S, PERM>(i, hi, l >> (i + 1)));
      Bf<LAZY>::gs(u[l], u[l + span], w, q);
    }
  }
}

// the column pass's high digit holds the transform's final stage (half-span
// N/2): scale by N^-1 there
template <int LOG_S, int LAZY>
__device__ __forceinline__ void inv_high_s(uint64_t (&v)[Sub<LOG_S>::E], uint32_t itw, uint64_t q, ShoupW ninv,
                                           ShoupW ninv_w1) {
  using D = Sub<LOG_S>;
#pragma unroll
  for (int i = 0; i < D::HI; i++) {
    const int span = 1 << i;
#pragma unroll
    for (int h = 0; h < D::E; h++) {
      if (h & span) continue;
      if (i == D::HI - 1) {
        Bf<LAZY>::gs_last(v[h], v[h + span], ninv, ninv_w1, q);
      } else {
        const ShoupW w = ldsw(itw + 16 * ((1 << (D::HI - 1 - i)) + (h >> (i + 1))));
        Bf<LAZY>::gs(v[h], v[h + span], w, q);
      }
    }
  }
}

// ---- row-pass twiddles ---------------------------------------------------------
// High digit: per row, at row_tw[2^(HI-1-i) - 1 + g] (shared memory).
// Low digit: per thread in registers, list order j = 2^(LO-1-i) - 1 + g.

template <int LOG_S>
__device__ __forceinline__ void load_low_tw(ShoupW (&w)[Sub<LOG_S>::G][Sub<LOG_S>::L - 1],
                                            const ShoupW* __restrict__ tw, uint32_t K, int t) {
  using D = Sub<LOG_S>;
#pragma unroll
  for (int gg = 0; gg < D::G; gg++) {
    const uint32_t hi = t * D::G + gg;
#pragma unroll
    for (int j = 0; j < D::L - 1; j++) {
      const int lvl = 31 - __clz(j + 1);       // entry j: stage with 2^lvl twiddles, group g
      const int g = j + 1 - (1 << lvl);
      w[gg][j] = tw[(K << (LOG_S - D::LO + lvl)) + (hi << lvl) + g];
    }
  }
}

template <int LOG_S, int LAZY>
__device__ __forceinline__ void fwd_low_r(uint64_t (&u)[Sub<LOG_S>::L], const ShoupW (&w)[Sub<LOG_S>::L - 1],
                                          uint64_t q) {
  using D = Sub<LOG_S>;
#pragma unroll
  for (int i = D::LO - 1; i >= 0; i--) {
    const int span = 1 << i;
#pragma unroll
    for (int l = 0; l < D::L; l++) {
      if (l & span) continue;
      Bf<LAZY>::ct(u[l], u[l + span], w[(1 << (D::LO - 1 - i)) - 1 + (l >> (i + 1))], q,
                   ((D::HI + D::LO - 1 - i) & 1) == 0);
    }
  }
}

template <int LOG_S, int LAZY>
__device__ __forceinline__ void inv_low_r(uint64_t (&u)[Sub<LOG_S>::L], const ShoupW (&w)[Sub<LOG_S>::L - 1],
                                          uint64_t q) {
  using D = Sub<LOG_S>;
#pragma unroll
  for (int i = 0; i < D::LO; i++) {
    const int span = 1 << i;
#pragma unroll
    for (int l = 0; l < D::L; l++) {
      if (l & span) continue;
      Bf<LAZY>::gs(u[l], u[l + span], w[(1 << (D::LO - 1 - i)) - 1 + (l >> (i + 1))], q);
    }
  }
}

// ---- fused epilogue of a forward transform ----------------------------------------
__device__ __forceinline__ void epi_store(const NttEpi& e, long N, long p, int limb, int prime, long c, uint64_t v,
                                          const PrimeConst& P) {
  const long off = (long)(limb + e.limb_base) * N + c;
  if (e.mode == kEpiKeyProduct) {
    const uint64_t kb = e.key[(long)prime * N + c], ka = e.key[e.key_half + (long)prime * N + c];
    uint64_t* o = e.out + p * e.out_stride + off;
    o[0] = mul_mod(v, kb, P);
    o[e.out_poly1] = mul_mod(v, ka, P);
  } else {
    const uint64_t q = P.q;
    const uint64_t kv = e.ks[p * e.ks_stride + off];
    const uint64_t bv = p < e.base_polys ? e.base[p * e.base_stride + off] : 0;
    uint64_t r;
    if (e.resc) r = shoup(sub_mod(add_mod(bv, shoup(kv, e.binv[prime], q), q), v, q), e.resc[prime], q);
    else r = add_mod(bv, shoup(sub_mod(kv, v, q), e.binv[prime], q), q);
    uint64_t* o = e.use_ptrs ? e.outp.p[p] : e.out + p * e.out_stride;
    o[off] = r;
  }
}

// the same epilogue as a separate pass over transformed data (small rings)
__global__ void ntt_epilogue_kernel(const uint64_t* data, long poly_stride, int npolys, int nlimbs, int first_prime,
                                    int prime_shift, const PrimeConst* pc, int log_n, const __grid_constant__ NttEpi e) {
  const long N = 1L << log_n;
  const long total = (long)npolys * nlimbs * N;
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (long)gridDim.x * blockDim.x) {
    const long c = i % N;
    const int limb = (int)((i / N) % nlimbs);
    const long p = i / N / nlimbs;
    const int prime = first_prime + (limb >> prime_shift);
    epi_store(e, N, p, limb, prime, c, data[(p * poly_stride + limb) * N + c], pc[prime]);
  }
}

// ---- kernels ---------------------------------------------------------------
// Work items: limb l of poly p (item j = l * npolys + p) lives at
// data + (p * poly_stride + l) * N under prime first_prime + l.  grid =
// (tiles per limb, G): CTA (x, y) handles tile x of the contiguous item range
// [y * nitems / G, (y + 1) * nitems / G) — consecutive polys of one limb share
// their twiddles, which are reloaded only when the limb changes — and streams
// the items through two shared-memory buffers filled by bulk copies, so the
// next item's tile arrives while the current one is transformed.

struct NttBatch {
  uint64_t* data;
  const ShoupW* tw;        // [nprimes][N] forward twiddles (psi^bitrev)
  const ShoupW* itw;       // [nprimes][N] inverse twiddles
  const PrimeConst* pc;    // [nprimes]
  unsigned* err;           // device error word
  int log_n, log_r, log_c; // N = R * C
  int first_prime;
  int prime_shift;         // limb l uses prime first_prime + (l >> prime_shift)
  long poly_stride;        // limbs between consecutive polys
  int npolys, nitems;      // nitems = nlimbs * npolys
  const uint64_t* src;     // this pass loads from src (out of place) when set
  long src_poly_stride;
  int poly_base;           // poly index of the launch's first poly within the call
  int spin;                // polls of a bounded wait for this kernel's own copies (engine knob)
  int use_tma;             // column pass: tiles by one tensor-map load (the kernel's tmap argument)
};

// Threads per SM the pass kernels are compiled for (register budget).
#ifndef AOA_COLS_TPSM
#define AOA_COLS_TPSM 768
#endif
#ifndef AOA_ROWS_TPSM
#define AOA_ROWS_TPSM 384
#endif

// Tile widths: a column-pass CTA takes W = PER_CTA >> DIV columns (at least 2,
// so that a row segment is a multiple of 16 bytes), a row-pass CTA takes
// PER_CTA >> DIV rows (at least 1).  DIV is a tuning choice (0, 1, 2).
template <int LOG_S, int DIV>
struct ColTile {
  static constexpr int W0 = Sub<LOG_S>::PER_CTA >> DIV;
  static constexpr int W = W0 < 2 ? 2 : W0;
  static constexpr int THREADS = Sub<LOG_S>::T * W;
  static constexpr int MIN_BLOCKS = AOA_COLS_TPSM / THREADS < 1 ? 1 : (AOA_COLS_TPSM / THREADS > 32 ? 32 : AOA_COLS_TPSM / THREADS);
  static constexpr size_t SMEM = 2 * (size_t)Sub<LOG_S>::S * W * 8 + 2 * (size_t)Sub<LOG_S>::S * sizeof(ShoupW);
};

template <int LOG_S, int DIV>
struct RowTile {
  static constexpr int R0 = Sub<LOG_S>::PER_CTA >> DIV;
  static constexpr int ROWS = R0 < 1 ? 1 : R0;
  static constexpr int THREADS = Sub<LOG_S>::T * ROWS;
  // 384 threads per SM: up to 170 registers, so the low-digit twiddles held in
  // registers do not spill (measured 1% faster than 512 threads with spills)
  static constexpr int MIN_BLOCKS = AOA_ROWS_TPSM / THREADS < 1 ? 1 : (AOA_ROWS_TPSM / THREADS > 32 ? 32 : AOA_ROWS_TPSM / THREADS);
  static constexpr size_t SMEM =
      2 * (size_t)ROWS * Sub<LOG_S>::S * 8 + 2 * (size_t)ROWS * (Sub<LOG_S>::E - 1) * sizeof(ShoupW);
};

// Column pass.  Tile = S rows x W columns of one limb; its load is S bulk copies
// of W*8 bytes (one per row) issued by warp 0.  Shared layout [S][W].  Two
// CTA barriers per item: the first (after the tile's mbarrier) also marks
// that every thread has finished the previous item, so the next tile's copy
// into that item's buffer is issued right after it; the second is the
// exchange between the two digit rounds.  The prime's twiddles alternate
// between two buffers, so a new limb's twiddles can be written before the
// first barrier: the buffer's previous users finished at least one item
// earlier.
template <int LOG_R, int DIV, int LAZY, bool FWD>
__global__ void __launch_bounds__(ColTile<LOG_R, DIV>::THREADS, ColTile<LOG_R, DIV>::MIN_BLOCKS)
ntt_cols(NttBatch b, const __grid_constant__ CUtensorMap tmap) {
  using D = Sub<LOG_R>;
  constexpr int W = ColTile<LOG_R, DIV>::W;
  constexpr int TILE = D::S * W;
  // Row r of the tile sits at shared row sigma(r) = r ^ ((r >> (LO + G - 1)) & M):
  // the low-digit accesses (rows (t G + g) 2^LO + l, threads t of one warp)
  // then spread over the 128-byte bank line instead of hitting one W-word
  // slice of it, while the high-digit accesses stay contiguous.
  constexpr int LINE_ROWS = W >= 16 ? 1 : 16 / W;
  constexpr int M = (LINE_ROWS < D::T ? LINE_ROWS : D::T) - 1;
  auto sig = [](int r) { return r ^ ((r >> (D::LO + D::G - 1)) & M); };
  extern __shared__ __align__(128) uint64_t dyn[];
  __shared__ __align__(8) uint64_t mbar[2];
  const uint32_t sbuf = smem_u32(dyn);                          // [2][S][W] words
  ShoupW* tws = (ShoupW*)(dyn + 2 * TILE);                      // [2][S] ShoupW
  const int w = threadIdx.x % W, t = threadIdx.x / W;
  const long N = 1L << b.log_n, C = 1L << b.log_c;
  const int G = gridDim.y;
  if (threadIdx.x == 0) {
    mbar_init(&mbar[0], 1);
    mbar_init(&mbar[1], 1);
    mbar_init_fence();
  }
  __syncthreads();
  auto src_of = [&](int j) -> const uint64_t* {
    const int limb = j / b.npolys, p = j % b.npolys;
    if (b.src) return b.src + ((long)p * b.src_poly_stride + limb) * N + (long)blockIdx.x * W;
    return b.data + ((long)p * b.poly_stride + limb) * N + (long)blockIdx.x * W;
  };
  auto dst_of = [&](int j) -> uint64_t* {
    const int limb = j / b.npolys, p = j % b.npolys;
    return b.data + ((long)p * b.poly_stride + limb) * N + (long)blockIdx.x * W;
  };
  // S row segments of W words, spread over all threads (one each when
  // S = blockDim), so no warp lags behind the others into the next barrier;
  // a copy may complete before thread 0's expect_tx (the transaction count
  // may go below zero until then)
  auto issue = [&](int j, int bi) {
    if (b.use_tma) {                     // one tensor-map load of the S x W tile (rows in order: M == 0)
      if (threadIdx.x == 0) {
        mbar_expect_tx(&mbar[bi], TILE * 8);
        tma_load_4d(sbuf + bi * TILE * 8, &tmap, (int)blockIdx.x * W, 0, j / b.npolys, j % b.npolys, &mbar[bi]);
      }
      return;
    }
    if (threadIdx.x == 0) mbar_expect_tx(&mbar[bi], TILE * 8);
    const uint64_t* src = src_of(j);
    for (int r = threadIdx.x; r < D::S; r += blockDim.x)
      bulk_g2s(sbuf + (bi * TILE + sig(r) * W) * 8, src + r * C, W * 8, &mbar[bi]);
  };
  int cur_limb = -1, tb = 1;
  const int j_lo = (int)((long)blockIdx.y * b.nitems / G), j_hi = (int)((long)(blockIdx.y + 1) * b.nitems / G);
  if (j_lo < j_hi) issue(j_lo, 0);
  for (int j = j_lo, it = 0; j < j_hi; j++, it++) {
    const int bi = it & 1;
    const int limb = j / b.npolys, prime = b.first_prime + (limb >> b.prime_shift);
    if (limb != cur_limb) {                // the other buffer's users are at least one item behind
      tb ^= 1;
      const ShoupW* tw = (FWD ? b.tw : b.itw) + (long)prime * N;
      for (int e = threadIdx.x; e < D::S; e += blockDim.x) tws[tb * D::S + e] = tw[e];
      cur_limb = limb;
    }
    const bool ok = mbar_wait(&mbar[bi], (it >> 1) & 1, b.spin);
    if (__syncthreads_or(!ok)) {
      if (threadIdx.x == 0) {
        atomicOr(b.err, kErrWaitTimeout);
        mbar_wait(&mbar[bi], (it >> 1) & 1);   // the copy in flight: give it one more bounded wait
      }
      return;
    }
    // every thread is past item j - 1: its buffer takes the next tile
    if (j + 1 < j_hi) issue(j + 1, bi ^ 1);
    const uint32_t stw = smem_u32(tws + tb * D::S);
    const PrimeConst& P = b.pc[prime];
    const uint64_t q = P.q;
    const uint32_t sm = sbuf + bi * TILE * 8 + w * 8;            // + row * W * 8
    uint64_t* x = dst_of(j) + w;
    if (FWD) {
      uint64_t v[D::E];
#pragma unroll
      for (int h = 0; h < D::E; h++) v[h] = lds64(sm + sig((h << D::LO) + t) * W * 8);
      fwd_high_s<LOG_R, LAZY>(v, stw, q);
#pragma unroll
      for (int h = 0; h < D::E; h++) sts64(sm + sig((h << D::LO) + t) * W * 8, v[h]);
      __syncthreads();
#pragma unroll
      for (int g = 0; g < D::G; g++) {
        const int hi = t * D::G + g;
        uint64_t u[D::L];
#pragma unroll
        for (int l = 0; l < D::L; l++) u[l] = lds64(sm + sig((hi << D::LO) + l) * W * 8);
        fwd_low_s<LOG_R, LAZY>(u, stw, hi, q);
#pragma unroll
        for (int l = 0; l < D::L; l++) x[(long)((hi << D::LO) + l) * C] = u[l];
      }
    } else {
      const ShoupW ninv{P.ninv, P.ninv_sh}, ninv_w1{P.ninv_w1, P.ninv_w1_sh};
#pragma unroll
      for (int g = 0; g < D::G; g++) {
        const int hi = t * D::G + g;
        uint64_t u[D::L];
#pragma unroll
        for (int l = 0; l < D::L; l++) u[l] = lds64(sm + sig((hi << D::LO) + l) * W * 8);
        inv_low_s<LOG_R, LAZY>(u, stw, hi, q);
#pragma unroll
        for (int l = 0; l < D::L; l++) sts64(sm + sig((hi << D::LO) + l) * W * 8, u[l]);
      }
      __syncthreads();
      uint64_t v[D::E];
#pragma unroll
      for (int h = 0; h < D::E; h++) v[h] = lds64(sm + sig((h << D::LO) + t) * W * 8);
      inv_high_s<LOG_R, LAZY>(v, stw, q, ninv, ninv_w1);
#pragma unroll
      for (int h = 0; h < D::E; h++) x[(long)((h << D::LO) + t) * C] = v[h];
    }
    // generic-proxy accesses of buffer bi end here; the next bulk copy into it
    // (issued after the next item's first barrier) is an async-proxy write
    fence_proxy_async();
  }
}

// ---- column pass with warp-owned columns ----------------------------------------
// The same column transforms as ntt_cols, with every column's T threads in
// one warp (a warp holds 32 / T whole columns), so the exchange between the
// two digit rounds needs only the warp: no CTA barrier inside an item.  A
// producer warp streams the tiles (and the prime's twiddles when they change,
// entry by entry into the order low_tw_perm gives, so that the lanes of a
// warp, which hold different low digits, read consecutive twiddles) into two
// buffers through full / empty mbarrier pairs; compute warps wait only for
// their buffer.  Row r of a tile sits at word
//   P(r) = (W + 2) r + CW (k mod M) + 16 (k div M),  k = r >> (LO + G - 1),
// M = 16 / CW: rows start 16-byte aligned and, for both digit access patterns
// (rows (h << LO) + t and ((t G + g) << LO) + l over a warp's T lanes and CW
// columns), the warp's 32 words fall twice on each 8-byte bank slot, so every
// shared-memory access is conflict-free.
template <int LOG_R, int NW>
struct WoTile {
  using D = Sub<LOG_R>;
  static constexpr int CW = 32 / D::T;           // whole columns per warp
  static constexpr int W = NW * CW;              // columns per tile
  static constexpr int RS = W + 2;
  static constexpr int M = 16 / CW;
  static constexpr int SH = D::LO + D::G - 1;
  static constexpr __host__ __device__ int row(int r) {
    return RS * r + CW * ((r >> SH) % M) + 16 * ((r >> SH) / M);
  }
  static constexpr int WORDS = ((row(D::S - 1) + W + 15) / 16) * 16;   // one buffer, 128-byte multiple
  static constexpr int THREADS = (NW + 1) * 32;
  static constexpr size_t SMEM = 2 * (size_t)WORDS * 8 + 2 * (size_t)D::S * sizeof(ShoupW);
  static constexpr int BY_SMEM = (int)((232448 - 1024) / (SMEM + 1024));
  static constexpr int MIN_BLOCKS = BY_SMEM < 1 ? 1 : (BY_SMEM > 16 ? 16 : BY_SMEM);
};

template <int LOG_R, int NW, bool FWD>
__global__ void __launch_bounds__(WoTile<LOG_R, NW>::THREADS, WoTile<LOG_R, NW>::MIN_BLOCKS)
ntt_cols_wo(NttBatch b) {
  using D = Sub<LOG_R>;
  using Tl = WoTile<LOG_R, NW>;
  constexpr int W = Tl::W, CW = Tl::CW, WORDS = Tl::WORDS;
  extern __shared__ __align__(128) uint64_t dyn[];
  __shared__ __align__(8) uint64_t full[2], empty[2];
  const uint32_t sbuf = smem_u32(dyn);                       // [2][WORDS] words
  ShoupW* tws = (ShoupW*)(dyn + 2 * WORDS);                   // [2][S]
  const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
  const long N = 1L << b.log_n, C = 1L << b.log_c;
  const int G = gridDim.y;
  if (threadIdx.x == 0) {
    mbar_init(&full[0], 1);
    mbar_init(&full[1], 1);
    mbar_init(&empty[0], NW);
    mbar_init(&empty[1], NW);
    mbar_init_fence();
  }
  __syncthreads();
  const int j_lo = (int)((long)blockIdx.y * b.nitems / G), j_hi = (int)((long)(blockIdx.y + 1) * b.nitems / G);
  auto prime_of = [&](int j) { return b.first_prime + ((j / b.npolys) >> b.prime_shift); };
  if (warp == NW) {
    // producer: tile rows of W words (one bulk copy each) and, when the prime
    // of the buffer changes, its S twiddles
    int prime_in0 = -1, prime_in1 = -1;      // prime whose twiddles each buffer holds
    int issued = 0;
    bool ok = true;
    for (int j = j_lo, it = 0; j < j_hi; j++, it++) {
      const int bi = it & 1;
      if (it >= 2 && !mbar_wait(&empty[bi], ((it - 2) >> 1) & 1, b.spin)) {
        ok = false;
        break;
      }
      const int limb = j / b.npolys, p = j % b.npolys;
      const int prime = prime_of(j);
      const bool new_tw = (bi ? prime_in1 : prime_in0) != prime;
      if (bi) prime_in1 = prime;
      else prime_in0 = prime;
      if (lane == 0) mbar_expect_tx(&full[bi], (unsigned)(D::S * W * 8 + (new_tw ? D::S * 16 : 0)));
      __syncwarp();
      const uint64_t* src = (b.src ? b.src + ((long)p * b.src_poly_stride + limb) * N
                                   : b.data + ((long)p * b.poly_stride + limb) * N) + (long)blockIdx.x * W;
      for (int r = lane; r < D::S; r += 32)
        bulk_g2s(sbuf + (bi * WORDS + Tl::row(r)) * 8, src + r * C, W * 8, &full[bi]);
      if (new_tw) {                       // one 16-byte copy per entry, into the PERM order
        const ShoupW* tsrc = (FWD ? b.tw : b.itw) + (long)prime * N;
        for (int e = lane; e < D::S; e += 32)
          bulk_g2s(smem_u32(tws + bi * D::S + low_tw_perm<LOG_R>(e)), tsrc + e, 16, &full[bi]);
      }
      issued = it + 1;
    }
    if (!ok && lane == 0) atomicOr(b.err, kErrWaitTimeout);
    // the last copies into each buffer land before the CTA may exit (bounded)
    if (issued >= 1) mbar_wait(&full[(issued - 1) & 1], ((issued - 1) >> 1) & 1);
    if (issued >= 2) mbar_wait(&full[(issued - 2) & 1], ((issued - 2) >> 1) & 1);
    return;
  }
  // compute warps: lanes (column w of the tile, thread t of its column)
  const int t = lane % D::T;
  const int w = warp * CW + lane / D::T;
  for (int j = j_lo, it = 0; j < j_hi; j++, it++) {
    const int bi = it & 1;
    if (!mbar_wait(&full[bi], (it >> 1) & 1, b.spin)) {
      if (lane == 0) atomicOr(b.err, kErrWaitTimeout);
      return;
    }
    const int limb = j / b.npolys, p = j % b.npolys;
    const PrimeConst& P = b.pc[prime_of(j)];
    const uint64_t q = P.q;
    const uint32_t sm = sbuf + (bi * WORDS + w) * 8;          // + row(r) * 8
    const uint32_t stw = smem_u32(tws + bi * D::S);
    uint64_t* x = b.data + ((long)p * b.poly_stride + limb) * N + (long)blockIdx.x * W + w;
    if (FWD) {
      uint64_t v[D::E];
#pragma unroll
      for (int h = 0; h < D::E; h++) v[h] = lds64(sm + Tl::row((h << D::LO) + t) * 8);
      fwd_high_s<LOG_R, kButterflyLazy>(v, stw, q);
#pragma unroll
      for (int h = 0; h < D::E; h++) sts64(sm + Tl::row((h << D::LO) + t) * 8, v[h]);
      __syncwarp();
#pragma unroll
      for (int g = 0; g < D::G; g++) {
        const int hi = t * D::G + g;
        uint64_t u[D::L];
#pragma unroll
        for (int l = 0; l < D::L; l++) u[l] = lds64(sm + Tl::row((hi << D::LO) + l) * 8);
        fwd_low_s<LOG_R, kButterflyLazy, true>(u, stw, hi, q);
#pragma unroll
        for (int l = 0; l < D::L; l++) x[(long)((hi << D::LO) + l) * C] = u[l];
      }
    } else {
      const ShoupW ninv{P.ninv, P.ninv_sh}, ninv_w1{P.ninv_w1, P.ninv_w1_sh};
#pragma unroll
      for (int g = 0; g < D::G; g++) {
        const int hi = t * D::G + g;
        uint64_t u[D::L];
#pragma unroll
        for (int l = 0; l < D::L; l++) u[l] = lds64(sm + Tl::row((hi << D::LO) + l) * 8);
        inv_low_s<LOG_R, kButterflyLazy, true>(u, stw, hi, q);
#pragma unroll
        for (int l = 0; l < D::L; l++) sts64(sm + Tl::row((hi << D::LO) + l) * 8, u[l]);
      }
      __syncwarp();
      uint64_t v[D::E];
#pragma unroll
      for (int h = 0; h < D::E; h++) v[h] = lds64(sm + Tl::row((h << D::LO) + t) * 8);
      inv_high_s<LOG_R, kButterflyLazy>(v, stw, q, ninv, ninv_w1);
#pragma unroll
      for (int h = 0; h < D::E; h++) x[(long)((h << D::LO) + t) * C] = v[h];
    }
    // the buffer (tile and twiddles) is free once every lane has read it;
    // the async-proxy refill is ordered after these generic accesses
    fence_proxy_async();
    __syncwarp();
    if (lane == 0) mbar_arrive(&empty[bi]);
  }
}

// swizzled word offset inside one row of shared memory
template <int LOG_S>
__device__ __forceinline__ int swz(int hi, int lo) {
  return (hi << Sub<LOG_S>::LO) + (lo ^ (hi & (Sub<LOG_S>::L - 1)));
}

// Row pass.  Tile = ROWS contiguous rows of one limb: one bulk copy.  A row's
// threads share a warp, so the exchange needs only the warp; the one CTA
// barrier per item (after the tile's mbarrier) also frees the previous
// item's buffer for the next copy, and the high-digit twiddles alternate
// between two buffers per limb, as in the column pass.
template <int LOG_C, int DIV, int LAZY, bool FWD>
__global__ void __launch_bounds__(RowTile<LOG_C, DIV>::THREADS, RowTile<LOG_C, DIV>::MIN_BLOCKS)
ntt_rows(NttBatch b, const __grid_constant__ NttEpi epi) {
  using D = Sub<LOG_C>;
  constexpr int ROWS = RowTile<LOG_C, DIV>::ROWS;
  constexpr int TILE = ROWS * D::S;
  constexpr int NT1 = D::E - 1;                           // high-digit twiddles per row
  extern __shared__ __align__(128) uint64_t dyn[];
  __shared__ __align__(8) uint64_t mbar[2];
  const uint32_t sbuf = smem_u32(dyn);                    // [2][ROWS][S] words
  ShoupW* tw1 = (ShoupW*)(dyn + 2 * TILE);                 // [2][ROWS][NT1], alternating per limb
  const int t = threadIdx.x % D::T, rho = threadIdx.x / D::T;
  const long N = 1L << b.log_n;
  const int G = gridDim.y;
  const uint32_t row0 = blockIdx.x * ROWS;
  const uint32_t Kbase = (1u << b.log_r) + row0;

  if (threadIdx.x == 0) {
    mbar_init(&mbar[0], 1);
    mbar_init(&mbar[1], 1);
    mbar_init_fence();
  }
  __syncthreads();
  auto src_of = [&](int j) -> const uint64_t* {
    const int limb = j / b.npolys, p = j % b.npolys;
    if (b.src) return b.src + ((long)p * b.src_poly_stride + limb) * N + ((long)row0 << LOG_C);
    return b.data + ((long)p * b.poly_stride + limb) * N + ((long)row0 << LOG_C);
  };
  auto dst_of = [&](int j) -> uint64_t* {
    const int limb = j / b.npolys, p = j % b.npolys;
    return b.data + ((long)p * b.poly_stride + limb) * N + ((long)row0 << LOG_C);
  };
  auto issue = [&](int j, int bi) {
    mbar_expect_tx(&mbar[bi], TILE * 8);
    bulk_g2s(sbuf + bi * TILE * 8, src_of(j), TILE * 8, &mbar[bi]);
  };
  ShoupW w2[D::G][D::L - 1];
  int cur_limb = -1, tb = 1;
  uint64_t q = 0;
  const int j_lo = (int)((long)blockIdx.y * b.nitems / G), j_hi = (int)((long)(blockIdx.y + 1) * b.nitems / G);
  if (threadIdx.x == 0 && j_lo < j_hi) issue(j_lo, 0);
  for (int j = j_lo, it = 0; j < j_hi; j++, it++) {
    const int bi = it & 1;
    const int limb = j / b.npolys;
    if (limb != cur_limb) {                // the other buffer's users are at least one item behind
      tb ^= 1;
      const int prime = b.first_prime + (limb >> b.prime_shift);
      const ShoupW* tw = (FWD ? b.tw : b.itw) + (long)prime * N;
      for (int e = threadIdx.x; e < ROWS * NT1; e += blockDim.x) {
        const int r = e / NT1, jj = e % NT1;
        const int lvl = 31 - __clz(jj + 1);
        tw1[tb * ROWS * NT1 + e] = tw[((Kbase + r) << lvl) + jj + 1 - (1 << lvl)];
      }
      load_low_tw<LOG_C>(w2, tw, Kbase + rho, t);
      q = b.pc[prime].q;
      cur_limb = limb;
    }
    const bool ok = mbar_wait(&mbar[bi], (it >> 1) & 1, b.spin);
    if (__syncthreads_or(!ok)) {
      if (threadIdx.x == 0) {
        atomicOr(b.err, kErrWaitTimeout);
        mbar_wait(&mbar[bi], (it >> 1) & 1);   // the copy in flight: give it one more bounded wait
      }
      return;
    }
    // every thread is past item j - 1: its buffer takes the next tile
    if (threadIdx.x == 0 && j + 1 < j_hi) issue(j + 1, bi ^ 1);
    const uint32_t st1 = smem_u32(tw1 + tb * ROWS * NT1 + rho * NT1);
    const uint32_t s = sbuf + (bi * TILE + rho * D::S) * 8;
    uint64_t* x = dst_of(j) + rho * D::S;
    uint64_t v[D::E];
    if (FWD) {
#pragma unroll
      for (int h = 0; h < D::E; h++) v[h] = lds64(s + ((h << D::LO) + t) * 8);
#pragma unroll
      for (int i = D::HI - 1; i >= 0; i--) {
        const int span = 1 << i;
#pragma unroll
        for (int h = 0; h < D::E; h++) {
          if (h & span) continue;
          const ShoupW wv = ldsw(st1 + 16 * ((1 << (D::HI - 1 - i)) - 1 + (h >> (i + 1))));
          Bf<LAZY>::ct(v[h], v[h + span], wv, q, ((D::HI - 1 - i) & 1) == 0);
        }
      }
      __syncwarp();
#pragma unroll
      for (int h = 0; h < D::E; h++) sts64(s + swz<LOG_C>(h, t) * 8, v[h]);
      __syncwarp();
#pragma unroll
      for (int gg = 0; gg < D::G; gg++) {
        const int hi = t * D::G + gg;
        uint64_t u[D::L];
#pragma unroll
        for (int l = 0; l < D::L; l++) u[l] = lds64(s + swz<LOG_C>(hi, l) * 8);
        fwd_low_r<LOG_C, LAZY>(u, w2[gg], q);
#pragma unroll
        for (int l = 0; l < D::L; l++) sts64(s + swz<LOG_C>(hi, l) * 8, u[l]);
      }
      __syncwarp();
      if (epi.mode == kEpiStore) {
#pragma unroll
        for (int h = 0; h < D::E; h++) x[(h << D::LO) + t] = Bf<LAZY>::fwd_out(lds64(s + swz<LOG_C>(h, t) * 8), q);
      } else {
        const int limb = j / b.npolys;
        const long p = b.poly_base + j % b.npolys;
        const int prime = b.first_prime + (limb >> b.prime_shift);
        const PrimeConst& P = b.pc[prime];
        const long c0 = (long)(row0 + rho) << LOG_C;
#pragma unroll
        for (int h = 0; h < D::E; h++)
          epi_store(epi, N, p, limb, prime, c0 + (h << D::LO) + t, Bf<LAZY>::fwd_out(lds64(s + swz<LOG_C>(h, t) * 8), q),
                    P);
      }
    } else {
#pragma unroll
      for (int h = 0; h < D::E; h++) v[h] = lds64(s + ((h << D::LO) + t) * 8);
      __syncwarp();
#pragma unroll
      for (int h = 0; h < D::E; h++) sts64(s + swz<LOG_C>(h, t) * 8, v[h]);
      __syncwarp();
#pragma unroll
      for (int gg = 0; gg < D::G; gg++) {
        const int hi = t * D::G + gg;
        uint64_t u[D::L];
#pragma unroll
        for (int l = 0; l < D::L; l++) u[l] = lds64(s + swz<LOG_C>(hi, l) * 8);
        inv_low_r<LOG_C, LAZY>(u, w2[gg], q);
#pragma unroll
        for (int l = 0; l < D::L; l++) sts64(s + swz<LOG_C>(hi, l) * 8, u[l]);
      }
      __syncwarp();
#pragma unroll
      for (int h = 0; h < D::E; h++) v[h] = lds64(s + swz<LOG_C>(h, t) * 8);
#pragma unroll
      for (int i = 0; i < D::HI; i++) {
        const int span = 1 << i;
#pragma unroll
        for (int h = 0; h < D::E; h++) {
          if (h & span) continue;
          const ShoupW wv = ldsw(st1 + 16 * ((1 << (D::HI - 1 - i)) - 1 + (h >> (i + 1))));
          Bf<LAZY>::gs(v[h], v[h + span], wv, q);
        }
      }
#pragma unroll
      for (int h = 0; h < D::E; h++) x[(h << D::LO) + t] = v[h];
    }
    // generic-proxy accesses of buffer bi end here (see the column pass)
    fence_proxy_async();
  }
}

// ---- host launchers ----------------------------------------------------------

// CTAs per tile column: about one resident wave of CTAs (blocks_per_sm per SM)
static int ctas_per_tile(const Engine& E, int tiles, int items, int blocks_per_sm) {
  // large launches balance better with more, shorter-lived CTAs (the hardware
  // hands later waves to the SMs that finish first); small ones pay per CTA
  const double waves = items >= kLargeItems ? E.tune.ntt_waves_large : E.tune.ntt_waves;
  const int target = std::max(1, (int)(waves * E.num_sms * blocks_per_sm) / std::max(1, tiles));
  return std::max(1, std::min(items, target));
}

// The column pass's tile as a 4-D tensor map over the launch's limbs: (column,
// row, limb, poly) with strides 8 B, 8C B, 8N B and 8 N poly_stride B, box
// (W, R, 1, 1); x = blockIdx.x W is a multiple of 16 bytes.  False when the
// tile does not fit a box (R > 256) or the driver has no encoder.
static bool col_tensor_map(const NttBatch& b, int W, CUtensorMap* map) {
  using EncodeFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
  static EncodeFn encode = [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      return (EncodeFn) nullptr;
    return (EncodeFn)p;
  }();
  const long R = 1L << b.log_r, C = 1L << b.log_c, N = 1L << b.log_n;
  if (!encode || R > 256 || W * 8 % 16) return false;
  const uint64_t* base = b.src ? b.src : b.data;
  const long pstride = b.src ? b.src_poly_stride : b.poly_stride;
  const cuuint64_t dims[4] = {(cuuint64_t)C, (cuuint64_t)R, (cuuint64_t)(b.nitems / b.npolys), (cuuint64_t)b.npolys};
  const cuuint64_t strides[3] = {(cuuint64_t)C * 8, (cuuint64_t)N * 8, (cuuint64_t)pstride * N * 8};
  const cuuint32_t box[4] = {(cuuint32_t)W, (cuuint32_t)R, 1, 1};
  const cuuint32_t estride[4] = {1, 1, 1, 1};
  return encode(map, CU_TENSOR_MAP_DATA_TYPE_UINT64, 4, (void*)base, dims, strides, box, estride,
                CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

template <int LOG_R, int DIV, int LAZY>
static void launch_cols(const Engine& E, const NttBatch& b0, bool fwd, cudaStream_t st) {
  using Tl = ColTile<LOG_R, DIV>;
  const int C = 1 << b0.log_c;
  if (C % Tl::W) throw AoaError(AOA_ERR_BAD_PARAM, "ntt: column tile does not divide C");
  NttBatch b = b0;
  CUtensorMap map{};
  // a tensor-map tile load needs the rows of the tile in order (no row swizzle: W = 16)
  b.use_tma = E.tune.ntt_cols_tma && Tl::W == 16 && col_tensor_map(b, Tl::W, &map) ? 1 : 0;
  dim3 grid(C / Tl::W, ctas_per_tile(E, C / Tl::W, b.nitems, Tl::MIN_BLOCKS));
  // the inverse column pass keeps the general remainder on primes
  // q = 1 mod 2^32: with the short one it measured 3% slower (more carries on
  // the multiply pipe in its Gentleman-Sande butterflies)
  constexpr int INV = LAZY == kButterflyLazyQ1 ? kButterflyLazy : LAZY;
  if (fwd) ntt_cols<LOG_R, DIV, LAZY, true><<<grid, Tl::THREADS, Tl::SMEM, st>>>(b, map);
  else ntt_cols<LOG_R, DIV, INV, false><<<grid, Tl::THREADS, Tl::SMEM, st>>>(b, map);
  note_launch();
}

template <int LOG_R, int NW>
static void launch_cols_wo(const Engine& E, const NttBatch& b, bool fwd, cudaStream_t st) {
  using Tl = WoTile<LOG_R, NW>;
  const int C = 1 << b.log_c;
  if (C % Tl::W) throw AoaError(AOA_ERR_BAD_PARAM, "ntt: column tile does not divide C");
  dim3 grid(C / Tl::W, ctas_per_tile(E, C / Tl::W, b.nitems, Tl::MIN_BLOCKS));
  if (fwd) ntt_cols_wo<LOG_R, NW, true><<<grid, Tl::THREADS, Tl::SMEM, st>>>(b);
  else ntt_cols_wo<LOG_R, NW, false><<<grid, Tl::THREADS, Tl::SMEM, st>>>(b);
  note_launch();
}

template <int LOG_C, int DIV, int LAZY>
static void launch_rows(const Engine& E, const NttBatch& b, bool fwd, cudaStream_t st, const NttEpi& epi) {
  using Tl = RowTile<LOG_C, DIV>;
  const int R = 1 << b.log_r;
  if (R % Tl::ROWS) throw AoaError(AOA_ERR_BAD_PARAM, "ntt: row tile does not divide R");
  dim3 grid(R / Tl::ROWS, ctas_per_tile(E, R / Tl::ROWS, b.nitems, Tl::MIN_BLOCKS));
  if (fwd) ntt_rows<LOG_C, DIV, LAZY, true><<<grid, Tl::THREADS, Tl::SMEM, st>>>(b, epi);
  else ntt_rows<LOG_C, DIV, LAZY, false><<<grid, Tl::THREADS, Tl::SMEM, st>>>(b, epi);
  note_launch();
}

#define AOA_NTT_SIZES(X) X(5) X(6) X(7) X(8) X(9) X(10)

// Tile width choice (DIV) for a launch: the engine's tuning for lazy
// transforms; strict transforms (primes of 62 bits or more) use the widest.
template <int LAZY>
static int tile_div(int knob) { return LAZY ? std::max(0, std::min(2, knob)) : 0; }

template <int LAZY>
static void run_cols(const Engine& E, const NttBatch& b, bool fwd, cudaStream_t st) {
  const int div = tile_div<LAZY>(E.tune.ntt_cols_div);
  if (LAZY && E.tune.ntt_cols_kind == 1 && b.log_r >= 6 && b.log_r <= 9) {
    // warp-owned columns: 8, 4 or 2 compute warps per CTA
    switch (b.log_r * 4 + div) {
#define AOA_WO(s)                                                    \
  case s * 4 + 0: launch_cols_wo<s, 8>(E, b, fwd, st); return;       \
  case s * 4 + 1: launch_cols_wo<s, 4>(E, b, fwd, st); return;       \
  case s * 4 + 2: launch_cols_wo<s, 2>(E, b, fwd, st); return;
      AOA_WO(6) AOA_WO(7) AOA_WO(8) AOA_WO(9)
#undef AOA_WO
      default: break;
    }
  }
  switch (b.log_r) {
#define AOA_CASE(s)                                                \
  case s:                                                          \
    if constexpr (!LAZY) launch_cols<s, 0, LAZY>(E, b, fwd, st);     \
    else if (div == 0) launch_cols<s, 0, LAZY>(E, b, fwd, st);      \
    else if (div == 1) launch_cols<s, 1, LAZY>(E, b, fwd, st);      \
    else launch_cols<s, 2, LAZY>(E, b, fwd, st);                    \
    break;
    AOA_NTT_SIZES(AOA_CASE)
#undef AOA_CASE
    default: throw AoaError(AOA_ERR_BAD_PARAM, "ntt: unsupported column size");
  }
}

template <int LAZY>
static void run_rows(const Engine& E, const NttBatch& b, bool fwd, cudaStream_t st, const NttEpi& epi) {
  const int div = tile_div<LAZY>(E.tune.ntt_rows_div);
  switch (b.log_c) {
#define AOA_CASE(s)                                                \
  case s:                                                          \
    if constexpr (!LAZY) launch_rows<s, 0, LAZY>(E, b, fwd, st, epi);     \
    else if (div == 0) launch_rows<s, 0, LAZY>(E, b, fwd, st, epi);      \
    else if (div == 1) launch_rows<s, 1, LAZY>(E, b, fwd, st, epi);      \
    else launch_rows<s, 2, LAZY>(E, b, fwd, st, epi);                    \
    break;
    AOA_NTT_SIZES(AOA_CASE)
#undef AOA_CASE
    default: throw AoaError(AOA_ERR_BAD_PARAM, "ntt: unsupported row size");
  }
}

template <class K>
static void allow_smem(K kernel, size_t bytes) {
  AOA_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
}

template <int S, int DIV, int KIND>
static void allow_kind() {
  allow_smem(ntt_cols<S, DIV, KIND, true>, ColTile<S, DIV>::SMEM);
  if constexpr (KIND != kButterflyLazyQ1) allow_smem(ntt_cols<S, DIV, KIND, false>, ColTile<S, DIV>::SMEM);
  allow_smem(ntt_rows<S, DIV, KIND, true>, RowTile<S, DIV>::SMEM);
  allow_smem(ntt_rows<S, DIV, KIND, false>, RowTile<S, DIV>::SMEM);
}

template <int S, int DIV>
static void allow_size() {
  allow_kind<S, DIV, kButterflyLazy>();
  allow_kind<S, DIV, kButterflyLazyQ1>();
  if (DIV == 0) allow_kind<S, 0, kButterflyCanonical>();
}

// Once per engine: opt every transform kernel in to its dynamic shared memory.
template <int S, int NW>
static void allow_wo() {
  allow_smem(ntt_cols_wo<S, NW, true>, WoTile<S, NW>::SMEM);
  allow_smem(ntt_cols_wo<S, NW, false>, WoTile<S, NW>::SMEM);
}

void ntt_init(Engine& E) {
#define AOA_ALLOW(s) allow_size<s, 0>(); allow_size<s, 1>(); allow_size<s, 2>();
  AOA_NTT_SIZES(AOA_ALLOW)
#undef AOA_ALLOW
#define AOA_ALLOW_WO(s) allow_wo<s, 8>(); allow_wo<s, 4>(); allow_wo<s, 2>();
  AOA_ALLOW_WO(6) AOA_ALLOW_WO(7) AOA_ALLOW_WO(8) AOA_ALLOW_WO(9)
#undef AOA_ALLOW_WO
  int sms = 0;
  AOA_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, E.device));
  E.num_sms = sms;
}

// Small transforms (N < 1024): one CTA per item, the whole limb in shared
// memory, one radix-2 stage per step, canonical (strict) butterflies with the
// same merged tables as the large kernels.
__global__ void ntt_small(NttBatch b, bool fwd) {
  extern __shared__ __align__(16) uint64_t xs[];
  const int N = 1 << b.log_n;
  for (int j = blockIdx.x; j < b.nitems; j += gridDim.x) {
    const int limb = j / b.npolys, p = j % b.npolys;
    const int prime = b.first_prime + (limb >> b.prime_shift);
    uint64_t* x = b.data + ((long)p * b.poly_stride + limb) * N;
    const PrimeConst& P = b.pc[prime];
    const uint64_t q = P.q;
    const ShoupW* tw = (fwd ? b.tw : b.itw) + (long)prime * N;
    __syncthreads();
    for (int i = threadIdx.x; i < N; i += blockDim.x) xs[i] = x[i];
    __syncthreads();
    if (fwd) {
      for (int m = 1; m < N; m <<= 1) {
        const int t = N / (2 * m);
        for (int bf = threadIdx.x; bf < N / 2; bf += blockDim.x) {
          const int g = bf / t, l = bf % t, i0 = 2 * g * t + l;
          const uint64_t u = xs[i0], v = shoup(xs[i0 + t], tw[m + g], q);
          xs[i0] = add_mod(u, v, q);
          xs[i0 + t] = sub_mod(u, v, q);
        }
        __syncthreads();
      }
      for (int i = threadIdx.x; i < N; i += blockDim.x) x[i] = xs[i];
    } else {
      for (int m = N / 2; m >= 1; m >>= 1) {
        const int t = N / (2 * m);
        for (int bf = threadIdx.x; bf < N / 2; bf += blockDim.x) {
          const int g = bf / t, l = bf % t, i0 = 2 * g * t + l;
          const uint64_t u = xs[i0], v = xs[i0 + t];
          xs[i0] = add_mod(u, v, q);
          xs[i0 + t] = shoup(sub_mod(u, v, q), tw[m + g], q);
        }
        __syncthreads();
      }
      for (int i = threadIdx.x; i < N; i += blockDim.x) x[i] = shoup(xs[i], P.ninv, P.ninv_sh, q);
    }
  }
}

// Transform limbs [0, nlimbs) of npolys polys (layout [npolys][poly_stride][N],
// N = 2^T.log_n) with the tables T; limb l under prime first_prime +
// (l >> T.prime_shift).  Large transforms are split into chunks of whole polys
// of at most tune.ntt_chunk_bytes, column and row pass per chunk.
void ntt_batch_tables(const Engine& E, const NttTables& T, uint64_t* data, int npolys, int first_prime, int nlimbs,
                      long poly_stride, bool forward, cudaStream_t st, const NttIo* io) {
  if (npolys <= 0 || nlimbs <= 0) return;
  if (first_prime < 0 || first_prime + ((nlimbs - 1) >> T.prime_shift) >= E.nprimes)
    throw AoaError(AOA_ERR_BAD_PARAM, "ntt: prime range out of bounds");
  if (T.prime_kind && T.log_n >= 10) {
    // Primes of different butterfly kinds (the reference's prime sets put a
    // 63-bit q0 before its 45..55-bit buckets): the limbs run in maximal runs
    // of one kind, the lazy kernels for primes below 2^kLazyPrimeBits (with
    // the shorter remainder where q = 1 mod 2^32), the canonical ones for the
    // rest.  Runs start at prime boundaries; each run's data, source and
    // epilogue limbs are offset by its first limb.
    const long n = 1L << T.log_n;
    auto kind_at = [&](int l) { return (int)T.prime_kind[first_prime + (l >> T.prime_shift)]; };
    for (int l0 = 0; l0 < nlimbs;) {
      const int kind = kind_at(l0);
      int l1 = l0 + 1;
      while (l1 < nlimbs && kind_at(l1) == kind) l1++;
      NttTables T2 = T;
      T2.kind = kind;
      T2.prime_kind = nullptr;
      if (l0 == 0 && l1 == nlimbs) {
        ntt_batch_tables(E, T2, data, npolys, first_prime, nlimbs, poly_stride, forward, st, io);
        return;
      }
      NttIo run;
      if (io) run = *io;
      if (run.src) run.src += (long)l0 * n;
      run.epi.limb_base += l0;
      ntt_batch_tables(E, T2, data + (long)l0 * n, npolys, first_prime + (l0 >> T.prime_shift), l1 - l0,
                       poly_stride, forward, st, &run);
      l0 = l1;
    }
    return;
  }
  const NttEpi no_epi{};
  const NttEpi& epi = io ? io->epi : no_epi;
  if (epi.mode != kEpiStore && !forward) throw AoaError(AOA_ERR_BAD_PARAM, "ntt: epilogues are for forward transforms");
  // the passes move tiles with bulk / tensor-map copies, which need 16-byte
  // aligned addresses: limbs start at data + multiples of N words (N >= 2^10)
  if (((uintptr_t)data & 15) || (io && io->src && ((uintptr_t)io->src & 15)))
    throw AoaError(AOA_ERR_BAD_PARAM, "ntt: device data must be 16-byte aligned");
  NttBatch b;
  b.tw = T.tw; b.itw = T.itw; b.pc = T.pc; b.err = E.d_err;
  b.spin = E.tune.spin_limit;
  b.log_n = T.log_n;
  b.log_c = T.log_n / 2 + T.split;
  b.log_c = std::max(std::max(5, T.log_n - 10), std::min(std::min(10, T.log_n - 5), b.log_c));
  b.log_r = T.log_n - b.log_c;
  b.first_prime = first_prime; b.prime_shift = T.prime_shift; b.poly_stride = poly_stride;
  b.src = nullptr; b.src_poly_stride = 0; b.poly_base = 0; b.use_tma = 0;
  const long n = 1L << T.log_n;
  if (T.log_n < 10) {
    // small rings: the out-of-place source is copied first and the epilogue
    // runs as its own pass
    if (io && io->src)
      AOA_CUDA(cudaMemcpy2DAsync(data, poly_stride * n * 8, io->src, io->src_poly_stride * n * 8,
                                 (size_t)nlimbs * n * 8, npolys, cudaMemcpyDeviceToDevice, st));
    b.npolys = npolys;
    b.nitems = npolys * nlimbs;
    b.data = data;
    const int grid = std::min(b.nitems, 8 * E.num_sms);
    ntt_small<<<grid, std::max(32, std::min((int)n / 2, 256)), n * 8, st>>>(b, forward);
    note_launch();
    if (epi.mode != kEpiStore) {
      ntt_epilogue_kernel<<<2 * E.num_sms, 256, 0, st>>>(data, poly_stride, npolys, nlimbs, first_prime,
                                                         T.prime_shift, T.pc, T.log_n, epi);
      note_launch();
    }
    AOA_CHECK_LAUNCH();
    return;
  }
  const long limb_bytes = 8 * n;
  const long chunk = std::max(1L, E.tune.ntt_chunk_bytes / (limb_bytes * nlimbs));
  for (long c0 = 0; c0 < npolys; c0 += chunk) {
    const int np = (int)std::min<long>(chunk, npolys - c0);
    b.npolys = np;
    b.nitems = np * nlimbs;
    b.data = data + c0 * poly_stride * n;
    b.poly_base = (int)c0;
    NttBatch first = b;                    // the first pass may read out of place
    if (io && io->src) {
      first.src = io->src + c0 * io->src_poly_stride * n;
      first.src_poly_stride = io->src_poly_stride;
    }
    switch (T.kind) {
#define AOA_KIND(K)                                                                   \
  case K:                                                                             \
    if (forward) { run_cols<K>(E, first, true, st); run_rows<K>(E, b, true, st, epi); }  \
    else { run_rows<K>(E, first, false, st, no_epi); run_cols<K>(E, b, false, st); }     \
    break;
      AOA_KIND(kButterflyCanonical) AOA_KIND(kButterflyLazy) AOA_KIND(kButterflyLazyQ1)
#undef AOA_KIND
      default: throw AoaError(AOA_ERR_BAD_PARAM, "ntt: unknown butterfly kind");
    }
  }
  AOA_CHECK_LAUNCH();
}

// Negacyclic limb transforms of the engine's ring (psi^bitrev tables).
void ntt_batch(const Engine& E, uint64_t* data, int npolys, int first_prime, int nlimbs,
               long poly_stride, bool forward, cudaStream_t st) {
  NttTables T;
  T.tw = E.d_tw; T.itw = E.d_itw; T.pc = E.d_pc;
  T.log_n = E.log_n; T.prime_shift = 0; T.kind = std::max(E.ntt_kind, 0);
  T.split = E.tune.ntt_split;
  if (E.ntt_kind < 0) T.prime_kind = E.prime_kind.data();
  ntt_batch_tables(E, T, data, npolys, first_prime, nlimbs, poly_stride, forward, st, nullptr);
}

// Limb transforms with a fused source and / or epilogue (NttIo).
void ntt_batch_io(const Engine& E, uint64_t* data, int npolys, int first_prime, int nlimbs, long poly_stride,
                  bool forward, const NttIo& io, cudaStream_t st) {
  NttTables T;
  T.tw = E.d_tw; T.itw = E.d_itw; T.pc = E.d_pc;
  T.log_n = E.log_n; T.prime_shift = 0; T.kind = std::max(E.ntt_kind, 0);
  T.split = E.tune.ntt_split;
  if (E.ntt_kind < 0) T.prime_kind = E.prime_kind.data();
  ntt_batch_tables(E, T, data, npolys, first_prime, nlimbs, poly_stride, forward, st, &io);
}

}  // namespace aoa
