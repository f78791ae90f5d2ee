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
// passes.  Passes run in place; the host launches them over chunks of limbs
// sized so that the column-pass output is still in L2 when the row pass reads
// it.
#include "aoa_internal.h"

namespace aoa {

template <int LOG_S>
struct Sub {
  static constexpr int S = 1 << LOG_S;
  static constexpr int HI = (LOG_S + 1) / 2;   // high digit width (round 1)
  static constexpr int LO = LOG_S / 2;         // low digit width (round 2)
  static constexpr int T = 1 << LO;            // threads per sub-transform
  static constexpr int E = 1 << HI;            // elements per thread
  static constexpr int G = 1 << (HI - LO);     // low-digit groups per thread (1 or 2)
  static constexpr int L = 1 << LO;            // elements per low-digit group
  // sub-transforms per CTA: <= 256 threads, <= 32 KiB shared memory, <= 32
  static constexpr int PER_CTA_A = 256 / T < 4096 / S ? 256 / T : 4096 / S;
  static constexpr int PER_CTA = PER_CTA_A < 32 ? PER_CTA_A : 32;
};

// ---- butterflies ------------------------------------------------------------
// Strict mode keeps every value canonical in [0, q) (any q < 2^63).  Lazy mode
// (all primes < 2^62) follows Harvey's bounds: forward values live in [0, 4q),
// inverse values in [0, 2q); the last stage of each transform reduces to [0, q).

template <bool LAZY>
struct Bf;

template <>
struct Bf<false> {
  static __device__ __forceinline__ void ct(uint64_t& x, uint64_t& y, ShoupW w, uint64_t q) {
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

template <>
struct Bf<true> {
  static __device__ __forceinline__ void ct(uint64_t& x, uint64_t& y, ShoupW w, uint64_t q) {
    const uint64_t q2 = q << 1;
    uint64_t U = x >= q2 ? x - q2 : x;          // [0, 2q)
    uint64_t V = shoup_lazy(y, w.w, w.wp, q);   // [0, 2q)
    x = U + V;                                  // [0, 4q)
    y = U - V + q2;                             // (0, 4q)
  }
  static __device__ __forceinline__ void gs(uint64_t& x, uint64_t& y, ShoupW w, uint64_t q) {
    const uint64_t q2 = q << 1;
    uint64_t U = x, V = y;                      // [0, 2q)
    uint64_t s = U + V;
    x = s >= q2 ? s - q2 : s;                   // [0, 2q)
    y = shoup_lazy(U - V + q2, w.w, w.wp, q);   // [0, 2q)
  }
  static __device__ __forceinline__ void gs_last(uint64_t& x, uint64_t& y, ShoupW n0, ShoupW n1, uint64_t q) {
    const uint64_t q2 = q << 1;
    uint64_t U = x, V = y;
    uint64_t a = shoup_lazy(U + V, n0.w, n0.wp, q);
    uint64_t b = shoup_lazy(U - V + q2, n1.w, n1.wp, q);
    x = a >= q ? a - q : a;
    y = b >= q ? b - q : b;
  }
  static __device__ __forceinline__ uint64_t fwd_out(uint64_t x, uint64_t q) {
    const uint64_t q2 = q << 1;
    x = x >= q2 ? x - q2 : x;
    return x >= q ? x - q : x;
  }
};

// ---- forward (Cooley-Tukey, merged twist) ---------------------------------
// twiddle index for local half-span 2^j and local group g: K * S/2^(j+1) + g

template <int LOG_S, bool LAZY>
__device__ __forceinline__ void fwd_high(uint64_t (&v)[Sub<LOG_S>::E], const ShoupW* __restrict__ tw,
                                         uint32_t K, uint64_t q) {
  using D = Sub<LOG_S>;
#pragma unroll
  for (int i = D::HI - 1; i >= 0; i--) {
    const int span = 1 << i;
#pragma unroll
    for (int g = 0; g < (1 << (D::HI - 1 - i)); g++) {
      const ShoupW w = tw[(K << (D::HI - 1 - i)) + g];
#pragma unroll
      for (int o = 0; o < span; o++) {
        const int h = (g << (i + 1)) + o;
        Bf<LAZY>::ct(v[h], v[h + span], w, q);
      }
    }
  }
}

template <int LOG_S, bool LAZY>
__device__ __forceinline__ void fwd_low(uint64_t (&u)[Sub<LOG_S>::L], const ShoupW* __restrict__ tw,
                                        uint32_t K, uint32_t hi, uint64_t q) {
  using D = Sub<LOG_S>;
#pragma unroll
  for (int i = D::LO - 1; i >= 0; i--) {
    const int span = 1 << i;
#pragma unroll
    for (int g = 0; g < (1 << (D::LO - 1 - i)); g++) {
      const ShoupW w = tw[(K << (LOG_S - 1 - i)) + (hi << (D::LO - 1 - i)) + g];
#pragma unroll
      for (int o = 0; o < span; o++) {
        const int l = (g << (i + 1)) + o;
        Bf<LAZY>::ct(u[l], u[l + span], w, q);
      }
    }
  }
}

// ---- inverse (Gentleman-Sande) -------------------------------------------

template <int LOG_S, bool LAZY>
__device__ __forceinline__ void inv_low(uint64_t (&u)[Sub<LOG_S>::L], const ShoupW* __restrict__ itw,
                                        uint32_t K, uint32_t hi, uint64_t q) {
  using D = Sub<LOG_S>;
#pragma unroll
  for (int i = 0; i < D::LO; i++) {
    const int span = 1 << i;
#pragma unroll
    for (int g = 0; g < (1 << (D::LO - 1 - i)); g++) {
      const ShoupW w = itw[(K << (LOG_S - 1 - i)) + (hi << (D::LO - 1 - i)) + g];
#pragma unroll
      for (int o = 0; o < span; o++) {
        const int l = (g << (i + 1)) + o;
        Bf<LAZY>::gs(u[l], u[l + span], w, q);
      }
    }
  }
}

// LAST: this round holds the transform's final stage (half-span N/2): scale by N^-1.
template <int LOG_S, bool LAZY, bool LAST>
__device__ __forceinline__ void inv_high(uint64_t (&v)[Sub<LOG_S>::E], const ShoupW* __restrict__ itw,
                                         uint32_t K, uint64_t q, ShoupW ninv, ShoupW ninv_w1) {
  using D = Sub<LOG_S>;
#pragma unroll
  for (int i = 0; i < D::HI; i++) {
    const int span = 1 << i;
#pragma unroll
    for (int g = 0; g < (1 << (D::HI - 1 - i)); g++) {
      const ShoupW w = itw[(K << (D::HI - 1 - i)) + g];
#pragma unroll
      for (int o = 0; o < span; o++) {
        const int h = (g << (i + 1)) + o;
        if (LAST && i == D::HI - 1) Bf<LAZY>::gs_last(v[h], v[h + span], ninv, ninv_w1, q);
        else Bf<LAZY>::gs(v[h], v[h + span], w, q);
      }
    }
  }
}

// ---- kernels ---------------------------------------------------------------
// Batch addressing: limb (poly p, limb l) lives at data + (p*poly_stride + l)*N
// and uses prime first_prime + l.  grid = (tiles per limb, nlimbs, npolys).

struct NttBatch {
  uint64_t* data;
  const ShoupW* tw;        // [nprimes][N] forward twiddles (psi^bitrev)
  const ShoupW* itw;       // [nprimes][N] inverse twiddles
  const PrimeConst* pc;    // [nprimes]
  int log_n, log_r, log_c; // N = R * C
  int first_prime;
  long poly_stride;        // limbs between consecutive polys
};

template <int LOG_R, int W, bool LAZY>
__global__ void __launch_bounds__(Sub<LOG_R>::T * W)
ntt_fwd_cols(NttBatch b) {
  using D = Sub<LOG_R>;
  __shared__ uint64_t sm[D::S][W];
  const int w = threadIdx.x % W, t = threadIdx.x / W;
  const int prime = b.first_prime + blockIdx.y;
  const long N = 1L << b.log_n, C = 1L << b.log_c;
  const uint64_t q = b.pc[prime].q;
  uint64_t* x = b.data + ((long)blockIdx.z * b.poly_stride + blockIdx.y) * N + (long)blockIdx.x * W + w;
  const ShoupW* tw = b.tw + (long)prime * N;
  uint64_t v[D::E];
#pragma unroll
  for (int h = 0; h < D::E; h++) v[h] = x[(long)((h << D::LO) + t) * C];
  fwd_high<LOG_R, LAZY>(v, tw, 1, q);
#pragma unroll
  for (int h = 0; h < D::E; h++) sm[(h << D::LO) + t][w] = v[h];
  __syncthreads();
#pragma unroll
  for (int g = 0; g < D::G; g++) {
    const int hi = t * D::G + g;
    uint64_t u[D::L];
#pragma unroll
    for (int l = 0; l < D::L; l++) u[l] = sm[(hi << D::LO) + l][w];
    fwd_low<LOG_R, LAZY>(u, tw, 1, hi, q);
#pragma unroll
    for (int l = 0; l < D::L; l++) x[(long)((hi << D::LO) + l) * C] = u[l];
  }
}

template <int LOG_R, int W, bool LAZY>
__global__ void __launch_bounds__(Sub<LOG_R>::T * W)
ntt_inv_cols(NttBatch b) {
  using D = Sub<LOG_R>;
  __shared__ uint64_t sm[D::S][W];
  const int w = threadIdx.x % W, t = threadIdx.x / W;
  const int prime = b.first_prime + blockIdx.y;
  const long N = 1L << b.log_n, C = 1L << b.log_c;
  const PrimeConst& P = b.pc[prime];
  const uint64_t q = P.q;
  const ShoupW ninv{P.ninv, P.ninv_sh}, ninv_w1{P.ninv_w1, P.ninv_w1_sh};
  uint64_t* x = b.data + ((long)blockIdx.z * b.poly_stride + blockIdx.y) * N + (long)blockIdx.x * W + w;
  const ShoupW* itw = b.itw + (long)prime * N;
#pragma unroll
  for (int g = 0; g < D::G; g++) {
    const int hi = t * D::G + g;
    uint64_t u[D::L];
#pragma unroll
    for (int l = 0; l < D::L; l++) u[l] = x[(long)((hi << D::LO) + l) * C];
    inv_low<LOG_R, LAZY>(u, itw, 1, hi, q);
#pragma unroll
    for (int l = 0; l < D::L; l++) sm[(hi << D::LO) + l][w] = u[l];
  }
  __syncthreads();
  uint64_t v[D::E];
#pragma unroll
  for (int h = 0; h < D::E; h++) v[h] = sm[(h << D::LO) + t][w];
  inv_high<LOG_R, LAZY, true>(v, itw, 1, q, ninv, ninv_w1);
#pragma unroll
  for (int h = 0; h < D::E; h++) x[(long)((h << D::LO) + t) * C] = v[h];
}

// swizzled position inside one row of shared memory
template <int LOG_S>
__device__ __forceinline__ int swz(int hi, int lo) {
  return (hi << Sub<LOG_S>::LO) + (lo ^ (hi & (Sub<LOG_S>::L - 1)));
}

template <int LOG_C, int ROWS, bool LAZY>
__global__ void __launch_bounds__(Sub<LOG_C>::T * ROWS)
ntt_fwd_rows(NttBatch b) {
  using D = Sub<LOG_C>;
  __shared__ uint64_t sm[ROWS][D::S];
  const int t = threadIdx.x % D::T, rho = threadIdx.x / D::T;
  const int prime = b.first_prime + blockIdx.y;
  const long N = 1L << b.log_n;
  const uint32_t row = blockIdx.x * ROWS + rho;
  const uint64_t q = b.pc[prime].q;
  uint64_t* x = b.data + ((long)blockIdx.z * b.poly_stride + blockIdx.y) * N + ((long)row << LOG_C);
  const ShoupW* tw = b.tw + (long)prime * N;
  const uint32_t K = (1u << b.log_r) + row;
  uint64_t* s = sm[rho];
  uint64_t v[D::E];
#pragma unroll
  for (int h = 0; h < D::E; h++) v[h] = x[(h << D::LO) + t];
  fwd_high<LOG_C, LAZY>(v, tw, K, q);
#pragma unroll
  for (int h = 0; h < D::E; h++) s[swz<LOG_C>(h, t)] = v[h];
  __syncwarp();
#pragma unroll
  for (int g = 0; g < D::G; g++) {
    const int hi = t * D::G + g;
    uint64_t u[D::L];
#pragma unroll
    for (int l = 0; l < D::L; l++) u[l] = s[swz<LOG_C>(hi, l)];
    fwd_low<LOG_C, LAZY>(u, tw, K, hi, q);
#pragma unroll
    for (int l = 0; l < D::L; l++) s[swz<LOG_C>(hi, l)] = u[l];
  }
  __syncwarp();
#pragma unroll
  for (int h = 0; h < D::E; h++) x[(h << D::LO) + t] = Bf<LAZY>::fwd_out(s[swz<LOG_C>(h, t)], q);
}

template <int LOG_C, int ROWS, bool LAZY>
__global__ void __launch_bounds__(Sub<LOG_C>::T * ROWS)
ntt_inv_rows(NttBatch b) {
  using D = Sub<LOG_C>;
  __shared__ uint64_t sm[ROWS][D::S];
  const int t = threadIdx.x % D::T, rho = threadIdx.x / D::T;
  const int prime = b.first_prime + blockIdx.y;
  const long N = 1L << b.log_n;
  const uint32_t row = blockIdx.x * ROWS + rho;
  const uint64_t q = b.pc[prime].q;
  uint64_t* x = b.data + ((long)blockIdx.z * b.poly_stride + blockIdx.y) * N + ((long)row << LOG_C);
  const ShoupW* itw = b.itw + (long)prime * N;
  const uint32_t K = (1u << b.log_r) + row;
  uint64_t* s = sm[rho];
#pragma unroll
  for (int h = 0; h < D::E; h++) s[swz<LOG_C>(h, t)] = x[(h << D::LO) + t];
  __syncwarp();
#pragma unroll
  for (int g = 0; g < D::G; g++) {
    const int hi = t * D::G + g;
    uint64_t u[D::L];
#pragma unroll
    for (int l = 0; l < D::L; l++) u[l] = s[swz<LOG_C>(hi, l)];
    inv_low<LOG_C, LAZY>(u, itw, K, hi, q);
#pragma unroll
    for (int l = 0; l < D::L; l++) s[swz<LOG_C>(hi, l)] = u[l];
  }
  __syncwarp();
  uint64_t v[D::E];
#pragma unroll
  for (int h = 0; h < D::E; h++) v[h] = s[swz<LOG_C>(h, t)];
  inv_high<LOG_C, LAZY, false>(v, itw, K, q, ShoupW{0, 0}, ShoupW{0, 0});
#pragma unroll
  for (int h = 0; h < D::E; h++) x[(h << D::LO) + t] = v[h];
}

// ---- host launchers ----------------------------------------------------------

template <int LOG_R, bool LAZY>
static void launch_cols(const NttBatch& b, int nlimbs, int npolys, bool fwd, cudaStream_t st) {
  constexpr int T = Sub<LOG_R>::T;
  constexpr int W = Sub<LOG_R>::PER_CTA;        // columns per CTA
  const int C = 1 << b.log_c;
  if (C % W) throw AoaError(AOA_ERR_BAD_PARAM, "ntt: column tile does not divide C");
  dim3 grid(C / W, nlimbs, npolys);
  if (fwd) ntt_fwd_cols<LOG_R, W, LAZY><<<grid, T * W, 0, st>>>(b);
  else ntt_inv_cols<LOG_R, W, LAZY><<<grid, T * W, 0, st>>>(b);
  note_launch();
}

template <int LOG_C, bool LAZY>
static void launch_rows(const NttBatch& b, int nlimbs, int npolys, bool fwd, cudaStream_t st) {
  constexpr int T = Sub<LOG_C>::T;
  constexpr int ROWS = Sub<LOG_C>::PER_CTA;
  const int R = 1 << b.log_r;
  if (R % ROWS) throw AoaError(AOA_ERR_BAD_PARAM, "ntt: row tile does not divide R");
  dim3 grid(R / ROWS, nlimbs, npolys);
  if (fwd) ntt_fwd_rows<LOG_C, ROWS, LAZY><<<grid, T * ROWS, 0, st>>>(b);
  else ntt_inv_rows<LOG_C, ROWS, LAZY><<<grid, T * ROWS, 0, st>>>(b);
  note_launch();
}

template <bool LAZY>
static void run_cols(const NttBatch& b, int nlimbs, int npolys, bool fwd, cudaStream_t st) {
  switch (b.log_r) {
    case 5: launch_cols<5, LAZY>(b, nlimbs, npolys, fwd, st); break;
    case 6: launch_cols<6, LAZY>(b, nlimbs, npolys, fwd, st); break;
    case 7: launch_cols<7, LAZY>(b, nlimbs, npolys, fwd, st); break;
    case 8: launch_cols<8, LAZY>(b, nlimbs, npolys, fwd, st); break;
    case 9: launch_cols<9, LAZY>(b, nlimbs, npolys, fwd, st); break;
    case 10: launch_cols<10, LAZY>(b, nlimbs, npolys, fwd, st); break;
    default: throw AoaError(AOA_ERR_BAD_PARAM, "ntt: unsupported column size");
  }
}

template <bool LAZY>
static void run_rows(const NttBatch& b, int nlimbs, int npolys, bool fwd, cudaStream_t st) {
  switch (b.log_c) {
    case 5: launch_rows<5, LAZY>(b, nlimbs, npolys, fwd, st); break;
    case 6: launch_rows<6, LAZY>(b, nlimbs, npolys, fwd, st); break;
    case 7: launch_rows<7, LAZY>(b, nlimbs, npolys, fwd, st); break;
    case 8: launch_rows<8, LAZY>(b, nlimbs, npolys, fwd, st); break;
    case 9: launch_rows<9, LAZY>(b, nlimbs, npolys, fwd, st); break;
    case 10: launch_rows<10, LAZY>(b, nlimbs, npolys, fwd, st); break;
    default: throw AoaError(AOA_ERR_BAD_PARAM, "ntt: unsupported row size");
  }
}

// Transform limbs [0, nlimbs) of npolys polys (layout [npolys][poly_stride][N]),
// limb l under prime first_prime + l.  Work is split into chunks of whole polys
// whose total size stays within the L2 budget, column and row pass per chunk.
void ntt_batch(const Engine& E, uint64_t* data, int npolys, int first_prime, int nlimbs,
               long poly_stride, bool forward, cudaStream_t st) {
  if (npolys <= 0 || nlimbs <= 0) return;
  if (first_prime < 0 || first_prime + nlimbs > E.nprimes)
    throw AoaError(AOA_ERR_BAD_PARAM, "ntt: prime range out of bounds");
  NttBatch b;
  b.tw = E.d_tw; b.itw = E.d_itw; b.pc = E.d_pc;
  b.log_n = E.log_n; b.log_c = E.log_c; b.log_r = E.log_n - E.log_c;
  b.first_prime = first_prime; b.poly_stride = poly_stride;
  const long limb_bytes = (8L << E.log_n);
  long chunk = std::max(1L, E.tune.ntt_chunk_bytes / (limb_bytes * nlimbs));
  for (long p0 = 0; p0 < npolys; p0 += chunk) {
    int np = (int)std::min<long>(chunk, npolys - p0);
    b.data = data + p0 * poly_stride * (1L << E.log_n);
    if (E.lazy) {
      if (forward) { run_cols<true>(b, nlimbs, np, true, st); run_rows<true>(b, nlimbs, np, true, st); }
      else { run_rows<true>(b, nlimbs, np, false, st); run_cols<true>(b, nlimbs, np, false, st); }
    } else {
      if (forward) { run_cols<false>(b, nlimbs, np, true, st); run_rows<false>(b, nlimbs, np, true, st); }
      else { run_rows<false>(b, nlimbs, np, false, st); run_cols<false>(b, nlimbs, np, false, st); }
    }
  }
  AOA_CHECK_LAUNCH();
}

}  // namespace aoa
