// Internal declarations shared by the engine's translation units.
#pragma once
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <stdexcept>
#include <string>
#include <mutex>
#include <vector>

#include "../../include/aoa_ckks.h"
#include "modarith.cuh"

namespace aoa {

struct AoaError : public std::runtime_error {
  int status;
  AoaError(int s, const std::string& m) : std::runtime_error(m), status(s) {}
};

#define AOA_CUDA(call)                                                                     \
  do {                                                                                     \
    cudaError_t e_ = (call);                                                               \
    if (e_ != cudaSuccess)                                                                 \
      throw ::aoa::AoaError(AOA_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
  } while (0)

#define AOA_CHECK_LAUNCH()                                                                 \
  do {                                                                                     \
    cudaError_t e_ = cudaGetLastError();                                                   \
    if (e_ != cudaSuccess)                                                                 \
      throw ::aoa::AoaError(AOA_ERR_CUDA, std::string("kernel launch: ") + cudaGetErrorString(e_)); \
  } while (0)

constexpr unsigned kErrWaitTimeout = 1u;   // an mbarrier wait hit its iteration limit
// Lazy transforms need every prime below 2^kLazyPrimeBits: forward values
// stay below 16q < 2^64 (primes of more bits take canonical butterflies)
#ifndef AOA_LAZY_PRIME_BITS
#define AOA_LAZY_PRIME_BITS 60
#endif
constexpr int kLazyPrimeBits = AOA_LAZY_PRIME_BITS;
constexpr int kButterflyCanonical = 0, kButterflyLazy = 1, kButterflyLazyQ1 = 2;
constexpr int kLargeItems = 1536;           // limb-transform launches this large use ntt_waves_large

struct Tune {
  // Defaults: the shapes measured best on B200 at 2^16 for the batched HMult
  // pipeline (8-row tiles in the row pass) and for large transform calls
  // (4 GiB chunks, 8 waves); the autotuner can refine them per ring.
  long ntt_chunk_bytes = 1L << 32;    // limbs per transform launch pair (bytes); larger chunks
                                      // mean fewer launch tails (measured: 1 GiB beats an L2-sized chunk)
  double ntt_waves = 1.0;             // transform CTAs per pass, in resident waves
  double ntt_waves_large = 8.0;       // the same for launches of at least kLargeItems limbs
  bool conv_tensor_cores = true;      // basis conversion on the int8 tensor cores where it applies
  int ntt_split = 0;                  // log2(C) - floor(log2(N) / 2) of the R x C transform split
  // the same for the DGT's cyclic limb transforms (N/2 points): at N = 2^16
  // the 2^15-point transforms ran 2-3% faster with 256-point rows than with
  // the 128-point rows of split 0
  int dgt_split = 1;
  int ntt_cols_div = 0;               // column-pass tile width: widest >> div (0..2)
  int ntt_cols_kind = 0;              // column pass: 0 CTA-wide exchange, 1 warp-owned columns
  int ntt_rows_div = 1;               // row-pass tile height: tallest >> div (0..2)
  // transform ends fused with their neighbours (bit mask): 1 out-of-place
  // inverse instead of a copy, 2 key products in the special-limb forward
  // transform, 4 key-switch combine in the corrections' forward transform
  int fuse = 1;
  int batch_streams = 2;              // streams a large HMult batch is split over (1 or 2)
  // column pass: 16-column tiles by one tensor-map (TMA) load issued by one
  // thread instead of one bulk copy per tile row from every thread (+8% on
  // the forward transform at 2^16); 0 keeps the per-row copies
  int ntt_cols_tma = 1;
  // polls of a kernel's bounded mbarrier waits before it gives up, sets
  // kErrWaitTimeout in the error word and returns (aoa_ctx_sync then reports
  // AOA_ERR_TIMEOUT); the default 2^20 polls is far beyond any healthy wait
  int spin_limit = 1 << 20;
};

// Device copy of the basis-conversion / rescale constants.
struct RnsTables {
  // ModUp at level l (fast_conv_Q_to_B, manager.cu:180-223):
  //   modup_inv[l*k + i]          = (Q_l/q_i)^-1 mod q_i        (Shoup form)
  //   modup_hat[(l*k + i)*kl + j] = (Q_l/q_i) mod b_j
  ShoupW* modup_inv = nullptr;
  uint64_t* modup_hat = nullptr;
  // ModDown (fast_conv_B_to_Q, manager.cu:312-341):
  //   moddown_inv[j]         = ((B/b_j) mod b_j)^-1            (Shoup form)
  //   moddown_hat[j*k + i]   = (B/b_j) mod q_i
  //   moddown_binv[i]        = (B mod q_i)^-1                 (Shoup form)
  ShoupW* moddown_inv = nullptr;
  uint64_t* moddown_hat = nullptr;
  ShoupW* moddown_binv = nullptr;
  // Rescale (ckks_rescale, manager.cu:90-118): resc_inv[l*k + i] = q_l^-1 mod q_i
  ShoupW* resc_inv = nullptr;
  // B mod q_i for rho (manager.cu:149-160), Shoup form; zero on B primes
  ShoupW* bmodq = nullptr;
  // Tensor-core conversion images (k <= 32 and kl <= 32): for each table
  // (ModUp at level l, then ModDown) a 128 KiB byte matrix in the shared-memory
  // layout of the conversion's int8 MMA: [k-chunk 16][n 512][16 bytes], row
  // n = out*16 + d, byte k = in*8 + a holding byte (d - a) of the table entry.
  uint8_t* tc_modup = nullptr;     // [k][131072]
  uint8_t* tc_moddown = nullptr;   // [131072]
  uint8_t* tc_moddown_binv = nullptr;   // [131072], entries (B/b_j) B^-1 mod q_i (rescale modes)
};

struct Engine {
  int device = 0, num_sms = 148;
  int log_n = 0, log_c = 0;
  long N = 0;
  int k = 0, kl = 0, nprimes = 0;
  int scale_bits = 0;
  // butterfly kind per prime (kButterfly*): canonical, Harvey lazy (q <
  // 2^kLazyPrimeBits), or lazy with the remainder for q = 1 mod 2^32
  std::vector<char> prime_kind;
  int ntt_kind = kButterflyCanonical;   // the kind every prime shares, -1 when they differ
  std::vector<uint64_t> primes, gens;
  std::vector<PrimeConst> h_pc;
  PrimeConst* d_pc = nullptr;
  ShoupW* d_tw = nullptr;     // [nprimes][N]
  ShoupW* d_itw = nullptr;    // [nprimes][N]
  RnsTables rns;
  Tune tune;
  // Device error word: kernels OR in kErr* bits instead of trapping (a bounded
  // wait that expired, ...); aoa_ctx_sync reads and clears it.
  unsigned* d_err = nullptr;
  // Encoder tables: ksi[j] = exp(2 pi i j / M) for j <= M = 2N, as FP64 pairs
  // computed on the host; rot[j] = 5^j mod M for j < N/2.
  double2* d_ksi = nullptr;
  uint32_t* d_rot = nullptr;
  // DGT (folded Gaussian-integer transform of length N/2): cyclic merged
  // tables per prime, constants with N/2 inverses, and the twist by the
  // powers of a root r of i (r^(N/2) = i).  The twist tables hold r^n = c + di
  // (forward) and r^-n (inverse) for every n < N/2 in the form of a
  // three-product GI multiply, six planes [nprimes][6][N/2]: c, d - c, c + d
  // with their Shoup companions; they are built on the first DGT use
  // (dgt_twist_tables), so engines that never run a DGT do not hold them.
  std::vector<uint64_t> dgt_roots;   // 2 per prime (re, im of r)
  ShoupW* d_dtw = nullptr;
  ShoupW* d_ditw = nullptr;
  PrimeConst* d_dpc = nullptr;
  mutable std::mutex dgt_twist_mu;
  mutable uint64_t* d_twist = nullptr;
  mutable uint64_t* d_untwist = nullptr;
  mutable std::vector<void*> allocations;
};

struct Ctx {
  Engine* E = nullptr;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  void* scratch = nullptr;      // key-switch workspace (stream-ordered allocation)
  size_t scratch_bytes = 0;
  void* plain = nullptr;        // workspace of the reference-structured per-call path
  size_t plain_bytes = 0;
  void* batch = nullptr;        // workspace of batched HMult
  size_t batch_bytes = 0;
  void* conv = nullptr;         // domain-conversion buffer for downloads
  size_t conv_bytes = 0;
  void* enc = nullptr;          // encoder / key generation buffer
  size_t enc_bytes = 0;
  // second stream of the context: a large HMult batch runs as two halves on
  // `stream` and `aux`, forked and joined by events (each half its own workspace)
  cudaStream_t aux = nullptr;
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  void* batch2 = nullptr;
  size_t batch2_bytes = 0;
  int transform = AOA_NTT;      // transform domain of this context's evaluations (AOA_NTT / AOA_DGT)
};

// Per-launch pointer lists for batched kernels (passed by value).
constexpr int kMaxBatch = 64;
struct CtPtrs {
  const uint64_t* a[kMaxBatch];
  const uint64_t* b[kMaxBatch];
};
struct OutPtrs {
  uint64_t* p[2 * kMaxBatch];
};
// per-op Galois elements and switching keys of a batched automorphism
struct GaloisList {
  long g[kMaxBatch];
};
struct KeyPtrs {
  const uint64_t* k[kMaxBatch];
};

// count of kernel launches issued by this library (engine.cu)
void note_launch();

// C-ABI error plumbing (engine.cu)
int fail(int status, const std::string& msg);

template <class F>
int guarded(F&& f) {
  try {
    f();
    return AOA_OK;
  } catch (const AoaError& e) {
    return fail(e.status, e.what());
  } catch (const std::bad_alloc&) {
    return fail(AOA_ERR_OOM, "host allocation failed");
  } catch (const std::exception& e) {
    return fail(AOA_ERR_BAD_PARAM, e.what());
  }
}

// ntt.cu
// A family of limb transforms: merged Cooley-Tukey tables ([nprimes][2^log_n]
// forward / inverse with Shoup companions) and per-prime constants.
struct NttTables {
  const ShoupW* tw = nullptr;
  const ShoupW* itw = nullptr;
  const PrimeConst* pc = nullptr;
  int log_n = 0;
  int prime_shift = 0;     // limb l uses prime first + (l >> prime_shift)
  int kind = kButterflyCanonical;   // butterfly kind of every limb
  int split = 0;                     // log2(C) - floor(log2(n) / 2) of the R x C split
  // per prime butterfly kind, when the primes' kinds differ: the limbs run in
  // runs of one kind
  const char* prime_kind = nullptr;
};
// Fused ends of a limb transform.  NttIo::src: the first pass reads item
// (p, l) from src + p * src_poly_stride + l * N instead of the data (an
// out-of-place transform; the data is written).  NttIo::epi: what the last
// pass of a FORWARD transform does with the finished value v of coefficient c
// of item (p, l) under prime pr (p counts from the first poly of the call):
//   kEpiStore       data = v
//   kEpiKeyProduct  out + p*out_stride + l*N       = v * key[pr]           (b part)
//                   (same) + out_poly1             = v * key[key_half + pr] (a part)
//                   (the data is not written)
//   kEpiCombine     the key-switch epilogue with y = v (ks_combine):
//                   rescale: ((base + ks B^-1 - v) q_l^-1), else base + (ks - v) B^-1,
//                   base = 0 for p >= base_polys; written to outp.p[p] (use_ptrs)
//                   or out + p*out_stride, at l*N + c
enum { kEpiStore = 0, kEpiKeyProduct = 1, kEpiCombine = 2 };
enum { kFuseSource = 1, kFuseKeyProduct = 2, kFuseCombine = 4 };
struct NttEpi {
  int mode = kEpiStore;
  uint64_t* out = nullptr;
  long out_stride = 0, out_poly1 = 0;
  const uint64_t* key = nullptr;
  long key_half = 0;
  const uint64_t* base = nullptr;
  long base_stride = 0;
  int base_polys = 0;
  const uint64_t* ks = nullptr;
  long ks_stride = 0;
  const ShoupW* binv = nullptr;
  const ShoupW* resc = nullptr;
  int use_ptrs = 0;
  OutPtrs outp;
  int limb_base = 0;       // limb of the launch's first limb in out / ks / base
};
struct NttIo {
  const uint64_t* src = nullptr;
  long src_poly_stride = 0;
  NttEpi epi;
};
void ntt_init(Engine& E);
void ntt_batch_io(const Engine& E, uint64_t* data, int npolys, int first_prime, int nlimbs, long poly_stride,
                  bool forward, const NttIo& io, cudaStream_t st);
void ntt_batch_tables(const Engine& E, const NttTables& T, uint64_t* data, int npolys, int first_prime, int nlimbs,
                      long poly_stride, bool forward, cudaStream_t st, const NttIo* io = nullptr);
void ntt_batch(const Engine& E, uint64_t* data, int npolys, int first_prime, int nlimbs,
               long poly_stride, bool forward, cudaStream_t st);

// rns.cu
void rns_init(Engine& E);
void modup(const Engine& E, const uint64_t* in, long in_stride, uint64_t* out_b, long out_stride,
           int npolys, int level, cudaStream_t st);
void moddown(const Engine& E, const uint64_t* in_q, const uint64_t* in_b, long in_stride, uint64_t* out,
             long out_stride, int npolys, int level, cudaStream_t st);
void rescale(const Engine& E, uint64_t* d, long poly_stride, int npolys, int level, cudaStream_t st);
void moddown_conv(const Engine& E, const uint64_t* in_b, long in_stride, uint64_t* out, long out_stride,
                  int npolys, int nout, cudaStream_t st);
void rescale_corrections(const Engine& E, const uint64_t* in_b, long in_stride, const uint64_t* u_l,
                         long u_stride, uint64_t* cl_tmp, long cl_stride, uint64_t* y, long y_stride, int npolys,
                         int level, cudaStream_t st);
void ks_combine(const Engine& E, uint64_t* out, long out_stride, const uint64_t* base, long base_stride,
                const uint64_t* k, long k_stride, const uint64_t* y, long y_stride, int nlimbs, int npolys,
                int rescale_level, cudaStream_t st, int prime0 = 0);

// dgt.cu: folded Gaussian-integer transform.  A GI limb is N words: the
// real plane (N/2) then the imaginary plane (N/2), which is also the
// coefficient layout of the unfolded polynomial (a_j, a_{j+N/2}).
void dgt_init(Engine& E, const uint64_t* roots);
void dgt_batch(const Engine& E, uint64_t* data, int npolys, int first_prime, int nlimbs, long poly_stride,
               bool forward, cudaStream_t st);
void gi_mul_op(const Engine& E, uint64_t* c, long cs, const uint64_t* a, long as, const uint64_t* b, long bs,
               int prime0, int nlimbs, int npolys, cudaStream_t st);
void gi_tensor_op(const Engine& E, const uint64_t* a, long a_half, const uint64_t* b, long b_half, uint64_t* d0,
                  uint64_t* d1, uint64_t* d2, int nlimbs, cudaStream_t st);
void gi_keyswitch_mul_op(const Engine& E, const uint64_t* xq, const uint64_t* xb, const uint64_t* key, uint64_t* k0,
                         uint64_t* k1, int nq, cudaStream_t st);
// the same over a batch of n ops (one launch each)
void gi_tensor_batch_op(const Engine& E, const CtPtrs& ptr, long half, uint64_t* D, int n, int nlimbs,
                        cudaStream_t st);
void gi_keyswitch_mul_batch_op(const Engine& E, const uint64_t* xq, long xq_stride, const uint64_t* xb,
                               long xb_stride, const uint64_t* key, uint64_t* k, long k_stride, int n, int nq,
                               cudaStream_t st);
// ckks.cu: limb transforms of a kind (AOA_NTT / AOA_DGT) and domain changes
void xform(const Engine& E, int kind, uint64_t* d, int npolys, int first_prime, int nlimbs, long stride, bool fwd,
           cudaStream_t st);

// ops.cu  (op: 0 add, 1 sub, 2 mul, 3 neg)
void ew_binary_op(const Engine& E, uint64_t* c, long cs, const uint64_t* a, long as, const uint64_t* b, long bs,
                  int op, int prime0, int nlimbs, int npolys, cudaStream_t st);
void ew_scalar_op(const Engine& E, uint64_t* c, long cs, const uint64_t* a, long as, const uint64_t* d_scalars,
                  int op, int prime0, int nlimbs, int npolys, cudaStream_t st);
void ew_muladd_op(const Engine& E, uint64_t* d, long ds, const uint64_t* a, long as, const uint64_t* b, long bs,
                  const uint64_t* c, long cs, int prime0, int nlimbs, int npolys, cudaStream_t st);
void tensor_op(const Engine& E, const uint64_t* a, long a_half, const uint64_t* b, long b_half, uint64_t* d0,
               uint64_t* d1, uint64_t* d2, int nlimbs, cudaStream_t st);
void tensor_batch_op(const Engine& E, const CtPtrs& ptr, long half, uint64_t* D, int n, int nlimbs, cudaStream_t st);
void keyswitch_mul_batch_op(const Engine& E, const uint64_t* xq, long xq_stride, const uint64_t* xb, long xb_stride,
                            const uint64_t* key, uint64_t* k, long k_stride, int n, int nq, cudaStream_t st, int nb = -1);
void ks_combine_ptr(const Engine& E, const OutPtrs& outp, const uint64_t* base, long base_stride, const uint64_t* k,
                    long k_stride, const uint64_t* y, long y_stride, int nlimbs, int npolys, int rescale_level,
                    cudaStream_t st, int base_polys = -1);
void automorph_ntt_batch_op(const Engine& E, const CtPtrs& ptr, long half, uint64_t* out, int n,
                            const GaloisList& galois, int nlimbs, cudaStream_t st);
// key products with a key per op (keys.k[z], [b | a] over all primes)
void keyswitch_mul_keys_op(const Engine& E, const uint64_t* xq, long xq_stride, const uint64_t* xb, long xb_stride,
                           const KeyPtrs& keys, uint64_t* k, long k_stride, int n, int nq, cudaStream_t st);
void keyswitch_mul_op(const Engine& E, const uint64_t* xq, const uint64_t* xb, const uint64_t* key, uint64_t* k0,
                      uint64_t* k1, int nq, cudaStream_t st, int nb = -1);
void automorph_coef_op(const Engine& E, uint64_t* out, const uint64_t* in, long poly_stride, long galois,
                       int nlimbs, int npolys, cudaStream_t st);
void automorph_ntt_op(const Engine& E, uint64_t* out, const uint64_t* in, long poly_stride, long galois,
                      int nlimbs, int npolys, cudaStream_t st);

// host number theory (primes.cpp)
uint64_t h_mulmod(uint64_t a, uint64_t b, uint64_t q);
uint64_t h_powmod(uint64_t a, uint64_t e, uint64_t q);
uint64_t h_invmod(uint64_t a, uint64_t q);
bool h_is_prime(uint64_t n);
uint64_t h_smallest_primitive_root(uint64_t q);
uint64_t h_shoup_companion(uint64_t w, uint64_t q);
int h_search_primes(int bits, uint64_t modulus, int count, uint64_t* out);

}  // namespace aoa

// Ciphertext (cipher_t, aoa-ntt include/newckks/ckks/cipher_t.h:17-22):
// d = [c0 | c1], each k limbs of N words.
struct aoa_ct {
  uint64_t* d = nullptr;
  int level = 0;
  int slots = 0;
  uint64_t scale = 0;
  int domain = AOA_COEF;
};

// Switching key (SwitchKey, aoa-ntt include/newckks/defines.h:85-90):
// d = [b | a], each k + kl limbs, in the transform domain `domain`.
struct aoa_swk {
  uint64_t* d = nullptr;
  int domain = AOA_NTT;     // AOA_NTT or AOA_DGT
};

struct aoa_engine { aoa::Engine e; };
struct aoa_ctx { aoa::Ctx c; };
