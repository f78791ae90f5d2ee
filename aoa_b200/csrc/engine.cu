// Engine set-up (prime tables, transform twiddles, RNS constants) and the core
// of the C ABI declared in include/aoa_ckks.h.
#include <cstring>
#include <atomic>
#include <mutex>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "aoa_internal.h"
#include "async.cuh"

namespace aoa {

// One warp; thread 0 waits on a barrier that expects one arrival which
// nothing makes, with `spins` polls, and records the expiry like every other
// bounded wait of the engine (no copy or MMA targets the barrier, so nothing
// is in flight when the kernel returns).
__global__ void wait_check_kernel(unsigned* err, int spins) {
  __shared__ __align__(8) uint64_t mb;
  if (threadIdx.x == 0) {
    mbar_init(&mb, 1);
    mbar_init_fence();
  }
  __syncwarp();
  if (threadIdx.x == 0 && !mbar_wait(&mb, 0, spins)) atomicOr(err, kErrWaitTimeout);
}

static thread_local std::string g_last_error;
static std::atomic<long> g_launches{0};

void note_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }

int fail(int status, const std::string& msg) {
  g_last_error = msg;
  return status;
}

static long bitrev(uint32_t x, int bits) {
  uint32_t r = 0;
  for (int i = 0; i < bits; i++) r |= ((x >> i) & 1u) << (bits - 1 - i);
  return (long)r;
}

template <class T>
static T* dev_upload(Engine& E, const std::vector<T>& h) {
  T* d = nullptr;
  AOA_CUDA(cudaMalloc(&d, std::max<size_t>(1, h.size()) * sizeof(T)));
  E.allocations.push_back(d);
  if (!h.empty()) AOA_CUDA(cudaMemcpy(d, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice));
  return d;
}

static uint64_t neg_inv_2_64(uint64_t q) {   // -q^-1 mod 2^64 (Newton)
  uint64_t x = q;                           // correct to 3 bits for odd q
  for (int i = 0; i < 6; i++) x *= 2 - q * x;
  return (uint64_t)0 - x;
}

static void build_prime_tables(Engine& E) {
  const long N = E.N;
  const int np = E.nprimes;
  E.h_pc.resize(np);
  std::vector<ShoupW> tw((size_t)np * N), itw((size_t)np * N);
  bool bad = false;
#pragma omp parallel for schedule(dynamic)
  for (int p = 0; p < np; p++) {
    const uint64_t q = E.primes[p];
    if ((q - 1) % (2 * (uint64_t)N) != 0 || !h_is_prime(q)) { bad = true; continue; }
    const uint64_t g = E.gens[p];
    const uint64_t psi = h_powmod(g, (q - 1) / (2 * (uint64_t)N), q);
    const uint64_t ipsi = h_invmod(psi, q);
    uint64_t pw = 1, ipw = 1;
    for (long i = 0; i < N; i++) {       // psi^i, scattered to bit-reversed slots
      const long r = bitrev((uint32_t)i, E.log_n);
      tw[(size_t)p * N + r] = ShoupW{pw, h_shoup_companion(pw, q)};
      itw[(size_t)p * N + r] = ShoupW{ipw, h_shoup_companion(ipw, q)};
      pw = h_mulmod(pw, psi, q);
      ipw = h_mulmod(ipw, ipsi, q);
    }
    PrimeConst c;
    c.q = q;
    c.qinv_neg = neg_inv_2_64(q);
    unsigned __int128 one128 = 1;
    c.r1 = (uint64_t)((one128 << 64) % q);
    c.r2 = h_mulmod(c.r1, c.r1, q);
    c.r1_sh = h_shoup_companion(c.r1, q);
    c.one_sh = (uint64_t)((one128 << 64) / q);
    c.ninv = h_invmod((uint64_t)N % q, q);
    c.ninv_sh = h_shoup_companion(c.ninv, q);
    c.ninv_w1 = h_mulmod(c.ninv, itw[(size_t)p * N + 1].w, q);
    c.ninv_w1_sh = h_shoup_companion(c.ninv_w1, q);
    c.bar_sh = 0;
    c.bar_mu = 0;
    if (q >= (1ull << 33) && q < (1ull << 62)) {
      const int n = 64 - __builtin_clzll(q);
      c.bar_sh = (uint64_t)(n - 2);
      c.bar_mu = (uint64_t)((one128 << (64 + n - 2)) / q);
    }
    E.h_pc[p] = c;
  }
  if (bad) throw AoaError(AOA_ERR_BAD_PARAM, "every prime must be prime, < 2^63 and = 1 mod 2N");
  E.d_pc = dev_upload(E, E.h_pc);
  E.d_tw = dev_upload(E, tw);
  E.d_itw = dev_upload(E, itw);
  E.d_err = dev_upload(E, std::vector<unsigned>(1, 0u));
}

// Encoder tables (the reference computes them on the host per call,
// aoa-ntt src/ckks/encoder.cu:33-124).  ksi[j] = (cos(2 pi j / M), sin(2 pi j / M))
// with M = 2N, evaluated by the host libm exactly as written so that the
// device FFT uses the same doubles; rot[j] = 5^j mod M.
static void build_encoder_tables(Engine& E) {
  const long M = 2 * E.N;
  std::vector<double2> ksi(M + 1);
  for (long j = 0; j < M; ++j) {
    const double angle = 2.0 * M_PI * j / M;
    ksi[j] = make_double2(cos(angle), sin(angle));
  }
  ksi[M] = ksi[0];
  std::vector<uint32_t> rot(std::max<long>(1, E.N / 2));
  uint64_t v = 1;
  for (long j = 0; j < E.N / 2; ++j) {
    rot[j] = (uint32_t)v;
    v = (v * 5) % (uint64_t)M;
  }
  E.d_ksi = dev_upload(E, ksi);
  E.d_rot = dev_upload(E, rot);
}

// Basis-conversion and rescale constants (manager.cu:566-759).
static void build_rns_tables(Engine& E) {
  const int k = E.k, kl = E.kl;
  const std::vector<uint64_t>& P = E.primes;
  auto sh = [](uint64_t w, uint64_t q) { return ShoupW{w, h_shoup_companion(w, q)}; };
  std::vector<ShoupW> modup_inv((size_t)k * k, ShoupW{0, 0});
  std::vector<uint64_t> modup_hat((size_t)k * k * std::max(kl, 1), 0);
  for (int l = 0; l < k; l++) {
    for (int i = 0; i <= l; i++) {
      const uint64_t qi = P[i];
      uint64_t hat = 1;                               // (Q_l / q_i) mod q_i
      for (int t = 0; t <= l; t++)
        if (t != i) hat = h_mulmod(hat, P[t] % qi, qi);
      modup_inv[(size_t)l * k + i] = sh(h_invmod(hat, qi), qi);
      for (int j = 0; j < kl; j++) {
        const uint64_t bj = P[k + j];
        uint64_t hb = 1;                              // (Q_l / q_i) mod b_j
        for (int t = 0; t <= l; t++)
          if (t != i) hb = h_mulmod(hb, P[t] % bj, bj);
        modup_hat[((size_t)l * k + i) * kl + j] = hb;
      }
    }
  }
  std::vector<ShoupW> moddown_inv(std::max(kl, 1), ShoupW{0, 0}), moddown_binv(k);
  std::vector<uint64_t> moddown_hat((size_t)std::max(kl, 1) * k, 0);
  for (int j = 0; j < kl; j++) {
    const uint64_t bj = P[k + j];
    uint64_t hat = 1;                                 // (B / b_j) mod b_j
    for (int t = 0; t < kl; t++)
      if (t != j) hat = h_mulmod(hat, P[k + t] % bj, bj);
    moddown_inv[j] = sh(h_invmod(hat, bj), bj);
    for (int i = 0; i < k; i++) {
      const uint64_t qi = P[i];
      uint64_t hq = 1;                                // (B / b_j) mod q_i
      for (int t = 0; t < kl; t++)
        if (t != j) hq = h_mulmod(hq, P[k + t] % qi, qi);
      moddown_hat[(size_t)j * k + i] = hq;
    }
  }
  std::vector<ShoupW> bmodq(E.nprimes, ShoupW{0, 0});
  for (int i = 0; i < k; i++) {
    const uint64_t qi = P[i];
    uint64_t b = 1;
    for (int t = 0; t < kl; t++) b = h_mulmod(b, P[k + t] % qi, qi);
    bmodq[i] = sh(b, qi);
    moddown_binv[i] = kl ? sh(h_invmod(b, qi), qi) : sh(1, qi);
  }
  std::vector<ShoupW> resc((size_t)k * k, ShoupW{0, 0});
  for (int l = 1; l < k; l++)
    for (int i = 0; i < l; i++) resc[(size_t)l * k + i] = sh(h_invmod(P[l] % P[i], P[i]), P[i]);
  if (k <= 32 && kl >= 1 && kl <= 32 && E.N % 128 == 0) {
    // [16 k-chunks][256 columns][16 B]: byte k = 8 in + a of column n = 8 out + b
    // holds byte b of h 2^(8a) mod p_out (the conversion kernel's B operand)
    constexpr size_t kImg = 65536;
    auto image = [](const uint64_t* mat, int ld, int nin, int nout, const uint64_t* outp, uint8_t* img) {
      for (int out = 0; out < nout; out++) {
        const uint64_t p = outp[out];
        uint64_t sh[8];
        sh[0] = 1 % p;
        for (int a = 1; a < 8; a++) sh[a] = h_mulmod(sh[a - 1], 256 % p, p);
        for (int in = 0; in < nin; in++) {
          const uint64_t h = mat[(size_t)in * ld + out] % p;
          for (int a = 0; a < 8; a++) {
            const uint64_t g = h_mulmod(h, sh[a], p);
            for (int b = 0; b < 8; b++) {
              const int kb = in * 8 + a, n = out * 8 + b;
              img[((size_t)(kb / 16) * 256 + n) * 16 + kb % 16] = (uint8_t)(g >> (8 * b));
            }
          }
        }
      }
    };
    std::vector<uint8_t> up((size_t)k * kImg, 0), down(kImg, 0), down_binv(kImg, 0);
    for (int l = 0; l < k; l++)
      image(modup_hat.data() + (size_t)l * k * kl, kl, l + 1, kl, P.data() + k, up.data() + l * kImg);
    image(moddown_hat.data(), k, kl, k, P.data(), down.data());
    // the rescale modes scale the conversion by B^-1 mod q_i: fold it into the table
    std::vector<uint64_t> hat_binv(moddown_hat.size());
    for (int j = 0; j < kl; j++)
      for (int i = 0; i < k; i++)
        hat_binv[(size_t)j * k + i] = h_mulmod(moddown_hat[(size_t)j * k + i], moddown_binv[i].w, P[i]);
    image(hat_binv.data(), k, kl, k, P.data(), down_binv.data());
    E.rns.tc_modup = dev_upload(E, up);
    E.rns.tc_moddown = dev_upload(E, down);
    E.rns.tc_moddown_binv = dev_upload(E, down_binv);
  }
  E.rns.modup_inv = dev_upload(E, modup_inv);
  E.rns.modup_hat = dev_upload(E, modup_hat);
  E.rns.moddown_inv = dev_upload(E, moddown_inv);
  E.rns.moddown_hat = dev_upload(E, moddown_hat);
  E.rns.moddown_binv = dev_upload(E, moddown_binv);
  E.rns.resc_inv = dev_upload(E, resc);
  E.rns.bmodq = dev_upload(E, bmodq);
}

}  // namespace aoa

using namespace aoa;

extern "C" {

const char* aoa_last_error(void) { return g_last_error.c_str(); }

long aoa_kernel_launches(void) { return g_launches.load(); }

const char* aoa_status_string(int s) {
  switch (s) {
    case AOA_OK: return "ok";
    case AOA_ERR_BAD_PARAM: return "bad parameter";
    case AOA_ERR_LEVEL_EXHAUSTED: return "level exhausted";
    case AOA_ERR_NO_KEY: return "missing key";
    case AOA_ERR_OOM: return "out of memory";
    case AOA_ERR_CUDA: return "cuda error";
    case AOA_ERR_TIMEOUT: return "timeout";
    case AOA_ERR_SLOT_MISMATCH: return "slot mismatch";
    case AOA_ERR_NOT_INITIALIZED: return "not initialized";
    case AOA_ERR_NO_DEVICE: return "no cuda device";
    default: return "unknown";
  }
}

int aoa_engine_create(const aoa_params* p, aoa_engine** out) {
  if (!p || !out) return fail(AOA_ERR_BAD_PARAM, "null argument");
  *out = nullptr;
  aoa_engine* h = new aoa_engine();
  int st = guarded([&] {
    Engine& E = h->e;
    if (p->log_n < 10 || p->log_n > 17) throw AoaError(AOA_ERR_BAD_PARAM, "log_n must be in [10, 17]");
    if (p->k < 1 || p->kl < 0 || p->k + p->kl > 512 || !p->primes)
      throw AoaError(AOA_ERR_BAD_PARAM, "need k >= 1, kl >= 0 and a prime list");
    if (p->dnum != 0 && p->dnum != 1) throw AoaError(AOA_ERR_BAD_PARAM, "only dnum = 1 is supported");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
      throw AoaError(AOA_ERR_NO_DEVICE, "no CUDA device visible");
    AOA_CUDA(cudaGetDevice(&E.device));
    {   // keep stream-ordered allocations cached across synchronisations
      cudaMemPool_t pool;
      AOA_CUDA(cudaDeviceGetDefaultMemPool(&pool, E.device));
      uint64_t keep = ~0ull;
      AOA_CUDA(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep));
    }
    E.log_n = p->log_n;
    E.N = 1L << p->log_n;
    E.log_c = p->log_n / 2;
    E.k = p->k;
    E.kl = p->kl;
    E.nprimes = p->k + p->kl;
    E.scale_bits = p->scale_bits;
    E.primes.assign(p->primes, p->primes + E.nprimes);
    for (uint64_t q : E.primes)
      if (q >= (1ull << 63) || q < 3) throw AoaError(AOA_ERR_BAD_PARAM, "primes must be odd and < 2^63");
    for (int i = 0; i < E.nprimes; i++)
      for (int j = 0; j < i; j++)
        if (E.primes[i] == E.primes[j]) throw AoaError(AOA_ERR_BAD_PARAM, "primes must be distinct");
    E.prime_kind.clear();
    for (uint64_t q : E.primes) {
      const int kind = q >= (1ull << kLazyPrimeBits) ? kButterflyCanonical
                       : (q & 0xffffffffull) == 1 ? kButterflyLazyQ1 : kButterflyLazy;
      E.prime_kind.push_back((char)kind);
    }
    E.ntt_kind = E.prime_kind[0];
    for (char kind : E.prime_kind)
      if (kind != E.ntt_kind) E.ntt_kind = -1;
    E.gens.resize(E.nprimes);
    for (int i = 0; i < E.nprimes; i++)
      E.gens[i] = p->generators ? p->generators[i] : h_smallest_primitive_root(E.primes[i]);
    build_prime_tables(E);
    build_rns_tables(E);
    build_encoder_tables(E);
    dgt_init(E, p->dgt_roots);
    rns_init(E);
    ntt_init(E);
    AOA_CUDA(cudaDeviceSynchronize());
  });
  if (st != AOA_OK) {
    for (void* a : h->e.allocations) cudaFree(a);
    delete h;
    return st;
  }
  *out = h;
  return AOA_OK;
}

int aoa_engine_destroy(aoa_engine* h) {
  if (!h) return AOA_OK;
  int st = guarded([&] {
    AOA_CUDA(cudaDeviceSynchronize());
    for (void* a : h->e.allocations) AOA_CUDA(cudaFree(a));
  });
  delete h;
  return st;
}

// Launch-shape knobs of the engine's kernels (the reference fixes its kernel
// shapes at compile time); names, ranges and defaults in include/aoa_ckks.h.
// Set before the engine is used from several streams at once.
int aoa_engine_tune(aoa_engine* h, const char* knob, double value) {
  if (!h || !knob) return fail(AOA_ERR_BAD_PARAM, "null argument");
  const std::string k(knob);
  if (k == "ntt_chunk_bytes" && value >= (1 << 20) && value <= 6.4e10) h->e.tune.ntt_chunk_bytes = (long)value;
  else if (k == "ntt_waves" && value > 0 && value <= 64) h->e.tune.ntt_waves = value;
  else if (k == "ntt_waves_large" && value > 0 && value <= 64) h->e.tune.ntt_waves_large = value;
  else if (k == "conv_tensor_cores" && (value == 0 || value == 1)) h->e.tune.conv_tensor_cores = value != 0;
  else if (k == "ntt_split" && value >= -2 && value <= 2 && value == (int)value) h->e.tune.ntt_split = (int)value;
  else if (k == "dgt_split" && value >= -2 && value <= 2 && value == (int)value) h->e.tune.dgt_split = (int)value;
  else if (k == "ntt_cols_div" && value >= 0 && value <= 2 && value == (int)value) h->e.tune.ntt_cols_div = (int)value;
  else if (k == "ntt_rows_div" && value >= 0 && value <= 2 && value == (int)value) h->e.tune.ntt_rows_div = (int)value;
  else if (k == "ntt_cols_kind" && (value == 0 || value == 1)) h->e.tune.ntt_cols_kind = (int)value;
  else if (k == "batch_streams" && (value == 1 || value == 2)) h->e.tune.batch_streams = (int)value;
  else if (k == "fuse" && value >= 0 && value <= 7 && value == (int)value) h->e.tune.fuse = (int)value;
  else if (k == "ntt_cols_tma" && (value == 0 || value == 1)) h->e.tune.ntt_cols_tma = (int)value;
  else if (k == "spin_limit" && value >= 0 && value <= (1 << 30) && value == (int)value)
    h->e.tune.spin_limit = (int)value;
  else return fail(AOA_ERR_BAD_PARAM, "unknown knob or value out of range: " + k);
  return AOA_OK;
}

int aoa_engine_tune_get(const aoa_engine* h, const char* knob, double* value) {
  if (!h || !knob || !value) return fail(AOA_ERR_BAD_PARAM, "null argument");
  const std::string k(knob);
  const Tune& t = h->e.tune;
  if (k == "ntt_chunk_bytes") *value = (double)t.ntt_chunk_bytes;
  else if (k == "ntt_waves") *value = t.ntt_waves;
  else if (k == "ntt_waves_large") *value = t.ntt_waves_large;
  else if (k == "conv_tensor_cores") *value = t.conv_tensor_cores ? 1 : 0;
  else if (k == "ntt_split") *value = t.ntt_split;
  else if (k == "dgt_split") *value = t.dgt_split;
  else if (k == "ntt_cols_div") *value = t.ntt_cols_div;
  else if (k == "ntt_rows_div") *value = t.ntt_rows_div;
  else if (k == "ntt_cols_kind") *value = t.ntt_cols_kind;
  else if (k == "batch_streams") *value = t.batch_streams;
  else if (k == "fuse") *value = t.fuse;
  else if (k == "spin_limit") *value = t.spin_limit;
  else if (k == "ntt_cols_tma") *value = t.ntt_cols_tma;
  else return fail(AOA_ERR_BAD_PARAM, "unknown knob: " + k);
  return AOA_OK;
}

int aoa_engine_info(const aoa_engine* h, int* log_n, int* k, int* kl, uint64_t* primes_out) {
  if (!h) return fail(AOA_ERR_BAD_PARAM, "null engine");
  if (log_n) *log_n = h->e.log_n;
  if (k) *k = h->e.k;
  if (kl) *kl = h->e.kl;
  if (primes_out) std::memcpy(primes_out, h->e.primes.data(), h->e.primes.size() * sizeof(uint64_t));
  return AOA_OK;
}

int aoa_ctx_create(aoa_engine* e, void* stream, aoa_ctx** out) {
  if (!e || !out) return fail(AOA_ERR_BAD_PARAM, "null argument");
  aoa_ctx* h = new aoa_ctx();
  int st = guarded([&] {
    h->c.E = &e->e;
    if (stream) {
      h->c.stream = (cudaStream_t)stream;
    } else {
      AOA_CUDA(cudaStreamCreateWithFlags(&h->c.stream, cudaStreamNonBlocking));
      h->c.own_stream = true;
    }
  });
  if (st != AOA_OK) { delete h; return st; }
  *out = h;
  return AOA_OK;
}

int aoa_ctx_destroy(aoa_ctx* h) {
  if (!h) return AOA_OK;
  int st = guarded([&] {
    if (h->c.scratch) AOA_CUDA(cudaFreeAsync(h->c.scratch, h->c.stream));
    if (h->c.plain) AOA_CUDA(cudaFreeAsync(h->c.plain, h->c.stream));
    if (h->c.batch) AOA_CUDA(cudaFreeAsync(h->c.batch, h->c.stream));
    if (h->c.conv) AOA_CUDA(cudaFreeAsync(h->c.conv, h->c.stream));
    if (h->c.enc) AOA_CUDA(cudaFreeAsync(h->c.enc, h->c.stream));
    if (h->c.aux) {
      if (h->c.batch2) AOA_CUDA(cudaFreeAsync(h->c.batch2, h->c.aux));
      AOA_CUDA(cudaStreamSynchronize(h->c.aux));
      AOA_CUDA(cudaStreamDestroy(h->c.aux));
      AOA_CUDA(cudaEventDestroy(h->c.ev_fork));
      AOA_CUDA(cudaEventDestroy(h->c.ev_join));
    }
    AOA_CUDA(cudaStreamSynchronize(h->c.stream));
    if (h->c.own_stream) AOA_CUDA(cudaStreamDestroy(h->c.stream));
  });
  delete h;
  return st;
}

int aoa_ctx_wait_check(aoa_ctx* h, int spins) {
  if (!h || spins < 0) return fail(AOA_ERR_BAD_PARAM, "bad argument");
  return guarded([&] {
    wait_check_kernel<<<1, 32, 0, h->c.stream>>>(h->c.E->d_err, spins);
    AOA_CHECK_LAUNCH();
    note_launch();
  });
}

int aoa_ctx_sync(aoa_ctx* h) {
  if (!h) return fail(AOA_ERR_BAD_PARAM, "null context");
  return guarded([&] {
    AOA_CUDA(cudaStreamSynchronize(h->c.stream));
    unsigned err = 0;
    AOA_CUDA(cudaMemcpy(&err, h->c.E->d_err, sizeof(err), cudaMemcpyDeviceToHost));
    if (err) {
      AOA_CUDA(cudaMemset(h->c.E->d_err, 0, sizeof(unsigned)));
      throw AoaError(AOA_ERR_TIMEOUT, "a device-side bounded wait expired (error bits 0x" + std::to_string(err) +
                                          "); the affected results are invalid");
    }
  });
}

int aoa_ctx_stream(aoa_ctx* h, void** s) {
  if (!h || !s) return fail(AOA_ERR_BAD_PARAM, "null argument");
  *s = (void*)h->c.stream;
  return AOA_OK;
}

int aoa_device_alloc(aoa_ctx* h, size_t bytes, void** out) {
  if (!h || !out) return fail(AOA_ERR_BAD_PARAM, "null argument");
  return guarded([&] {
    cudaError_t e = cudaMallocAsync(out, bytes, h->c.stream);
    if (e != cudaSuccess) {
      cudaGetLastError();
      throw AoaError(e == cudaErrorMemoryAllocation ? AOA_ERR_OOM : AOA_ERR_CUDA, cudaGetErrorString(e));
    }
  });
}

int aoa_device_free(aoa_ctx* h, void* p) {
  if (!h) return fail(AOA_ERR_BAD_PARAM, "null context");
  return guarded([&] { AOA_CUDA(cudaFreeAsync(p, h->c.stream)); });
}

int aoa_search_primes(int bits, uint64_t modulus, int count, uint64_t* out) {
  if (!out || count < 0) return fail(AOA_ERR_BAD_PARAM, "bad argument");
  return h_search_primes(bits, modulus, count, out);
}

uint64_t aoa_primitive_root(uint64_t q) { return h_is_prime(q) ? h_smallest_primitive_root(q) : 0; }

int aoa_host_alloc(size_t bytes, void** out) {
  if (!out) return fail(AOA_ERR_BAD_PARAM, "null argument");
  return guarded([&] {
    cudaError_t e = cudaHostAlloc(out, bytes, cudaHostAllocDefault);
    if (e != cudaSuccess) {
      cudaGetLastError();
      throw AoaError(AOA_ERR_OOM, std::string("pinned host allocation failed: ") + cudaGetErrorString(e));
    }
  });
}

int aoa_host_free(void* p) {
  return guarded([&] { AOA_CUDA(cudaFreeHost(p)); });
}

int aoa_memcpy_h2d(aoa_ctx* h, void* dst, const void* src, size_t n) {
  if (!h) return fail(AOA_ERR_BAD_PARAM, "null context");
  return guarded([&] { AOA_CUDA(cudaMemcpyAsync(dst, src, n, cudaMemcpyHostToDevice, h->c.stream)); });
}

int aoa_memcpy_d2h(aoa_ctx* h, void* dst, const void* src, size_t n) {
  if (!h) return fail(AOA_ERR_BAD_PARAM, "null context");
  return guarded([&] { AOA_CUDA(cudaMemcpyAsync(dst, src, n, cudaMemcpyDeviceToHost, h->c.stream)); });
}

int aoa_memcpy_d2d(aoa_ctx* h, void* dst, const void* src, size_t n) {
  if (!h) return fail(AOA_ERR_BAD_PARAM, "null context");
  return guarded([&] { AOA_CUDA(cudaMemcpyAsync(dst, src, n, cudaMemcpyDeviceToDevice, h->c.stream)); });
}

int aoa_ntt_fwd(aoa_ctx* h, uint64_t* d, int npolys, int first, int nlimbs, int stride) {
  if (!h || !d) return fail(AOA_ERR_BAD_PARAM, "null argument");
  return guarded([&] {
    if (stride < nlimbs) throw AoaError(AOA_ERR_BAD_PARAM, "poly_stride < nlimbs");
    ntt_batch(*h->c.E, d, npolys, first, nlimbs, stride, true, h->c.stream);
  });
}

int aoa_ntt_inv(aoa_ctx* h, uint64_t* d, int npolys, int first, int nlimbs, int stride) {
  if (!h || !d) return fail(AOA_ERR_BAD_PARAM, "null argument");
  return guarded([&] {
    if (stride < nlimbs) throw AoaError(AOA_ERR_BAD_PARAM, "poly_stride < nlimbs");
    ntt_batch(*h->c.E, d, npolys, first, nlimbs, stride, false, h->c.stream);
  });
}

}  // extern "C"
