// Runs the reference evaluator's own transform and RNS kernels through its
// public API (pdroalves/aoa aoa-ntt: CUDAManager::init, Context, poly_t,
// COMMONEngine::execute, poly_modup, poly_moddown, poly_rescale) on seeded
// inputs, and writes their outputs to a file.  The outputs become golden
// fixtures that pin the oracle to the reference's results
// (tests/golden/make_reference_outputs.py, tests/test_oracle_reference_outputs.py).
//
// Built by oracle/ref/Makefile from the reference's unmodified sources where
// they lie, with two stand-ins for libraries that are absent here: NTL
// (oracle/ref/shim/NTL: exact integer arithmetic for the reference's host
// precompute) and rapidjson (declarations only; JSON export is not used).
// Test infrastructure only: nothing in the product links or runs it.
//
// usage: ref_harness <out file> <log2 N> <k> <kl> <prec> <transform only 0|1>
//        ref_harness --time <log2 N> <k> <kl> <prec> <polys>   (see time_transforms)
// Inputs: word j of limb i of an input polynomial is output i N + j of
// splitmix64 seeded with the case's seed, reduced mod p_i; seeds: forward
// transform 1, inverse transform 2, ModUp 2 + 1000 level, ModDown
// 3 + 1000 level, rescale 4 + 1000 level and 5 + 1000 level (the two polys).
// Output file (little-endian u64): "AOAREF01", N, k, kl, prec, k + kl primes,
// then records {tag, level, nwords, words}:
//   1 forward transform of a QB poly           (all k + kl limbs)
//   2 inverse transform of a QB poly            (input taken as transform domain)
//   3 ModUp at `level` of a Q poly              (the kl B limbs)
//   4 ModDown at `level` of a QB poly           (Q limbs 0..level)
//   5 rescale at `level` of two Q polys         (limbs 0..level-1 of each)
//   6 ModUp at `level` of a Q poly of all (q_i - 1)
//   7 forward transform of a QB poly of all (p_i - 1)
#include <newckks/cuda/manager.h>
#include <newckks/cuda/htrans/common.h>
#include <newckks/arithmetic/poly_t.h>
#include <newckks/tool/context.h>

#include <chrono>
#include <cstdio>
#include <cstring>
#include <vector>

static uint64_t splitmix(uint64_t& s) {
  uint64_t z = (s += 0x9E3779B97F4A7C15ull);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

static std::vector<uint64_t> g_primes;
static int g_N;

// nlimbs limbs (primes first_prime..) of uniform residues from `seed`, or all p - 1
static std::vector<uint64_t> residues(uint64_t seed, int first_prime, int nlimbs, bool max) {
  std::vector<uint64_t> v((size_t)nlimbs * g_N);
  uint64_t s = seed;
  for (int i = 0; i < nlimbs; i++) {
    const uint64_t p = g_primes[first_prime + i];
    for (int j = 0; j < g_N; j++) v[(size_t)i * g_N + j] = max ? p - 1 : splitmix(s) % p;
  }
  return v;
}

static std::vector<uint64_t> download(Context* ctx, const poly_t* p, int first_limb, int nlimbs) {
  std::vector<uint64_t> h((size_t)nlimbs * g_N);
  cudaStreamSynchronize(ctx->get_stream());
  cudaMemcpy(h.data(), p->d_coefs + (size_t)first_limb * g_N, h.size() * 8, cudaMemcpyDeviceToHost);
  return h;
}

static FILE* g_out;
static void record(uint64_t tag, uint64_t level, const std::vector<uint64_t>& w) {
  const uint64_t hdr[3] = {tag, level, (uint64_t)w.size()};
  fwrite(hdr, 8, 3, g_out);
  fwrite(w.data(), 8, w.size(), g_out);
}

static bool check_cuda(const char* where) {
  const cudaError_t e = cudaDeviceSynchronize();
  if (e != cudaSuccess) {
    fprintf(stderr, "%s: %s\n", where, cudaGetErrorString(e));
    return false;
  }
  return true;
}

// Timing mode: forward, then inverse transforms (COMMONEngine::execute, one
// call per poly, as the reference's API runs them) of `polys` seeded polys
// of k limbs, after one warm-up round; host clock around each
// device-synchronised round.  Prints one JSON line with the primes, the
// times and the algorithmic rate (16 bytes per coefficient per direction).
static int time_transforms(int k, int polys) {
  Context* ctx = new Context();
  std::vector<poly_t> p(polys);
  for (int i = 0; i < polys; i++) {
    std::vector<uint64_t> x = residues(1 + i, 0, k, false);
    poly_init(ctx, &p[i], QBase);
    poly_copy_to_device(ctx, &p[i], x.data());
  }
  if (!check_cuda("upload")) return 1;
  double ms[2] = {0, 0};
  for (int round = 0; round < 2; round++) {
    for (int dir = 0; dir < 2; dir++) {
      const auto t0 = std::chrono::steady_clock::now();
      for (int i = 0; i < polys; i++) COMMONEngine::execute(ctx, &p[i], dir == 0 ? FORWARD : INVERSE);
      if (!check_cuda("transforms")) return 1;
      ms[dir] = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    }
  }
  const double bytes = 16.0 * polys * k * g_N;
  printf("{\"N\": %d, \"polys\": %d, \"limbs\": %d, \"fwd_ms\": %.4f, \"inv_ms\": %.4f, "
         "\"fwd_gbs\": %.2f, \"inv_gbs\": %.2f, \"primes\": [",
         g_N, polys, k, ms[0], ms[1], bytes / ms[0] / 1e6, bytes / ms[1] / 1e6);
  for (int i = 0; i < k; i++) printf("%s%llu", i ? ", " : "", (unsigned long long)g_primes[i]);
  printf("]}\n");
  return 0;
}

int main(int argc, char** argv) {
  if (argc == 7 && strcmp(argv[1], "--time") == 0) {
    g_N = 1 << atoi(argv[2]);
    const int k = atoi(argv[3]);
    CUDAManager::init(k, atoi(argv[4]), g_N, atoi(argv[5]));
    if (!check_cuda("init")) return 1;
    g_primes = CUDAManager::RNSQPrimes;
    g_primes.insert(g_primes.end(), CUDAManager::RNSBPrimes.begin(), CUDAManager::RNSBPrimes.end());
    return time_transforms(k, atoi(argv[6]));
  }
  if (argc != 7) {
    fprintf(stderr, "usage: ref_harness <out> <log2 N> <k> <kl> <prec> <transform only 0|1>\n"
                    "       ref_harness --time <log2 N> <k> <kl> <prec> <polys>\n");
    return 2;
  }
  g_N = 1 << atoi(argv[2]);
  const int k = atoi(argv[3]), kl = atoi(argv[4]), prec = atoi(argv[5]);
  const bool transform_only = atoi(argv[6]) != 0;

  CUDAManager::init(k, kl, g_N, prec);                    // the reference's prime choice and precompute
  if (!check_cuda("init")) return 1;
  g_primes = CUDAManager::RNSQPrimes;
  g_primes.insert(g_primes.end(), CUDAManager::RNSBPrimes.begin(), CUDAManager::RNSBPrimes.end());
  const int nqb = k + kl;
  Context* ctx = new Context();

  g_out = fopen(argv[1], "wb");
  if (!g_out) return 1;
  const char magic[8] = {'A', 'O', 'A', 'R', 'E', 'F', '0', '1'};
  fwrite(magic, 1, 8, g_out);
  const uint64_t hdr[4] = {(uint64_t)g_N, (uint64_t)k, (uint64_t)kl, (uint64_t)prec};
  fwrite(hdr, 8, 4, g_out);
  fwrite(g_primes.data(), 8, g_primes.size(), g_out);

  bool ok = true;
  for (int max = 0; max < 2; max++) {                     // forward transform (tags 1 and 7)
    std::vector<uint64_t> x = residues(1, 0, nqb, max);
    poly_t p;
    poly_init(ctx, &p, QBBase);
    poly_copy_to_device(ctx, &p, x.data());
    COMMONEngine::execute(ctx, &p, FORWARD);
    record(max ? 7 : 1, 0, download(ctx, &p, 0, nqb));
    COMMONEngine::execute(ctx, &p, INVERSE);
    if (download(ctx, &p, 0, nqb) != x) {
      fprintf(stderr, "the reference's inverse transform did not restore its input\n");
      ok = false;
    }
    poly_free(ctx, &p);
  }
  {                                                       // inverse transform (tag 2)
    std::vector<uint64_t> y = residues(2, 0, nqb, false);
    poly_t p;
    poly_init(ctx, &p, QBBase);
    poly_copy_to_device(ctx, &p, y.data());
    p.state = TRANSSTATE;
    COMMONEngine::execute(ctx, &p, INVERSE);
    record(2, 0, download(ctx, &p, 0, nqb));
    poly_free(ctx, &p);
  }
  if (!transform_only) {
    const int levels[2] = {k - 1, 1};
    for (int li = 0; li < 2; li++) {
      const int level = levels[li];
      for (int max = 0; max < 2; max++) {                 // ModUp (tags 3 and 6)
        std::vector<uint64_t> x = residues(2 + 1000 * level, 0, k, max);
        poly_t b, a;
        poly_init(ctx, &b, QBase);
        poly_copy_to_device(ctx, &b, x.data());
        poly_modup(ctx, &a, &b, level);
        record(max ? 6 : 3, level, download(ctx, &a, k, kl));
        poly_free(ctx, &a);
        poly_free(ctx, &b);
      }
      {                                                   // ModDown (tag 4)
        const int dl = level == 1 ? 0 : level;
        std::vector<uint64_t> x = residues(3 + 1000 * dl, 0, nqb, false);
        poly_t b, a;
        poly_init(ctx, &b, QBBase);
        poly_copy_to_device(ctx, &b, x.data());
        poly_moddown(ctx, &a, &b, dl);
        record(4, dl, download(ctx, &a, 0, dl + 1));
        poly_free(ctx, &a);
        poly_free(ctx, &b);
      }
      {                                                   // rescale (tag 5)
        std::vector<uint64_t> x0 = residues(4 + 1000 * level, 0, k, false);
        std::vector<uint64_t> x1 = residues(5 + 1000 * level, 0, k, false);
        poly_t a, b;
        poly_init(ctx, &a, QBase);
        poly_init(ctx, &b, QBase);
        poly_copy_to_device(ctx, &a, x0.data());
        poly_copy_to_device(ctx, &b, x1.data());
        poly_rescale(ctx, &a, &b, level);
        std::vector<uint64_t> w = download(ctx, &a, 0, level);
        std::vector<uint64_t> w1 = download(ctx, &b, 0, level);
        w.insert(w.end(), w1.begin(), w1.end());
        record(5, level, w);
        poly_free(ctx, &a);
        poly_free(ctx, &b);
      }
    }
  }
  ok = check_cuda("kernels") && ok;
  fclose(g_out);
  delete ctx;
  CUDAManager::destroy();
  printf("%s: N=%d k=%d kl=%d prec=%d %s\n", argv[1], g_N, k, kl, prec, ok ? "ok" : "FAILED");
  return ok ? 0 : 1;
}
