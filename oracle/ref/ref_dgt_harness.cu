// Runs the reference's DGT evaluator kernels through its public API
// (pdroalves/aoa aoa-dgt: CUDAEngine::init, Context, poly_t,
// DGTEngine::execute_dgt, poly_mul, poly_modup, poly_moddown,
// poly_ckks_rescale) on seeded inputs, and writes their outputs to a file.
// The outputs become golden fixtures that pin the oracle's DGT and the
// coefficient-wise RNS kernels on a DGT engine to the reference's results
// (tests/golden/make_reference_outputs.py, tests/test_oracle_reference_dgt.py).
//
// Built by oracle/ref/Makefile from aoa-dgt's unmodified sources where they
// lie, with the NTL and rapidjson stand-ins of oracle/ref/shim.  aoa-dgt's
// encoder and CKKS layer need FFTW, which is absent, and are not built.  Test
// infrastructure only: nothing in the product links or runs it.
//
// usage: ref_dgt_harness <out file> <log2 nphi> <k> <kl> <prec> <transform only 0|1>
//        ref_dgt_harness --time <log2 nphi> <k> <kl> <prec> <polys>   (see time_transforms)
// A polynomial of nphi coefficients is held folded as nphi / 2 Gaussian
// integers per residue (a_j + i a_{j + nphi/2}, poly_copy_to_device).
// Inputs: coefficient j of residue i of an input polynomial is output
// i nphi + j of splitmix64 seeded with the case's seed, reduced mod p_i (the
// same rule as ref_harness).  Seeds: forward transform 1, inverse transform
// 2 (its words taken as transform-domain Gaussian integers, word 2j the real
// and 2j + 1 the imaginary part of entry j), product 3 and 4, ModUp
// 10 + level, ModDown 20 + level, rescale 30 + level and 40 + level.
// Output file (little-endian u64): "AOAREF03", nphi, k, kl, prec, k + kl
// primes, then records {tag, level, nwords, words}:
//   1 forward DGT of a QB poly     (raw Gaussian integers: re, im per entry)
//   2 inverse DGT of a QB poly     (raw Gaussian integers)
//   3 poly_mul of two Q polys      (coefficients, unfolded)
//   4 ModUp at `level` of a Q poly (the kl B residues, coefficients)
//   5 ModDown at `level`           (Q residues 0..level, coefficients)
//   6 rescale at `level` of two Q polys (residues 0..level-1 of each)
#include <AOADGT/arithmetic/polynomial.h>
#include <AOADGT/arithmetic/context.h>
#include <AOADGT/cuda/cudaengine.h>
#include <AOADGT/cuda/dgt.h>

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
static int g_nphi, g_k, g_kl;
static FILE* g_out;

// nlimbs residues of nphi coefficients (primes 0..nlimbs-1) from `seed`
static std::vector<uint64_t> residues(uint64_t seed, int nlimbs) {
  std::vector<uint64_t> v((size_t)nlimbs * g_nphi);
  uint64_t s = seed;
  for (int i = 0; i < nlimbs; i++)
    for (int j = 0; j < g_nphi; j++) v[(size_t)i * g_nphi + j] = splitmix(s) % g_primes[i];
  return v;
}

static void record(uint64_t tag, uint64_t level, const std::vector<uint64_t>& w) {
  const uint64_t hdr[3] = {tag, level, (uint64_t)w.size()};
  fwrite(hdr, 8, 3, g_out);
  fwrite(w.data(), 8, w.size(), g_out);
}

// residues first..first+n-1 of p as stored (Gaussian integers, 2 words each)
static std::vector<uint64_t> raw(Context* ctx, const poly_t* p, int first, int n) {
  const int half = g_nphi / 2;
  std::vector<uint64_t> h((size_t)n * g_nphi);
  cudaStreamSynchronize(ctx->get_stream());
  cudaMemcpy(h.data(), p->d_coefs + (size_t)first * half, h.size() * 8, cudaMemcpyDeviceToHost);
  return h;
}

// the same residues unfolded to coefficients (re parts, then im parts)
static std::vector<uint64_t> unfolded(Context* ctx, const poly_t* p, int first, int n) {
  const int half = g_nphi / 2;
  const std::vector<uint64_t> g = raw(ctx, p, first, n);
  std::vector<uint64_t> c(g.size());
  for (int r = 0; r < n; r++)
    for (int j = 0; j < half; j++) {
      c[(size_t)r * g_nphi + j] = g[(size_t)r * g_nphi + 2 * j];
      c[(size_t)r * g_nphi + half + j] = g[(size_t)r * g_nphi + 2 * j + 1];
    }
  return c;
}

static void upload(Context* ctx, poly_t* p, poly_bases base, const std::vector<uint64_t>& coefs) {
  poly_init(ctx, p, base);
  std::vector<uint64_t> full((size_t)CUDAEngine::get_n_residues(base) * g_nphi, 0);
  std::copy(coefs.begin(), coefs.end(), full.begin());
  poly_copy_to_device(ctx, p, full.data());
  cudaStreamSynchronize(ctx->get_stream());             // the staging buffer is reused
}

static bool check_cuda(const char* where) {
  const cudaError_t e = cudaDeviceSynchronize();
  if (e != cudaSuccess) {
    fprintf(stderr, "%s: %s\n", where, cudaGetErrorString(e));
    return false;
  }
  return true;
}

// Timing mode: forward, then inverse DGTs (DGTEngine::execute_dgt, one call
// per poly) of `polys` seeded polys of k residues, after one warm-up round;
// host clock around each device-synchronised round.  Prints one JSON line
// (16 bytes per coefficient per direction).
static int time_transforms(int polys) {
  Context* ctx = new Context();
  std::vector<poly_t> p(polys);
  for (int i = 0; i < polys; i++) upload(ctx, &p[i], QBase, residues(1 + i, g_k));
  if (!check_cuda("upload")) return 1;
  double ms[2] = {0, 0};
  for (int round = 0; round < 2; round++) {
    for (int dir = 0; dir < 2; dir++) {
      const auto t0 = std::chrono::steady_clock::now();
      for (int i = 0; i < polys; i++) DGTEngine::execute_dgt(ctx, &p[i], dir == 0 ? FORWARD : INVERSE);
      if (!check_cuda("transforms")) return 1;
      ms[dir] = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    }
  }
  const double bytes = 16.0 * polys * g_k * g_nphi;
  printf("{\"nphi\": %d, \"polys\": %d, \"limbs\": %d, \"fwd_ms\": %.4f, \"inv_ms\": %.4f, "
         "\"fwd_gbs\": %.2f, \"inv_gbs\": %.2f, \"primes\": [",
         g_nphi, polys, g_k, ms[0], ms[1], bytes / ms[0] / 1e6, bytes / ms[1] / 1e6);
  for (int i = 0; i < g_k; i++) printf("%s%llu", i ? ", " : "", (unsigned long long)g_primes[i]);
  printf("]}\n");
  return 0;
}

int main(int argc, char** argv) {
  if (argc == 7 && strcmp(argv[1], "--time") == 0) {
    g_nphi = 1 << atoi(argv[2]);
    g_k = atoi(argv[3]);
    g_kl = atoi(argv[4]);
    CUDAEngine::init(g_k, g_kl, g_nphi, atoi(argv[5]));
    if (!check_cuda("init")) return 1;
    g_primes = CUDAEngine::RNSPrimes;
    g_primes.insert(g_primes.end(), CUDAEngine::RNSBPrimes.begin(), CUDAEngine::RNSBPrimes.end());
    return time_transforms(atoi(argv[6]));
  }
  if (argc != 7) {
    fprintf(stderr, "usage: ref_dgt_harness <out> <log2 nphi> <k> <kl> <prec> <transform only 0|1>\n");
    return 2;
  }
  g_nphi = 1 << atoi(argv[2]);
  g_k = atoi(argv[3]);
  g_kl = atoi(argv[4]);
  const int prec = atoi(argv[5]);
  const bool transform_only = atoi(argv[6]) != 0;
  CUDAEngine::init(g_k, g_kl, g_nphi, prec);             // the reference's prime choice and tables
  if (!check_cuda("init")) return 1;
  g_primes = CUDAEngine::RNSPrimes;
  g_primes.insert(g_primes.end(), CUDAEngine::RNSBPrimes.begin(), CUDAEngine::RNSBPrimes.end());
  const int nqb = g_k + g_kl;
  if ((int)g_primes.size() != nqb || CUDAEngine::N * 2 != g_nphi) {
    fprintf(stderr, "unexpected engine shape\n");
    return 1;
  }
  Context* ctx = new Context();

  g_out = fopen(argv[1], "wb");
  if (!g_out) return 1;
  const char magic[8] = {'A', 'O', 'A', 'R', 'E', 'F', '0', '3'};
  fwrite(magic, 1, 8, g_out);
  const uint64_t hdr[4] = {(uint64_t)g_nphi, (uint64_t)g_k, (uint64_t)g_kl, (uint64_t)prec};
  fwrite(hdr, 8, 4, g_out);
  fwrite(g_primes.data(), 8, g_primes.size(), g_out);

  bool ok = true;
  {                                                       // forward DGT (tag 1)
    const std::vector<uint64_t> x = residues(1, nqb);
    poly_t p;
    upload(ctx, &p, QBBase, x);
    DGTEngine::execute_dgt(ctx, &p, FORWARD);
    record(1, 0, raw(ctx, &p, 0, nqb));
    DGTEngine::execute_dgt(ctx, &p, INVERSE);
    if (unfolded(ctx, &p, 0, nqb) != x) {
      fprintf(stderr, "the reference's inverse DGT did not restore its input\n");
      ok = false;
    }
    poly_free(ctx, &p);
  }
  {                                                       // inverse DGT (tag 2)
    const std::vector<uint64_t> y = residues(2, nqb);
    poly_t p;
    poly_init(ctx, &p, QBBase);
    cudaMemcpyAsync(p.d_coefs, y.data(), y.size() * 8, cudaMemcpyHostToDevice, ctx->get_stream());
    p.state = TRANSSTATE;
    DGTEngine::execute_dgt(ctx, &p, INVERSE);
    record(2, 0, raw(ctx, &p, 0, nqb));
    poly_free(ctx, &p);
  }
  if (!transform_only) {                                  // product (tag 3)
    poly_t a, b, c;
    upload(ctx, &a, QBase, residues(3, g_k));
    upload(ctx, &b, QBase, residues(4, g_k));
    poly_init(ctx, &c, QBase);
    poly_mul(ctx, &c, &a, &b);
    DGTEngine::execute_dgt(ctx, &c, INVERSE);
    record(3, 0, unfolded(ctx, &c, 0, g_k));
    poly_free(ctx, &a);
    poly_free(ctx, &b);
    poly_free(ctx, &c);
  }
  const int levels[2] = {g_k - 1, 1};
  for (int level : levels) {
    if (transform_only) break;
    {                                                     // ModUp (tag 4)
      poly_t a, b;
      upload(ctx, &b, QBase, residues(10 + level, g_k));
      poly_init(ctx, &a, QBBase);                         // the output holds QB
      poly_modup(ctx, &a, &b, level);
      record(4, level, unfolded(ctx, &a, g_k, g_kl));
      poly_free(ctx, &a);
      poly_free(ctx, &b);
    }
    {                                                     // ModDown (tag 5)
      poly_t a, b;
      upload(ctx, &b, QBBase, residues(20 + level, nqb));
      poly_init(ctx, &a, QBase);
      poly_moddown(ctx, &a, &b, level);
      record(5, level, unfolded(ctx, &a, 0, level + 1));
      poly_free(ctx, &a);
      poly_free(ctx, &b);
    }
    {                                                     // rescale (tag 6)
      poly_t a, b;
      upload(ctx, &a, QBase, residues(30 + level, g_k));
      upload(ctx, &b, QBase, residues(40 + level, g_k));
      poly_ckks_rescale(ctx, &a, &b, level);
      std::vector<uint64_t> w = unfolded(ctx, &a, 0, level);
      const std::vector<uint64_t> w1 = unfolded(ctx, &b, 0, level);
      w.insert(w.end(), w1.begin(), w1.end());
      record(6, level, w);
      poly_free(ctx, &a);
      poly_free(ctx, &b);
    }
  }
  ok = check_cuda("kernels") && ok;
  fclose(g_out);
  delete ctx;
  printf("%s: nphi=%d k=%d kl=%d prec=%d %s\n", argv[1], g_nphi, g_k, g_kl, prec, ok ? "ok" : "FAILED");
  return ok ? 0 : 1;
}
