// Runs the reference's DGT evaluator CKKS operations through its public API
// (pdroalves/aoa aoa-dgt: CKKSContext, ckks_mul, ckks_mul_without_rescale,
// ckks_rotate_left, ckks_conjugate, ckks_add, ckks_sub, CKKSContext::encode,
// ckks_new_sk, ckks_keygen, ckks_encrypt, ckks_decrypt) and writes their
// outputs to a file, with the records, seeds and value rules of
// ref_ckks_harness (magic "AOAREF04").  Polynomials are written as
// coefficients (poly_copy_to_host: inverse DGT, then unfolded from the
// reference's Gaussian integers); operands and keys go in the same way
// (poly_copy_to_device folds them).  The outputs pin the engine on a DGT
// context (the AOADGT drop-in) to the reference's DGT evaluator.
//
// Built by oracle/ref/Makefile beside ref_dgt_harness, from aoa-dgt's
// unmodified sources, with the NTL, rapidjson and FFTW stand-ins of
// oracle/ref/shim.  Test infrastructure only: nothing in the product links or
// runs it.
//
// usage: ref_dgt_ckks_harness <out file> <log2 nphi> <k> <kl> <prec>
//        ref_dgt_ckks_harness --digest <log2 nphi> <k> <kl> <prec>   (see digests)
// Records (little-endian u64): {tag, level, nwords, words}; a ciphertext
// record holds [aux, scale, slots, c0 limbs 0..n-1, c1 limbs 0..n-1]:
//   20 ckks_mul(a, b), 21 ckks_mul_without_rescale(a, b), 22 ckks_rotate_left
//   (c, r) (aux = r), 23 ckks_conjugate(c), 24 ckks_add(a, c), 25 ckks_sub(a,
//   c) at input levels k - 1 and 1 (record level = output level); seeds:
//   a = (101, 102), b = (103, 104), c = (105, 106), evaluation key (b, a) =
//   (111, 112), rotation key for r = (113 + 10 r, 114 + 10 r), conjugation
//   key (115, 116); scales 2^40 + 3 (a, c) and 2^40 + 5 (b); slots nphi / 2;
//   26 CKKSContext::encode of `level` slots ([scale, k limbs]), values of seed
//      200 + slots (re, im = 2 u - 1, u = top 53 bits x 2^-53, re first);
//   40 secret key (nphi signed coefficients), 41 evaluation key
//   ([b limbs 0..k+kl-1, a limbs]), 42 / 43 ckks_encrypt of the values of
//   seeds 300 / 301 (nphi / 2 slots), 44 their ckks_mul, 47 ckks_rotate_left
//   of 42 by 1, 45 / 46 / 48 ckks_decrypt of 42 / 44 / 47 (re, im doubles).
#include <AOADGT/ckks.h>
#include <AOADGT/ckkscontext.h>
#include <AOADGT/keys.h>
#include <AOADGT/cuda/sampler.h>

#include <complex>
#include <cstdio>
#include <cstring>
#include <vector>

static const uint64_t kScaleA = (1ull << 40) + 3, kScaleB = (1ull << 40) + 5;

static uint64_t splitmix(uint64_t& s) {
  uint64_t z = (s += 0x9E3779B97F4A7C15ull);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

static std::vector<uint64_t> g_primes;
static int g_nphi, g_k, g_kl;
static FILE* g_out;

static std::vector<uint64_t> residues(uint64_t seed, int nlimbs) {
  std::vector<uint64_t> v((size_t)nlimbs * g_nphi);
  uint64_t s = seed;
  for (int i = 0; i < nlimbs; i++)
    for (int j = 0; j < g_nphi; j++) v[(size_t)i * g_nphi + j] = splitmix(s) % g_primes[i];
  return v;
}

static std::vector<std::complex<double>> values(uint64_t seed, int slots) {
  std::vector<std::complex<double>> v(slots);
  uint64_t s = seed;
  for (int i = 0; i < slots; i++) {
    const double re = 2.0 * ((double)(splitmix(s) >> 11) * 0x1.0p-53) - 1.0;
    const double im = 2.0 * ((double)(splitmix(s) >> 11) * 0x1.0p-53) - 1.0;
    v[i] = {re, im};
  }
  return v;
}

static void record(uint64_t tag, uint64_t level, const std::vector<uint64_t>& w) {
  const uint64_t hdr[3] = {tag, level, (uint64_t)w.size()};
  fwrite(hdr, 8, 3, g_out);
  fwrite(w.data(), 8, w.size(), g_out);
}

// coefficients of residues 0..nlimbs-1 of p
static std::vector<uint64_t> limbs(Context* ctx, poly_t* p, int nlimbs) {
  uint64_t* h = poly_copy_to_host(ctx, p);
  std::vector<uint64_t> v(h, h + (size_t)nlimbs * g_nphi);
  free(h);
  return v;
}

static void record_ct(uint64_t tag, Context* ctx, cipher_t* c, uint64_t aux) {
  const int n = c->level + 1;
  std::vector<uint64_t> w = {aux, (uint64_t)c->scale, (uint64_t)c->slots};
  const std::vector<uint64_t> c0 = limbs(ctx, &c->c[0], n), c1 = limbs(ctx, &c->c[1], n);
  w.insert(w.end(), c0.begin(), c0.end());
  w.insert(w.end(), c1.begin(), c1.end());
  record(tag, c->level, w);
}

static void upload(Context* ctx, poly_t* p, poly_bases base, uint64_t seed) {
  poly_init(ctx, p, base);
  std::vector<uint64_t> x = residues(seed, CUDAEngine::get_n_residues(base));
  poly_copy_to_device(ctx, p, x.data());
  cudaStreamSynchronize(ctx->get_stream());             // the staging buffer is reused
}

static void set_ct(Context* ctx, cipher_t* c, uint64_t seed0, uint64_t seed1, int level, uint64_t scale,
                   int slots) {
  cipher_init(ctx, c, slots);
  upload(ctx, &c->c[0], QBase, seed0);
  upload(ctx, &c->c[1], QBase, seed1);
  c->level = level;
  c->scale = (int64_t)scale;
  c->slots = slots;
}

static SwitchKey* new_key(Context* ctx, uint64_t seed_b, uint64_t seed_a) {
  SwitchKey* key = new SwitchKey;
  upload(ctx, &key->b, QBBase, seed_b);
  upload(ctx, &key->a, QBBase, seed_a);
  return key;
}

static void record_values(uint64_t tag, const std::complex<double>* v, int slots) {
  std::vector<uint64_t> w(2 * (size_t)slots);
  for (int i = 0; i < slots; i++) {
    const double re = v[i].real(), im = v[i].imag();
    memcpy(&w[2 * i], &re, 8);
    memcpy(&w[2 * i + 1], &im, 8);
  }
  record(tag, 0, w);
}

static bool check_cuda(const char* where) {
  const cudaError_t e = cudaDeviceSynchronize();
  if (e != cudaSuccess) {
    fprintf(stderr, "%s: %s\n", where, cudaGetErrorString(e));
    return false;
  }
  return true;
}

static void seeded_operands(CKKSContext* ctx) {
  const int slots = g_nphi / 2;
  ctx->evk = new_key(ctx, 111, 112);
  ctx->cjk = new_key(ctx, 115, 116);
  const int rots[2] = {1, 4};
  for (int r : rots) ctx->rtk_left[r] = new_key(ctx, 113 + 10 * r, 114 + 10 * r);
  const int levels[2] = {g_k - 1, 1};
  for (int level : levels) {
    cipher_t a, b, c, out;
    cipher_init(ctx, &out);
    set_ct(ctx, &a, 101, 102, level, kScaleA, slots);
    set_ct(ctx, &b, 103, 104, level, kScaleB, slots);
    ckks_mul(ctx, &out, &a, &b);
    record_ct(20, ctx, &out, 0);
    set_ct(ctx, &a, 101, 102, level, kScaleA, slots);
    set_ct(ctx, &b, 103, 104, level, kScaleB, slots);
    ckks_mul_without_rescale(ctx, &out, &a, &b);
    record_ct(21, ctx, &out, 0);
    for (int r : rots) {
      set_ct(ctx, &c, 105, 106, level, kScaleA, slots);
      ckks_rotate_left(ctx, &out, &c, r);
      record_ct(22, ctx, &out, r);
    }
    set_ct(ctx, &c, 105, 106, level, kScaleA, slots);
    ckks_conjugate(ctx, &out, &c);
    record_ct(23, ctx, &out, 0);
    set_ct(ctx, &a, 101, 102, level, kScaleA, slots);
    set_ct(ctx, &c, 105, 106, level, kScaleA, slots);
    ckks_add(ctx, &out, &a, &c);
    record_ct(24, ctx, &out, 0);
    set_ct(ctx, &a, 101, 102, level, kScaleA, slots);
    set_ct(ctx, &c, 105, 106, level, kScaleA, slots);
    ckks_sub(ctx, &out, &a, &c);
    record_ct(25, ctx, &out, 0);
    cipher_free(ctx, &a);
    cipher_free(ctx, &b);
    cipher_free(ctx, &c);
    cipher_free(ctx, &out);
  }
  const int encode_slots[2] = {g_nphi / 2, 8};
  for (int s : encode_slots) {
    std::vector<std::complex<double>> v = values(200 + s, s);
    poly_t m;
    poly_init(ctx, &m);
    int64_t scale = (int64_t)kScaleA;
    ctx->encode(&m, &scale, v.data(), s, 0);
    std::vector<uint64_t> w = {(uint64_t)scale};
    const std::vector<uint64_t> r = limbs(ctx, &m, g_k);
    w.insert(w.end(), r.begin(), r.end());
    record(26, s, w);
    poly_free(ctx, &m);
  }
  cudaStreamSynchronize(ctx->get_stream());
}

static void reference_keys(CKKSContext* ctx) {
  SecretKey* sk = ckks_new_sk(ctx);
  ckks_keygen(ctx, sk);
  ctx->sk = sk;
  const int slots = g_nphi / 2;
  {
    const std::vector<uint64_t> s = limbs(ctx, &sk->s, 1);
    std::vector<uint64_t> w(g_nphi);
    for (int j = 0; j < g_nphi; j++)     // residue 0 -> signed coefficient
      w[j] = s[j] > g_primes[0] / 2 ? (uint64_t)((int64_t)s[j] - (int64_t)g_primes[0]) : s[j];
    record(40, 0, w);
  }
  {
    std::vector<uint64_t> w = limbs(ctx, &ctx->evk->b, g_k + g_kl);
    const std::vector<uint64_t> a = limbs(ctx, &ctx->evk->a, g_k + g_kl);
    w.insert(w.end(), a.begin(), a.end());
    record(41, 0, w);
  }
  std::vector<std::complex<double>> v1 = values(300, slots), v2 = values(301, slots);
  cipher_t* c1 = ckks_encrypt(ctx, v1.data(), slots, 0);
  cipher_t* c2 = ckks_encrypt(ctx, v2.data(), slots, 0);
  record_ct(42, ctx, c1, 0);
  record_ct(43, ctx, c2, 0);
  std::vector<std::complex<double>> out(slots);
  ckks_decrypt(ctx, out.data(), c1, sk);
  record_values(45, out.data(), slots);
  cipher_t prod, rot;
  cipher_init(ctx, &prod);
  cipher_init(ctx, &rot);
  ckks_mul(ctx, &prod, c1, c2);
  record_ct(44, ctx, &prod, 0);
  ckks_decrypt(ctx, out.data(), &prod, sk);
  record_values(46, out.data(), slots);
  ckks_rotate_left(ctx, &rot, c1, 1);
  record_ct(47, ctx, &rot, 1);
  ckks_decrypt(ctx, out.data(), &rot, sk);
  record_values(48, out.data(), slots);
  cudaStreamSynchronize(ctx->get_stream());
}

// Digest mode, as ref_ckks_harness --digest: ckks_mul and ckks_rotate_left
// by 1 of the seeded operands at level k - 1, each output limb (coefficients)
// reduced to sum_j c_j (2 j + 1) G mod 2^64, G = 0x9E3779B97F4A7C15.
static uint64_t limb_digest(const uint64_t* c) {
  uint64_t d = 0;
  for (int j = 0; j < g_nphi; j++) d += c[j] * ((2 * (uint64_t)j + 1) * 0x9E3779B97F4A7C15ull);
  return d;
}

static void print_digests(const char* name, Context* ctx, cipher_t* c, bool last) {
  const int n = c->level + 1;
  const std::vector<uint64_t> c0 = limbs(ctx, &c->c[0], n), c1 = limbs(ctx, &c->c[1], n);
  printf("\"%s\": {\"level\": %d, \"scale\": %llu, \"digests\": [", name, c->level,
         (unsigned long long)c->scale);
  for (int i = 0; i < 2 * n; i++) {
    const uint64_t* base = (i < n ? c0.data() : c1.data()) + (size_t)(i % n) * g_nphi;
    printf("%s%llu", i ? ", " : "", (unsigned long long)limb_digest(base));
  }
  printf("]}%s", last ? "" : ", ");
}

static int digests() {
  CKKSContext* ctx = new CKKSContext();
  const int slots = g_nphi / 2, level = g_k - 1;
  ctx->evk = new_key(ctx, 111, 112);
  ctx->rtk_left[1] = new_key(ctx, 123, 124);
  cipher_t a, b, c, out;
  cipher_init(ctx, &out);
  set_ct(ctx, &a, 101, 102, level, kScaleA, slots);
  set_ct(ctx, &b, 103, 104, level, kScaleB, slots);
  ckks_mul(ctx, &out, &a, &b);
  if (!check_cuda("ckks_mul")) return 1;
  printf("{\"N\": %d, \"k\": %d, \"kl\": %d, \"primes\": [", g_nphi, g_k, g_kl);
  for (size_t i = 0; i < g_primes.size(); i++) printf("%s%llu", i ? ", " : "", (unsigned long long)g_primes[i]);
  printf("], ");
  print_digests("hmult", ctx, &out, false);
  set_ct(ctx, &c, 105, 106, level, kScaleA, slots);
  ckks_rotate_left(ctx, &out, &c, 1);
  if (!check_cuda("ckks_rotate_left")) return 1;
  print_digests("rotate1", ctx, &out, true);
  printf("}\n");
  return 0;
}

int main(int argc, char** argv) {
  if (argc == 6 && strcmp(argv[1], "--digest") == 0) {
    g_nphi = 1 << atoi(argv[2]);
    g_k = atoi(argv[3]);
    g_kl = atoi(argv[4]);
    CUDAEngine::init(g_k, g_kl, g_nphi, atoi(argv[5]));
    if (!check_cuda("init")) return 1;
    g_primes = CUDAEngine::RNSPrimes;
    g_primes.insert(g_primes.end(), CUDAEngine::RNSBPrimes.begin(), CUDAEngine::RNSBPrimes.end());
    return digests();
  }
  if (argc != 6) {
    fprintf(stderr, "usage: ref_dgt_ckks_harness <out> <log2 nphi> <k> <kl> <prec>\n"
                    "       ref_dgt_ckks_harness --digest <log2 nphi> <k> <kl> <prec>\n");
    return 2;
  }
  g_nphi = 1 << atoi(argv[2]);
  g_k = atoi(argv[3]);
  g_kl = atoi(argv[4]);
  const int prec = atoi(argv[5]);
  CUDAEngine::init(g_k, g_kl, g_nphi, prec);
  if (!check_cuda("init")) return 1;
  g_primes = CUDAEngine::RNSPrimes;
  g_primes.insert(g_primes.end(), CUDAEngine::RNSBPrimes.begin(), CUDAEngine::RNSBPrimes.end());
  if ((int)g_primes.size() != g_k + g_kl || CUDAEngine::N * 2 != g_nphi) {
    fprintf(stderr, "unexpected engine shape\n");
    return 1;
  }
  CKKSContext* ctx = new CKKSContext();
  Sampler::init(ctx);

  g_out = fopen(argv[1], "wb");
  if (!g_out) return 1;
  const char magic[8] = {'A', 'O', 'A', 'R', 'E', 'F', '0', '4'};
  fwrite(magic, 1, 8, g_out);
  const uint64_t hdr[4] = {(uint64_t)g_nphi, (uint64_t)g_k, (uint64_t)g_kl, (uint64_t)prec};
  fwrite(hdr, 8, 4, g_out);
  fwrite(g_primes.data(), 8, g_primes.size(), g_out);

  seeded_operands(ctx);
  bool ok = check_cuda("seeded operands");
  if (ok) {
    reference_keys(ctx);
    ok = check_cuda("reference keys");
  }
  fclose(g_out);
  printf("%s: nphi=%d k=%d kl=%d prec=%d %s\n", argv[1], g_nphi, g_k, g_kl, prec, ok ? "ok" : "FAILED");
  return ok ? 0 : 1;
}
