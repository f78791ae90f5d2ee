// A caller written against the reference evaluator's signatures
// (aoa-ntt include/newckks/ckks/ckks.h), compiled against the shim header
// include/newckks/ckks/ckks.h and linked with libaoa_b200.so; built with
// -DSHIM_DGT it includes AOADGT/ckks.h instead and initialises through
// CUDAEngine::init, as a caller of aoa-dgt does.
//
// usage: shim_check <input file> <output file>
// input (u64 words): log_n k kl prec slots r scale1 scale2 keys_in_transform_domain |
//   k + kl primes | evk b, a | rtk_left[r] b, a | rtk_right[r] b, a
//   ((k + kl) x N each, in the evaluator's transform domain or in coefficients)
//   | c1 (2 x k x N) | c2 (2 x k x N)                   (coefficients)
// output (u64 words): for ckks_mul, ckks_rotate_left, ckks_rotate_right,
//   ckks_rescale (of c1), ckks_add (c1 + c2), ckks_sub (c1 - c2): level,
//   slots, scale, then 2 x (level + 1) x N coefficient residues.
// Exit status 0 only if every call ran and every error case threw as the
// reference does; messages go to stderr.
#ifdef SHIM_DGT
#include <AOADGT/ckks.h>
#else
#include <newckks/ckks/ckks.h>
#endif

#include <cstdio>
#include <cstring>
#include <fstream>
#include <iostream>
#include <vector>

static std::vector<uint64_t> read_all(const char* path) {
  std::ifstream f(path, std::ios::binary);
  std::vector<char> raw((std::istreambuf_iterator<char>(f)), std::istreambuf_iterator<char>());
  std::vector<uint64_t> w(raw.size() / 8);
  std::memcpy(w.data(), raw.data(), w.size() * 8);
  return w;
}

static void emit(CKKSContext* x, cipher_t* c, std::vector<uint64_t>& out, long N) {
  out.push_back((uint64_t)c->level);
  out.push_back((uint64_t)c->slots);
  out.push_back((uint64_t)c->scale);
  std::vector<uint64_t> h((size_t)2 * (c->level + 1) * N);
  cipher_copy_to_host(x, c, h.data(), c->level + 1);
  out.insert(out.end(), h.begin(), h.end());
}

template <class F>
static bool throws(F f, const char* expect) {
  try {
    f();
  } catch (const std::runtime_error& e) {
    if (std::strcmp(e.what(), expect) == 0) return true;
    std::cerr << "unexpected message: " << e.what() << "\n";
    return false;
  }
  std::cerr << "no exception, expected: " << expect << "\n";
  return false;
}

int main(int argc, char** argv) {
  if (argc != 3) {
    std::cerr << "usage: shim_check <input> <output>\n";
    return 2;
  }
  const std::vector<uint64_t> in = read_all(argv[1]);
  size_t at = 0;
  auto take = [&](size_t n) {
    if (at + n > in.size()) throw std::runtime_error("input file too short");
    const uint64_t* p = in.data() + at;
    at += n;
    return p;
  };
  const uint64_t* hdr = take(9);
  const int log_n = (int)hdr[0], k = (int)hdr[1], kl = (int)hdr[2], prec = (int)hdr[3], slots = (int)hdr[4];
  const int r = (int)hdr[5];
  const int64_t scale1 = (int64_t)hdr[6], scale2 = (int64_t)hdr[7];
  const bool keys_transform = hdr[8] != 0;
  const long N = 1L << log_n;
  const size_t qb = (size_t)(k + kl) * N, ct = (size_t)2 * k * N;
  const uint64_t* p = take(k + kl);
  std::vector<uint64_t> primes(p, p + k + kl);
  const uint64_t *evk_b = take(qb), *evk_a = take(qb);
  const uint64_t *rl_b = take(qb), *rl_a = take(qb);
  const uint64_t *rr_b = take(qb), *rr_a = take(qb);
  const uint64_t *h1 = take(ct), *h2 = take(ct);

  bool ok = true;
  try {
#ifdef SHIM_DGT
    CUDAEngine::init(k, kl, (int)(2 * N), (uint64_t)prec, primes);
#else
    CUDAManager::init(k, kl, (int)N, prec, primes);
#endif
    CKKSContext* ctx = new CKKSContext();
    ctx->keys.evk = ckks_load_switchkey(ctx, evk_b, evk_a, keys_transform);
    ctx->keys.rtk_left[r] = ckks_load_switchkey(ctx, rl_b, rl_a, keys_transform);
    ctx->keys.rtk_right[r] = ckks_load_switchkey(ctx, rr_b, rr_a, keys_transform);

    cipher_t c1, c2;
    cipher_init(ctx, &c1, slots);
    cipher_init(ctx, &c2, slots);
    if (c1.level != k - 1 || c1.scale != ((int64_t)1 << prec)) {
      std::cerr << "cipher_init: level " << c1.level << " scale " << c1.scale << "\n";
      ok = false;
    }
    auto load = [&](cipher_t* c, const uint64_t* h, int64_t scale) {
      cipher_copy_to_device(ctx, c, h, k);
      c->level = k - 1;
      c->slots = slots;
      c->scale = scale;
    };
    std::vector<uint64_t> out;

    load(&c1, h1, scale1);
    load(&c2, h2, scale2);
    cipher_t* m = ckks_mul(ctx, &c1, &c2);            // the allocating overload
    emit(ctx, m, out, N);

    load(&c1, h1, scale1);
    cipher_t rl, rr;
    ckks_rotate_left(ctx, &rl, &c1, r);
    emit(ctx, &rl, out, N);
    load(&c1, h1, scale1);
    ckks_rotate_right(ctx, &rr, &c1, r);
    emit(ctx, &rr, out, N);

    load(&c1, h1, scale1);
    ckks_rescale(ctx, &c1);
    emit(ctx, &c1, out, N);

    load(&c1, h1, scale1);
    load(&c2, h2, scale2);
    cipher_t* s = ckks_add(ctx, &c1, &c2);
    emit(ctx, s, out, N);
    load(&c1, h1, scale1);
    load(&c2, h2, scale2);
    cipher_t* d = ckks_sub(ctx, &c1, &c2);
    emit(ctx, d, out, N);

    // the reference's error cases: level 0 (ckks.cpp:224-227, 281-284) and a
    // slot mismatch (ckks.cpp:286-289) throw std::runtime_error
    const char* lvl0 = "The ciphertext level is 0. No more rescaling is possible.";
    load(&c1, h1, scale1);
    load(&c2, h2, scale2);
    c1.level = 0;
    cipher_t t;
    ok &= throws([&] { ckks_mul(ctx, &t, &c1, &c2); }, lvl0);
    ok &= throws([&] { ckks_rescale(ctx, &c1); }, lvl0);
    load(&c1, h1, scale1);
    c2.slots = slots / 2;
    ok &= throws([&] { ckks_mul(ctx, &t, &c1, &c2); }, "Ciphertexts must have the same number of slots.");
    // a rotation step without a key
    try {
      ckks_rotate_left(ctx, &t, &c1, r + 1);
      std::cerr << "rotation without a key did not throw\n";
      ok = false;
    } catch (const std::out_of_range&) {
    }
    ctx->sync();

    std::ofstream f(argv[2], std::ios::binary);
    f.write((const char*)out.data(), (std::streamsize)(out.size() * 8));
    for (cipher_t* c : {m, s, d, &rl, &rr, &c1, &c2, &t}) cipher_free(ctx, c);
    delete m;
    delete s;
    delete d;
    ckks_free_switchkey(ctx, ctx->keys.evk);
    ckks_free_switchkey(ctx, ctx->keys.rtk_left[r]);
    ckks_free_switchkey(ctx, ctx->keys.rtk_right[r]);
    delete ctx;
#ifdef SHIM_DGT
    CUDAEngine::destroy();
#else
    CUDAManager::destroy();
#endif
  } catch (const std::exception& e) {
    std::cerr << "shim_check: " << e.what() << "\n";
    return 1;
  }
  return ok ? 0 : 1;
}
