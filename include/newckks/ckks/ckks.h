// newckks/ckks/ckks.h — drop-in shim for callers of the reference evaluator.
//
// Keeps the names and signatures of pdroalves/aoa's aoa-ntt evaluator
// (include/newckks/ckks/ckks.h:116-314, cipher_t.h:17-24, ckkskeys.h:10-17,
// cuda/manager.h:52-74) and forwards every call to the C ABI of
// libaoa_b200.so (aoa_ckks.h).  A caller compiled against the reference adds
// `-I <this repo>/include` ahead of the reference's include path and links
// `-laoa_b200`; the bodies below are all it needs.
//
// Differences a caller can see:
//  - the reference asserts or dereferences a null map entry where a key is
//    missing; here a missing rotation key throws std::out_of_range (map::at)
//    and a missing relinearisation key std::runtime_error;
//  - the reference exits the process on a CUDA error; here it is a
//    std::runtime_error carrying the library's message;
//  - CUDAManager::init(k, kl, N, prec) searches primes of the reference's
//    sizes (a 63-bit q0, k-1 primes of `prec` bits, kl primes of 55 bits, all
//    q = 1 mod 2N) instead of reading its tables; pass the reference's own
//    primes to the second overload for residues identical to its runs.
#pragma once

#include <complex>
#include <cstdint>
#include <map>
#include <stdexcept>
#include <string>
#include <vector>

#include "aoa_ckks.h"

// The transform of the evaluator this header stands in for: the NTT of
// newckks, or the DGT of AOADGT (set by AOADGT/ckks.h before including this).
#ifndef AOA_SHIM_TRANSFORM
#define AOA_SHIM_TRANSFORM AOA_NTT
#endif

namespace aoa_shim {

// The reference's exceptions for the same conditions (ckks.cpp:224-227, 284-290).
inline void check(int st) {
  if (st == AOA_OK) return;
  if (st == AOA_ERR_LEVEL_EXHAUSTED)
    throw std::runtime_error("The ciphertext level is 0. No more rescaling is possible.");
  if (st == AOA_ERR_SLOT_MISMATCH) throw std::runtime_error("Ciphertexts must have the same number of slots.");
  throw std::runtime_error(std::string("aoa_b200: ") + aoa_status_string(st) + ": " + aoa_last_error());
}

inline std::vector<uint64_t> search(int bits, uint64_t modulus, int count) {
  std::vector<uint64_t> out(count > 0 ? count : 0);
  if (count > 0 && aoa_search_primes(bits, modulus, count, out.data()) != count)
    throw std::runtime_error("not enough " + std::to_string(bits) + "-bit primes = 1 mod " + std::to_string(modulus));
  return out;
}

}  // namespace aoa_shim

// CUDAManager (manager.h:52-74): one default parameter set per process.
struct CUDAManager {
  static inline aoa_engine* engine = nullptr;
  static inline int N = 0, n_q = 0, n_b = 0, scalingfactor = 0;
  static inline bool is_init = false;

  // init(k, kl, N, scalingfactor): kl <= 0 means k + 1 (manager.cu:779)
  static void init(int k, int kl, int n, int prec) {
    if (kl <= 0) kl = k + 1;
    const uint64_t m = 2 * (uint64_t)n;
    std::vector<uint64_t> primes = aoa_shim::search(63, m, 1);
    const std::vector<uint64_t> q = aoa_shim::search(prec, m, k - 1);
    primes.insert(primes.end(), q.begin(), q.end());
    const std::vector<uint64_t> b = prec == 55 ? aoa_shim::search(55, m, k - 1 + kl) : aoa_shim::search(55, m, kl);
    primes.insert(primes.end(), b.end() - kl, b.end());
    init(k, kl, n, prec, primes);
  }
  // the same with explicit primes: k Q primes, then kl special primes
  static void init(int k, int kl, int n, int prec, const std::vector<uint64_t>& primes) {
    if (is_init) destroy();
    int log_n = 0;
    while ((1 << log_n) < n) log_n++;
    aoa_params p{};
    p.log_n = log_n;
    p.k = k;
    p.kl = kl;
    p.primes = primes.data();
    p.scale_bits = prec;
    p.dnum = 1;
    aoa_shim::check(aoa_engine_create(&p, &engine));
    N = n;
    n_q = k;
    n_b = kl;
    scalingfactor = prec;
    is_init = true;
  }
  static void destroy() {
    if (engine) aoa_engine_destroy(engine);
    engine = nullptr;
    is_init = false;
  }
};

// SwitchKey / EvaluationKey / RotationKey / ConjugationKey (defines.h:86-101)
struct SwitchKey {
  aoa_swk* k = nullptr;
};
typedef SwitchKey EvaluationKey;
typedef SwitchKey RotationKey;
typedef SwitchKey ConjugationKey;

// CKKSKeychain (ckkskeys.h:10-17)
struct CKKSKeychain {
  EvaluationKey* evk = nullptr;
  ConjugationKey* cjk = nullptr;
  std::map<int, RotationKey*> rtk_left, rtk_right;
};

// CKKSContext (ckkscontext.h:65-139): one stream, its keys
class CKKSContext {
 public:
  aoa_ctx* ctx = nullptr;
  CKKSKeychain keys;
  CKKSContext() {
    if (!CUDAManager::is_init) throw std::runtime_error("CUDAManager::init must come first");
    aoa_shim::check(aoa_ctx_create(CUDAManager::engine, nullptr, &ctx));
    if (AOA_SHIM_TRANSFORM == AOA_DGT) aoa_shim::check(aoa_ctx_set_transform(ctx, AOA_DGT));
  }
  ~CKKSContext() {
    if (ctx) aoa_ctx_destroy(ctx);
  }
  CKKSContext(const CKKSContext&) = delete;
  CKKSContext& operator=(const CKKSContext&) = delete;
  void sync() { aoa_shim::check(aoa_ctx_sync(ctx)); }
};

// cipher_t (cipher_t.h:17-22): level, slots and scale mirror the device object
struct cipher_t {
  aoa_ct* ct = nullptr;
  int level = 0;
  int slots = 0;
  int64_t scale = 0;
};

namespace aoa_shim {

inline void push(cipher_t* c) {   // caller-visible metadata -> device object
  int lv, sl, dom;
  uint64_t sc;
  check(aoa_ct_get(c->ct, &lv, &sl, &sc, &dom));
  check(aoa_ct_set(c->ct, c->level, c->slots, (uint64_t)c->scale, dom));
}
inline void pull(cipher_t* c) {   // device object -> caller-visible metadata
  int dom;
  uint64_t sc;
  check(aoa_ct_get(c->ct, &c->level, &c->slots, &sc, &dom));
  c->scale = (int64_t)sc;
}
inline void ensure(CKKSContext* x, cipher_t* c) {
  if (!c->ct) {
    check(aoa_ct_create(x->ctx, &c->ct));
    pull(c);
  }
}
inline const aoa_swk* key(const SwitchKey* k, const char* what) {
  if (!k || !k->k) throw std::runtime_error(std::string("missing ") + what);
  return k->k;
}

}  // namespace aoa_shim

// cipher_init (cipher_t.cpp:3-9): level k - 1, scale 2^scalingfactor
inline void cipher_init(CKKSContext* x, cipher_t* c, int slots = 1) {
  aoa_shim::check(aoa_ct_create(x->ctx, &c->ct));
  aoa_shim::pull(c);
  c->slots = slots;
  aoa_shim::push(c);
}
inline void cipher_free(CKKSContext* x, cipher_t* c) {
  if (c->ct) aoa_ct_destroy(x->ctx, c->ct);
  c->ct = nullptr;
}
// poly_copy_to_device / poly_copy_to_host (poly_t.cpp:33-100) for both polys:
// host holds 2 x nlimbs x N residues in coefficients
inline void cipher_copy_to_device(CKKSContext* x, cipher_t* c, const uint64_t* host, int nlimbs) {
  aoa_shim::ensure(x, c);
  aoa_shim::check(aoa_ct_upload(x->ctx, c->ct, host, nlimbs, AOA_COEF));
  aoa_shim::push(c);
}
inline void cipher_copy_to_host(CKKSContext* x, const cipher_t* c, uint64_t* host, int nlimbs) {
  aoa_shim::check(aoa_ct_download(x->ctx, c->ct, host, nlimbs, AOA_COEF));
}
// Switching keys given as residues (b then a, (k + kl) limbs each), in the
// reference's storage domain (its keys are kept in TRANSSTATE: the NTT domain
// of newckks, the DGT domain of AOADGT) or in coefficients
inline SwitchKey* ckks_load_switchkey(CKKSContext* x, const uint64_t* b, const uint64_t* a,
                                      bool transform_domain = true) {
  SwitchKey* k = new SwitchKey;
  aoa_shim::check(aoa_swk_create(x->ctx, b, a, transform_domain ? AOA_SHIM_TRANSFORM : AOA_COEF, &k->k));
  return k;
}
inline void ckks_free_switchkey(CKKSContext* x, SwitchKey* k) {
  if (k && k->k) aoa_swk_destroy(x->ctx, k->k);
  delete k;
}

// ckks.h:116 (ckks.cpp:220-230)
inline void ckks_rescale(CKKSContext* x, cipher_t* c) {
  aoa_shim::push(c);
  aoa_shim::check(aoa_rescale(x->ctx, c->ct));
  aoa_shim::pull(c);
}
// ckks.h:135-153 (ckks.cpp:232-271)
inline void ckks_add(CKKSContext* x, cipher_t* c3, cipher_t* c1, cipher_t* c2) {
  aoa_shim::ensure(x, c3);
  aoa_shim::push(c1);
  aoa_shim::push(c2);
  aoa_shim::check(aoa_add(x->ctx, c3->ct, c1->ct, c2->ct));
  aoa_shim::pull(c3);
}
inline cipher_t* ckks_add(CKKSContext* x, cipher_t* c1, cipher_t* c2) {
  cipher_t* c3 = new cipher_t;
  ckks_add(x, c3, c1, c2);
  return c3;
}
inline void ckks_sub(CKKSContext* x, cipher_t* c3, cipher_t* c1, cipher_t* c2) {
  aoa_shim::ensure(x, c3);
  aoa_shim::push(c1);
  aoa_shim::push(c2);
  aoa_shim::check(aoa_sub(x->ctx, c3->ct, c1->ct, c2->ct));
  aoa_shim::pull(c3);
}
inline cipher_t* ckks_sub(CKKSContext* x, cipher_t* c1, cipher_t* c2) {
  cipher_t* c3 = new cipher_t;
  ckks_sub(x, c3, c1, c2);
  return c3;
}
// ckks.h:164-172 (ckks.cpp:273-347)
inline void ckks_mul_without_rescale(CKKSContext* x, cipher_t* c3, cipher_t* c1, cipher_t* c2) {
  aoa_shim::ensure(x, c3);
  aoa_shim::push(c1);
  aoa_shim::push(c2);
  aoa_shim::check(aoa_hmult(x->ctx, c3->ct, c1->ct, c2->ct, aoa_shim::key(x->keys.evk, "evaluation key")));
  aoa_shim::pull(c3);
}
inline cipher_t* ckks_mul_without_rescale(CKKSContext* x, cipher_t* c1, cipher_t* c2) {
  cipher_t* c3 = new cipher_t;
  ckks_mul_without_rescale(x, c3, c1, c2);
  return c3;
}
inline void ckks_mul(CKKSContext* x, cipher_t* c3, cipher_t* c1, cipher_t* c2) {
  aoa_shim::ensure(x, c3);
  aoa_shim::push(c1);
  aoa_shim::push(c2);
  aoa_shim::check(
      aoa_hmult_relin_rescale(x->ctx, c3->ct, c1->ct, c2->ct, aoa_shim::key(x->keys.evk, "evaluation key")));
  aoa_shim::pull(c3);
}
inline cipher_t* ckks_mul(CKKSContext* x, cipher_t* c1, cipher_t* c2) {
  cipher_t* c3 = new cipher_t;
  ckks_mul(x, c3, c1, c2);
  return c3;
}
// ckks.h:310-313 (ckks.cpp:953-1040): keys by step, as CKKSKeychain holds them
inline void ckks_rotate_left(CKKSContext* x, cipher_t* c1, cipher_t* c2, int rotSlots) {
  aoa_shim::ensure(x, c1);
  aoa_shim::push(c2);
  aoa_shim::check(aoa_rotate(x->ctx, c1->ct, c2->ct, rotSlots, x->keys.rtk_left.at(rotSlots)->k));
  aoa_shim::pull(c1);
}
inline void ckks_rotate_right(CKKSContext* x, cipher_t* c1, cipher_t* c2, int rotSlots) {
  aoa_shim::ensure(x, c1);
  aoa_shim::push(c2);
  aoa_shim::check(aoa_rotate(x->ctx, c1->ct, c2->ct, -rotSlots, x->keys.rtk_right.at(rotSlots)->k));
  aoa_shim::pull(c1);
}
inline void ckks_conjugate(CKKSContext* x, cipher_t* c1, cipher_t* c2) {
  aoa_shim::ensure(x, c1);
  aoa_shim::push(c2);
  aoa_shim::check(aoa_conjugate(x->ctx, c1->ct, c2->ct, aoa_shim::key(x->keys.cjk, "conjugation key")));
  aoa_shim::pull(c1);
}
inline cipher_t* ckks_conjugate(CKKSContext* x, cipher_t* ct) {
  cipher_t* c = new cipher_t;
  ckks_conjugate(x, c, ct);
  return c;
}
