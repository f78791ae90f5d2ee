// Compositions of the hot operations that the reference's callers use for
// function approximation and logistic regression (aoa-ntt src/ckks/ckks.cpp:
// 423-455 inner products, 732-776 power, 778-811 polynomial evaluation by
// Horner's rule).  Each follows the reference's operation sequence and its
// metadata rules exactly (a cleared accumulator starts at level k-1 with scale
// 2^scalingfactor and keeps that scale through ckks_add), so the residues and
// the (level, scale, slots) of every result equal the reference's.
#include "aoa_internal.h"

using namespace aoa;

namespace aoa {
void hmult(Ctx& C, aoa_ct* out, aoa_ct* a, aoa_ct* b, const aoa_swk* evk, bool do_rescale);
}

namespace {

void ok(int status) {
  if (status != AOA_OK) throw AoaError(status, std::string(aoa_last_error()));
}

// a temporary ciphertext of the context (freed on scope exit)
struct TempCt {
  aoa_ctx* c;
  aoa_ct* ct = nullptr;
  explicit TempCt(aoa_ctx* ctx) : c(ctx) { ok(aoa_ct_create(ctx, &ct)); }
  ~TempCt() { aoa_ct_destroy(c, ct); }
  TempCt(const TempCt&) = delete;
  TempCt& operator=(const TempCt&) = delete;
};

// cipher_init / cipher_clear (cipher_t.cpp:3-21): zero residues, level k-1,
// scale 2^scalingfactor, the given slot count
void clear_ct(aoa_ctx* c, aoa_ct* ct, int slots) {
  const Engine& E = *c->c.E;
  AOA_CUDA(cudaMemsetAsync(ct->d, 0, (size_t)2 * E.k * E.N * 8, c->c.stream));
  ct->level = E.k - 1;
  ct->scale = E.scale_bits > 0 && E.scale_bits < 64 ? (1ull << E.scale_bits) : 1;
  ct->slots = slots;
  ct->domain = AOA_COEF;
}

void copy_ct(aoa_ctx* c, aoa_ct* dst, const aoa_ct* src) {
  const Engine& E = *c->c.E;
  AOA_CUDA(cudaMemcpyAsync(dst->d, src->d, (size_t)2 * E.k * E.N * 8, cudaMemcpyDeviceToDevice, c->c.stream));
  dst->level = src->level;
  dst->scale = src->scale;
  dst->slots = src->slots;
  dst->domain = src->domain;
}

}  // namespace

extern "C" {

// ckks_power (ckks.cpp:732-761): square-and-multiply from the lowest bit;
// the first factor is added to the cleared accumulator, later ones multiply
// it (HMult + relinearise + rescale); the running square is squared after
// every bit, the last one included.  x = 0 gives the noiseless encryption of
// 1 (c0 = the scale in every slot's constant term, c1 = 0); the reference
// encrypts 1 with its public key there.
int aoa_power(aoa_ctx* c, aoa_ct* out, aoa_ct* in, uint64_t x, const aoa_swk* evk) {
  if (!c || !out || !in) return fail(AOA_ERR_BAD_PARAM, "null argument");
  if (out == in) return fail(AOA_ERR_BAD_PARAM, "aoa_power: out must differ from in");
  return guarded([&] {
    clear_ct(c, out, in->slots);
    if (x == 0) {
      ok(aoa_add_const(c, out, out, 1.0));
      return;
    }
    TempCt aux(c);
    copy_ct(c, aux.ct, in);
    bool first = true;
    while (x > 0) {
      if (x & 1) {
        if (first) {
          ok(aoa_add(c, out, out, aux.ct));
          first = false;
        } else {
          hmult(c->c, out, out, aux.ct, evk, true);
        }
      }
      x >>= 1;
      hmult(c->c, aux.ct, aux.ct, aux.ct, evk, true);
    }
  });
}

// ckks_eval_polynomial (ckks.cpp:778-796), Horner's rule from the cleared
// accumulator: for i = n-1 .. 0: r = r * x (HMult + relinearise + rescale),
// r = r + coeffs[i] (constant at r's scale).
int aoa_eval_polynomial(aoa_ctx* c, aoa_ct* out, aoa_ct* x, const double* coeffs, int n, const aoa_swk* evk) {
  if (!c || !out || !x || (n > 0 && !coeffs)) return fail(AOA_ERR_BAD_PARAM, "null argument");
  if (out == x) return fail(AOA_ERR_BAD_PARAM, "aoa_eval_polynomial: out must differ from x");
  return guarded([&] {
    clear_ct(c, out, x->slots);
    for (int i = n - 1; i >= 0; i--) {
      hmult(c->c, out, out, x, evk, true);
      ok(aoa_add_const(c, out, out, coeffs[i]));
    }
  });
}

// ckks_inner_prod (ckks.cpp:423-441): sum_i a[i] * b[i] without rescale
// into the cleared accumulator (which keeps its scale through ckks_add),
// then one rescale.
int aoa_inner_prod(aoa_ctx* c, aoa_ct* out, aoa_ct* const* a, aoa_ct* const* b, int size, const aoa_swk* evk) {
  if (!c || !out || size < 1 || !a || !b) return fail(AOA_ERR_BAD_PARAM, "bad argument");
  return guarded([&] {
    TempCt aux(c);
    clear_ct(c, out, a[0]->slots);
    for (int i = 0; i < size; i++) {
      if (a[i]->slots != b[i]->slots)
        throw AoaError(AOA_ERR_SLOT_MISMATCH, "Ciphertexts must have the same number of slots.");
      hmult(c->c, aux.ct, a[i], b[i], evk, false);
      ok(aoa_add(c, out, out, aux.ct));
    }
    ok(aoa_rescale(c, out));
  });
}

// ckks_inner_prod with real weights (ckks.cpp:443-455): a[i] * w[i] through
// ckks_mul_without_rescale(ct, double), accumulated, one rescale.
int aoa_inner_prod_const(aoa_ctx* c, aoa_ct* out, aoa_ct* const* a, const double* w, int size) {
  if (!c || !out || size < 1 || !a || !w) return fail(AOA_ERR_BAD_PARAM, "bad argument");
  return guarded([&] {
    TempCt aux(c);
    clear_ct(c, out, a[0]->slots);
    for (int i = 0; i < size; i++) {
      ok(aoa_mul_const(c, aux.ct, a[i], w[i], 0));
      ok(aoa_add(c, out, out, aux.ct));
    }
    ok(aoa_rescale(c, out));
  });
}

}  // extern "C"
