// Key generation on the device from given randomness (CKKSKeychain,
// aoa-ntt src/ckks/ckkskeys.cpp:101-191; aoa-dgt src/keys.cpp): the sampler's
// draws (uniform a, Gaussian e) are inputs, so keys are reproducible and equal
// the reference's for the same draws.
//
//   switching key for s1 under s2:  b = rho(s1) + e - a s2,  a   over QB
//   (ckks_new_evk with s1 = s^2, ckks_new_rtk with s1 = s(X^g), ckks_new_cjk);
//   rho multiplies Q residue i by [B]_{q_i} and zeroes the B residues
//   (ckks_rho, aoa-ntt src/cuda/manager.cu:149-176);
//   public key:  b = e - a s,  a  over Q  (ckks_new_pk).
#include "aoa_internal.h"

using namespace aoa;

namespace {

// out[r] = rho(s1)[r] + e (coefficients); rho factor [B]_{q_r} on Q limbs, 0 on B.
__global__ void keygen_prep(uint64_t* out, const uint64_t* __restrict__ s1, const int64_t* __restrict__ e,
                            const ShoupW* __restrict__ bmodq, int k, long N, const PrimeConst* __restrict__ pc) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  const int r = blockIdx.y;
  const uint64_t q = pc[r].q;
  const int64_t ev = e[i];
  uint64_t v = ev >= 0 ? (uint64_t)ev : q - (uint64_t)(-ev);
  if (s1 && r < k) v = add_mod(v, shoup(s1[(long)r * N + i], bmodq[r], q), q);
  out[(long)r * N + i] = v;
}

uint64_t* ensure(Ctx& C, size_t need) {
  if (C.enc_bytes < need) {
    if (C.enc) AOA_CUDA(cudaFreeAsync(C.enc, C.stream));
    C.enc = nullptr;
    C.enc_bytes = 0;
    if (cudaMallocAsync(&C.enc, need, C.stream) != cudaSuccess) {
      cudaGetLastError();
      throw AoaError(AOA_ERR_OOM, "key-generation buffer allocation failed");
    }
    C.enc_bytes = need;
  }
  return (uint64_t*)C.enc;
}

// b (nl limbs, transform domain tk) -= a * s over limbs 0..nl-1; t is scratch.
void sub_product(Ctx& C, int tk, uint64_t* b, const uint64_t* a, const uint64_t* s, uint64_t* t, int nl) {
  const Engine& E = *C.E;
  if (tk == AOA_DGT) gi_mul_op(E, t, 0, a, 0, s, 0, 0, nl, 1, C.stream);
  else ew_binary_op(E, t, 0, a, 0, s, 0, 2, 0, nl, 1, C.stream);
  ew_binary_op(E, b, 0, b, 0, t, 0, 1, 0, nl, 1, C.stream);
}

dim3 limb_grid(const Engine& E, int nl) { return dim3((unsigned)((E.N + 255) / 256), (unsigned)nl); }

}  // namespace

extern "C" {

// Switching key (b, a) for s1 under s2 in the context's transform domain.
// d_s1, d_s2: [k+kl][N] residues in coefficients (d_s1 may be NULL for 0);
// d_a: [k+kl][N] uniform residues in a_domain; d_e: N signed noise values.
int aoa_swk_generate(aoa_ctx* c, const uint64_t* d_s1, const uint64_t* d_s2, const uint64_t* d_a, int a_domain,
                     const int64_t* d_e, aoa_swk** out) {
  if (!c || !d_s2 || !d_a || !d_e || !out) return fail(AOA_ERR_BAD_PARAM, "null argument");
  return guarded([&] {
    Ctx& C = c->c;
    const Engine& E = *C.E;
    const int tk = C.transform, nqb = E.nprimes;
    if (a_domain != AOA_COEF && a_domain != tk)
      throw AoaError(AOA_ERR_BAD_PARAM, "a must be in coefficients or in the context's transform domain");
    const size_t half = (size_t)nqb * E.N;
    uint64_t* S = ensure(C, 2 * half * 8);                // s2 copy, product scratch
    aoa_swk* k = new aoa_swk();
    if (cudaMallocAsync(&k->d, 2 * half * 8, C.stream) != cudaSuccess) {
      cudaGetLastError();
      delete k;
      throw AoaError(AOA_ERR_OOM, "key allocation failed");
    }
    k->domain = tk;
    uint64_t* B = k->d;
    uint64_t* A = k->d + half;
    keygen_prep<<<limb_grid(E, nqb), 256, 0, C.stream>>>(B, d_s1, d_e, E.rns.bmodq, E.k, E.N, E.d_pc);
    note_launch();
    AOA_CHECK_LAUNCH();
    AOA_CUDA(cudaMemcpyAsync(A, d_a, half * 8, cudaMemcpyDeviceToDevice, C.stream));
    AOA_CUDA(cudaMemcpyAsync(S, d_s2, half * 8, cudaMemcpyDeviceToDevice, C.stream));
    xform(E, tk, B, 1, 0, nqb, nqb, true, C.stream);
    xform(E, tk, S, 1, 0, nqb, nqb, true, C.stream);
    if (a_domain == AOA_COEF) xform(E, tk, A, 1, 0, nqb, nqb, true, C.stream);
    sub_product(C, tk, B, A, S, S + half, nqb);
    AOA_CUDA(cudaStreamSynchronize(C.stream));
    *out = k;
  });
}

// Public key (b, a) = (e - a s, a) over the Q primes as a ciphertext at level
// k-1 in the context's transform domain.  d_s: [k][N] (or longer) secret
// residues in coefficients; d_a: [k][N] uniform residues in a_domain.
int aoa_pk_generate(aoa_ctx* c, aoa_ct* out, const uint64_t* d_s, const uint64_t* d_a, int a_domain,
                    const int64_t* d_e) {
  if (!c || !out || !d_s || !d_a || !d_e) return fail(AOA_ERR_BAD_PARAM, "null argument");
  return guarded([&] {
    Ctx& C = c->c;
    const Engine& E = *C.E;
    const int tk = C.transform, k = E.k;
    if (a_domain != AOA_COEF && a_domain != tk)
      throw AoaError(AOA_ERR_BAD_PARAM, "a must be in coefficients or in the context's transform domain");
    const size_t half = (size_t)k * E.N;
    uint64_t* S = ensure(C, 2 * half * 8);
    uint64_t* B = out->d;
    uint64_t* A = out->d + half;
    keygen_prep<<<limb_grid(E, k), 256, 0, C.stream>>>(B, nullptr, d_e, E.rns.bmodq, k, E.N, E.d_pc);
    note_launch();
    AOA_CHECK_LAUNCH();
    AOA_CUDA(cudaMemcpyAsync(A, d_a, half * 8, cudaMemcpyDeviceToDevice, C.stream));
    AOA_CUDA(cudaMemcpyAsync(S, d_s, half * 8, cudaMemcpyDeviceToDevice, C.stream));
    xform(E, tk, B, 1, 0, k, k, true, C.stream);
    xform(E, tk, S, 1, 0, k, k, true, C.stream);
    if (a_domain == AOA_COEF) xform(E, tk, A, 1, 0, k, k, true, C.stream);
    sub_product(C, tk, B, A, S, S + half, k);
    out->level = k - 1;
    out->domain = tk;
    out->slots = 0;
  });
}

// Secret-key transforms for the switching keys, over `nlimbs` limbs of
// coefficient-domain residues ([nlimbs][N]):
//   square   s -> s^2                      (ckks_new_mtk, ckkskeys.cpp:101-131)
//   galois   s -> s(X^g), g odd mod 2N     (rotation: g = 5^r, ckkskeys.cpp:146-181;
//                                           conjugation: g = 2N - 1, ckkskeys.cpp:183-191)
int aoa_secret_square(aoa_ctx* c, const uint64_t* d_s, uint64_t* d_out, int nlimbs) {
  if (!c || !d_s || !d_out) return fail(AOA_ERR_BAD_PARAM, "null argument");
  return guarded([&] {
    Ctx& C = c->c;
    const Engine& E = *C.E;
    if (nlimbs < 1 || nlimbs > E.nprimes) throw AoaError(AOA_ERR_BAD_PARAM, "nlimbs out of range");
    const int tk = C.transform;
    uint64_t* S = ensure(C, (size_t)nlimbs * E.N * 8);
    AOA_CUDA(cudaMemcpyAsync(S, d_s, (size_t)nlimbs * E.N * 8, cudaMemcpyDeviceToDevice, C.stream));
    xform(E, tk, S, 1, 0, nlimbs, nlimbs, true, C.stream);
    if (tk == AOA_DGT) gi_mul_op(E, d_out, 0, S, 0, S, 0, 0, nlimbs, 1, C.stream);
    else ew_binary_op(E, d_out, 0, S, 0, S, 0, 2, 0, nlimbs, 1, C.stream);
    xform(E, tk, d_out, 1, 0, nlimbs, nlimbs, false, C.stream);
  });
}

int aoa_secret_galois(aoa_ctx* c, const uint64_t* d_s, uint64_t* d_out, long galois, int nlimbs) {
  if (!c || !d_s || !d_out) return fail(AOA_ERR_BAD_PARAM, "null argument");
  return guarded([&] {
    const Engine& E = *c->c.E;
    if (nlimbs < 1 || nlimbs > E.nprimes) throw AoaError(AOA_ERR_BAD_PARAM, "nlimbs out of range");
    if (!(galois & 1)) throw AoaError(AOA_ERR_BAD_PARAM, "the Galois element must be odd");
    if (d_s == d_out) throw AoaError(AOA_ERR_BAD_PARAM, "input and output must differ");
    const long g = ((galois % (2 * E.N)) + 2 * E.N) % (2 * E.N);
    automorph_coef_op(E, d_out, d_s, 0, g, nlimbs, 1, c->c.stream);
  });
}

}  // extern "C"
