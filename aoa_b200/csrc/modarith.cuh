// Modular arithmetic for 64-bit RNS residues on sm_100a CUDA cores.
//
// The reference reduces every product with a Barrett reduction specialised to
// its table primes (aoa-ntt src/cuda/htrans/common.cu:174-193, 257-291).  Any
// exact reduction yields the same canonical residues, so this engine uses the
// cheapest exact form per use:
//   * Shoup multiplication by a precomputed constant w with w' = floor(w 2^64/q)
//     (twiddles, CRT constants): one mul.hi and two mul.lo;
//   * Montgomery REDC for products of two variable residues;
//   * two Shoup steps to fold a 128-bit accumulator (basis conversion sums).
// All routines require q < 2^63 and return canonical values in [0, q)
// unless named *_lazy.
#pragma once
#include <cstdint>

#define AOA_HD __host__ __device__ __forceinline__

// Per-prime constants, one entry per prime of the Q|B list.
struct PrimeConst {
  uint64_t q;
  uint64_t qinv_neg;   // -q^-1 mod 2^64       (Montgomery)
  uint64_t r2;         // 2^128 mod q           (Montgomery R^2)
  uint64_t r1;         // 2^64 mod q
  uint64_t r1_sh;      // floor(r1 * 2^64 / q)  (Shoup companion of r1)
  uint64_t one_sh;     // floor(2^64 / q)       (Shoup companion of 1)
  uint64_t ninv, ninv_sh;          // N^-1 mod q
  uint64_t ninv_w1, ninv_w1_sh;    // N^-1 * psi^-bitrev(1) mod q (last inverse stage)
};

struct ShoupW {      // twiddle or constant w with its Shoup companion
  uint64_t w, wp;
};

AOA_HD uint64_t mulhi64(uint64_t a, uint64_t b) {
#ifdef __CUDA_ARCH__
  return __umul64hi(a, b);
#else
  return (uint64_t)(((unsigned __int128)a * b) >> 64);
#endif
}

AOA_HD uint64_t add_mod(uint64_t a, uint64_t b, uint64_t q) {
  uint64_t s = a + b;
  return s >= q ? s - q : s;
}

AOA_HD uint64_t sub_mod(uint64_t a, uint64_t b, uint64_t q) {
  return a >= b ? a - b : a + (q - b);
}

AOA_HD uint64_t neg_mod(uint64_t a, uint64_t q) { return a ? q - a : 0; }

// a * w mod q for any a < 2^64, w < q, wp = floor(w 2^64 / q); result in [0, 2q).
AOA_HD uint64_t shoup_lazy(uint64_t a, uint64_t w, uint64_t wp, uint64_t q) {
  uint64_t t = mulhi64(a, wp);
  return a * w - t * q;
}

AOA_HD uint64_t shoup(uint64_t a, uint64_t w, uint64_t wp, uint64_t q) {
  uint64_t r = shoup_lazy(a, w, wp, q);
  return r >= q ? r - q : r;
}

AOA_HD uint64_t shoup(uint64_t a, ShoupW w, uint64_t q) { return shoup(a, w.w, w.wp, q); }

// Montgomery REDC of x = hi*2^64 + lo with x < q*2^64: x * 2^-64 mod q.
AOA_HD uint64_t redc(uint64_t lo, uint64_t hi, uint64_t q, uint64_t qinv_neg) {
  uint64_t m = lo * qinv_neg;
  uint64_t t = hi + mulhi64(m, q) + (lo != 0);
  return t >= q ? t - q : t;
}

// a * b mod q for a, b < q (two REDC steps through R^2).
AOA_HD uint64_t mul_mod(uint64_t a, uint64_t b, const PrimeConst& P) {
  uint64_t lo = a * b, hi = mulhi64(a, b);
  uint64_t t = redc(lo, hi, P.q, P.qinv_neg);          // a b R^-1
  return redc(t * P.r2, mulhi64(t, P.r2), P.q, P.qinv_neg);   // a b
}

// a * b * 2^-64 mod q (one REDC) for a, b < q.
AOA_HD uint64_t mont_mul(uint64_t a, uint64_t b, uint64_t q, uint64_t qinv_neg) {
  return redc(a * b, mulhi64(a, b), q, qinv_neg);
}

// Exact reduction of an arbitrary 128-bit value hi*2^64 + lo modulo q.
AOA_HD uint64_t reduce128(uint64_t lo, uint64_t hi, const PrimeConst& P) {
  uint64_t h = shoup(hi, P.r1, P.r1_sh, P.q);     // hi * 2^64 mod q
  uint64_t l = shoup(lo, 1, P.one_sh, P.q);       // lo mod q
  return add_mod(h, l, P.q);
}

// 128-bit multiply-accumulate: (hi:lo) += a * b
AOA_HD void mac128(uint64_t& lo, uint64_t& hi, uint64_t a, uint64_t b) {
#ifdef __CUDA_ARCH__
  uint64_t pl = a * b, ph = __umul64hi(a, b);
  asm("add.cc.u64 %0, %0, %2;\n\taddc.u64 %1, %1, %3;" : "+l"(lo), "+l"(hi) : "l"(pl), "l"(ph));
#else
  unsigned __int128 s = ((unsigned __int128)hi << 64 | lo) + (unsigned __int128)a * b;
  lo = (uint64_t)s; hi = (uint64_t)(s >> 64);
#endif
}
