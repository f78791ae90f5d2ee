// Modular arithmetic for 64-bit RNS residues on sm_100a CUDA cores.
//
// The reference reduces every product with a Barrett reduction specialised to
// its table primes (aoa-ntt src/cuda/htrans/common.cu:174-193, 257-291).  Any
// exact reduction yields the same canonical residues, so this engine uses the
// cheapest exact form per use:
//   * Shoup multiplication by a precomputed constant w with w' = floor(w 2^64/q)
//     (twiddles, CRT constants): one mul.hi and two mul.lo;
//   * Barrett multiplication with a 64-bit quotient estimate for products of
//     two variable residues (2^33 <= q < 2^62), Montgomery REDC otherwise;
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
  uint64_t bar_mu;     // floor(2^(64+s) / q), s = bar_sh       (Barrett, 2^33 <= q < 2^62)
  uint64_t bar_sh;     // bit length of q minus 2; 0 outside that range (Montgomery instead)
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

// Shoup product for the limb transforms, which are bound by the integer
// multiply pipe, written as 32 x 32-bit multiply-adds.  With y = y1 2^32 + y0
// and wp = p1 2^32 + p0, the quotient is estimated from the three high partial
// products, t' = y1 p1 + hi(y0 p1) + hi(y1 p0): the dropped terms (the low
// words of the cross products and y0 p0) are below 3 * 2^64, so t - 2 <= t'
// <= t for t = floor(y wp / 2^64), and the remainder y w - t' q, formed as
// y w + t' (2^64 - q) mod 2^64 (nq = 2^64 - q) with its high word summed in
// 32 bits, lies in [0, 4q).
__device__ __forceinline__ uint64_t shoup_lazy_mad3(uint64_t y, uint64_t w, uint64_t wp, uint64_t nq) {
  uint64_t r;
#ifdef __CUDA_ARCH__
  asm("{\n\t"
      ".reg .u32 y0, y1, w0, w1, p0, p1, n0, n1, a1, b1, t0, t1, r0, r1;\n\t"
      ".reg .u64 S, T, R;\n\t"
      "mov.b64 {y0, y1}, %1;\n\t"
      "mov.b64 {w0, w1}, %2;\n\t"
      "mov.b64 {p0, p1}, %3;\n\t"
      "mov.b64 {n0, n1}, %4;\n\t"
      "mul.hi.u32 a1, y0, p1;\n\t"
      "mul.hi.u32 b1, y1, p0;\n\t"
      "cvt.u64.u32 S, a1;\n\t"
      "mad.wide.u32 T, y1, p1, S;\n\t"
      "mov.b64 {t0, t1}, T;\n\t"
      "add.cc.u32 t0, t0, b1;\n\t"
      "addc.u32 t1, t1, 0;\n\t"
      "mul.wide.u32 R, y0, w0;\n\t"
      "mad.wide.u32 R, t0, n0, R;\n\t"
      "mov.b64 {r0, r1}, R;\n\t"
      "mad.lo.u32 r1, y0, w1, r1;\n\t"
      "mad.lo.u32 r1, y1, w0, r1;\n\t"
      "mad.lo.u32 r1, t0, n1, r1;\n\t"
      "mad.lo.u32 r1, t1, n0, r1;\n\t"
      "mov.b64 %0, {r0, r1};\n\t"
      "}"
      : "=l"(r)
      : "l"(y), "l"(w), "l"(wp), "l"(nq));
#else
  r = y * w + mulhi64(y, wp) * nq;
#endif
  return r;
}

// The same product for primes whose low 32-bit word is 1 (q = q1 2^32 + 1,
// q = 1 mod 2^32): t' q = t' + (t'_0 q1) 2^32 mod 2^64, so the remainder
// y w - t' q is y0 w0 - t' + (y0 w1 + y1 w0 - t'_0 q1) 2^32 mod 2^64, one wide
// and three 32-bit multiplies instead of two wide and four (22 instead of 28
// multiply-pipe cycles per product).  Same quotient, same range [0, 4q).
__device__ __forceinline__ uint64_t shoup_lazy_mad3_q1(uint64_t y, uint64_t w, uint64_t wp, uint64_t q) {
  uint64_t r;
#ifdef __CUDA_ARCH__
  const uint32_t nq1 = 0u - (uint32_t)(q >> 32);   // -q1 mod 2^32
  asm("{\n\t"
      ".reg .u32 y0, y1, w0, w1, p0, p1, a1, b1, t0, t1, r0, r1;\n\t"
      ".reg .u64 S, T, R;\n\t"
      "mov.b64 {y0, y1}, %1;\n\t"
      "mov.b64 {w0, w1}, %2;\n\t"
      "mov.b64 {p0, p1}, %3;\n\t"
      "mul.hi.u32 a1, y0, p1;\n\t"
      "mul.hi.u32 b1, y1, p0;\n\t"
      "cvt.u64.u32 S, a1;\n\t"
      "mad.wide.u32 T, y1, p1, S;\n\t"
      "mov.b64 {t0, t1}, T;\n\t"
      "add.cc.u32 t0, t0, b1;\n\t"
      "addc.u32 t1, t1, 0;\n\t"
      "mul.wide.u32 R, y0, w0;\n\t"
      "mov.b64 {r0, r1}, R;\n\t"
      "sub.cc.u32 r0, r0, t0;\n\t"
      "subc.u32 r1, r1, t1;\n\t"
      "mad.lo.u32 r1, y0, w1, r1;\n\t"
      "mad.lo.u32 r1, y1, w0, r1;\n\t"
      "mad.lo.u32 r1, t0, %4, r1;\n\t"
      "mov.b64 %0, {r0, r1};\n\t"
      "}"
      : "=l"(r)
      : "l"(y), "l"(w), "l"(wp), "r"(nq1));
#else
  r = y * w - mulhi64(y, wp) * q;
#endif
  return r;
}

AOA_HD uint64_t shoup(uint64_t a, uint64_t w, uint64_t wp, uint64_t q) {
  uint64_t r = shoup_lazy(a, w, wp, q);
  return r >= q ? r - q : r;
}

AOA_HD uint64_t shoup(uint64_t a, ShoupW w, uint64_t q) { return shoup(a, w.w, w.wp, q); }

// t q mod 2^64 for q = q1 2^32 + 1 (q = 1 mod 2^32): t + (t_0 q1) 2^32, one
// 32-bit multiply instead of a wide one and two 32-bit ones.
AOA_HD uint64_t mul_q1(uint64_t t, uint64_t q) {
  return t + ((uint64_t)((uint32_t)t * (uint32_t)(q >> 32)) << 32);
}

// Exact Shoup product a w mod q in [0, q) for any a < 2^64 and q = 1 mod 2^32.
AOA_HD uint64_t shoup_q1(uint64_t a, uint64_t w, uint64_t wp, uint64_t q) {
  const uint64_t r = a * w - mul_q1(mulhi64(a, wp), q);
  return r >= q ? r - q : r;
}

// Montgomery REDC of x = hi*2^64 + lo with x < q*2^64: x * 2^-64 mod q.
AOA_HD uint64_t redc(uint64_t lo, uint64_t hi, uint64_t q, uint64_t qinv_neg) {
  uint64_t m = lo * qinv_neg;
  uint64_t t = hi + mulhi64(m, q) + (lo != 0);
  return t >= q ? t - q : t;
}

// x = hi 2^64 + lo mod q for x < 2^(64+s), q of bit length n in [34, 62],
// s = n - 2, by Barrett's method with a 64-bit quotient estimate:
// x1 = floor(x / 2^s) < 2^64 and mu = floor(2^(64+s) / q) < 2^63; the
// estimate qh = floor(x1 mu / 2^64) satisfies x/q - 2.5 < qh <= x/q (the
// truncations of x1 and mu cost < x / 2^(64+s) + 2^s/q <= 1.5, the final floor
// < 1), so r = x - qh q lies in [0, 3q) and is exact in 64 bits.  With
// s >= 32, x1 is two 32-bit funnel shifts of the words 1..3 of x.
AOA_HD uint32_t funnel_r32(uint32_t lo, uint32_t hi, uint32_t sh) {   // low word of (hi:lo) >> (sh % 32)
#ifdef __CUDA_ARCH__
  return __funnelshift_r(lo, hi, sh);
#else
  return (uint32_t)((((uint64_t)hi << 32) | lo) >> (sh & 31));
#endif
}

AOA_HD uint64_t barrett_wide(uint64_t lo, uint64_t hi, uint64_t q, uint64_t mu, uint32_t s) {
  const uint32_t t = s - 32;
  const uint32_t x1lo = funnel_r32((uint32_t)(lo >> 32), (uint32_t)hi, t);
  const uint32_t x1hi = funnel_r32((uint32_t)hi, (uint32_t)(hi >> 32), t);
  const uint64_t x1 = ((uint64_t)x1hi << 32) | x1lo;
  uint64_t r = lo - mulhi64(x1, mu) * q;
  r = r >= q ? r - q : r;
  return r >= q ? r - q : r;
}

// barrett_wide for q = 1 mod 2^32 (the quotient times q through mul_q1).
AOA_HD uint64_t barrett_wide_q1(uint64_t lo, uint64_t hi, uint64_t q, uint64_t mu, uint32_t s) {
  const uint32_t t = s - 32;
  const uint32_t x1lo = funnel_r32((uint32_t)(lo >> 32), (uint32_t)hi, t);
  const uint32_t x1hi = funnel_r32((uint32_t)hi, (uint32_t)(hi >> 32), t);
  const uint64_t x1 = ((uint64_t)x1hi << 32) | x1lo;
  uint64_t r = lo - mul_q1(mulhi64(x1, mu), q);
  r = r >= q ? r - q : r;
  return r >= q ? r - q : r;
}

// a * b mod q for a, b < 2^n (then a b < 2^2n <= 2^(64+s) for n <= 62).
AOA_HD uint64_t barrett_mul(uint64_t a, uint64_t b, uint64_t q, uint64_t mu, uint32_t s) {
  return barrett_wide(a * b, mulhi64(a, b), q, mu, s);
}

// (a b + c d) mod q for a, b, c, d < 2^n with n <= 61: the 128-bit sum is
// below 2^(2n+1) <= 2^(64+s), so one reduction serves both products.
AOA_HD uint64_t barrett_mul_add2(uint64_t a, uint64_t b, uint64_t c, uint64_t d, uint64_t q, uint64_t mu,
                                 uint32_t s) {
  uint64_t lo = a * b, hi = mulhi64(a, b);
  const uint64_t l2 = c * d;
  hi += mulhi64(c, d);
  lo += l2;
  hi += lo < l2;
  return barrett_wide(lo, hi, q, mu, s);
}

// a * b mod q for a, b < q: Barrett for 2^33 <= q < 2^62, else two REDC steps through R^2.
AOA_HD uint64_t mul_mod(uint64_t a, uint64_t b, const PrimeConst& P) {
  if (P.bar_sh) return barrett_mul(a, b, P.q, P.bar_mu, (uint32_t)P.bar_sh);
  uint64_t lo = a * b, hi = mulhi64(a, b);
  uint64_t t = redc(lo, hi, P.q, P.qinv_neg);          // a b R^-1
  return redc(t * P.r2, mulhi64(t, P.r2), P.q, P.qinv_neg);   // a b
}

// a * b * 2^-64 mod q (one REDC) for a, b < q.
AOA_HD uint64_t mont_mul(uint64_t a, uint64_t b, uint64_t q, uint64_t qinv_neg) {
  return redc(a * b, mulhi64(a, b), q, qinv_neg);
}

// x mod q for x < p, another prime: one conditional subtraction when p < 2q
// (primes of one bit length), else a Shoup reduction.
AOA_HD uint64_t cross_mod(uint64_t x, uint64_t p, const PrimeConst& P) {
  if (p < 2 * P.q) return x >= P.q ? x - P.q : x;
  return shoup(x, 1, P.one_sh, P.q);
}

// Exact reduction of an arbitrary 128-bit value hi*2^64 + lo modulo q.
AOA_HD uint64_t reduce128(uint64_t lo, uint64_t hi, const PrimeConst& P) {
  uint64_t h = shoup(hi, P.r1, P.r1_sh, P.q);     // hi * 2^64 mod q
  uint64_t l = shoup(lo, 1, P.one_sh, P.q);       // lo mod q
  return add_mod(h, l, P.q);
}

// 128-bit multiply-accumulate: (hi:lo) += a * b, as three 32-bit carry chains
// over the four partial products (a0 b0 + a1 b1 2^64, then a0 b1 2^32, a1 b0 2^32).
AOA_HD void mac128(uint64_t& lo, uint64_t& hi, uint64_t a, uint64_t b) {
#ifdef __CUDA_ARCH__
  uint32_t r0 = (uint32_t)lo, r1 = (uint32_t)(lo >> 32), r2 = (uint32_t)hi, r3 = (uint32_t)(hi >> 32);
  const uint32_t a0 = (uint32_t)a, a1 = (uint32_t)(a >> 32), b0 = (uint32_t)b, b1 = (uint32_t)(b >> 32);
  asm("mad.lo.cc.u32 %0, %4, %6, %0;\n\t"
      "madc.hi.cc.u32 %1, %4, %6, %1;\n\t"
      "madc.lo.cc.u32 %2, %5, %7, %2;\n\t"
      "madc.hi.u32 %3, %5, %7, %3;\n\t"
      "mad.lo.cc.u32 %1, %4, %7, %1;\n\t"
      "madc.hi.cc.u32 %2, %4, %7, %2;\n\t"
      "addc.u32 %3, %3, 0;\n\t"
      "mad.lo.cc.u32 %1, %5, %6, %1;\n\t"
      "madc.hi.cc.u32 %2, %5, %6, %2;\n\t"
      "addc.u32 %3, %3, 0;"
      : "+r"(r0), "+r"(r1), "+r"(r2), "+r"(r3)
      : "r"(a0), "r"(a1), "r"(b0), "r"(b1));
  lo = ((uint64_t)r1 << 32) | r0;
  hi = ((uint64_t)r3 << 32) | r2;
#else
  unsigned __int128 s = ((unsigned __int128)hi << 64 | lo) + (unsigned __int128)a * b;
  lo = (uint64_t)s; hi = (uint64_t)(s >> 64);
#endif
}
