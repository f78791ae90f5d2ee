// Host-side check of the device modular arithmetic (aoa_b200/csrc/modarith.cuh),
// compiled by nvcc as host code: Barrett products for every modulus bit length
// 34..62 (extreme and random operands below 2^n), the fused two-product
// reduction for 34..61 bits, the Montgomery products used outside that range
// (3..33 and 63 bits), and for moduli q = 1 mod 2^32 (34..60 bits) the Barrett
// reduction and exact Shoup product whose quotient times q takes one 32-bit
// multiply, against exact 128-bit arithmetic.  Prints "ok <count>".
#include <cstdio>
#include <random>

#include "../aoa_b200/csrc/modarith.cuh"

static PrimeConst constants(uint64_t q) {
  PrimeConst c{};
  c.q = q;
  uint64_t x = q;
  for (int i = 0; i < 6; i++) x *= 2 - q * x;
  c.qinv_neg = (uint64_t)0 - x;
  const unsigned __int128 one = 1;
  c.r1 = (uint64_t)((one << 64) % q);
  c.r2 = (uint64_t)(((unsigned __int128)c.r1 * c.r1) % q);
  if (q >= (1ull << 33) && q < (1ull << 62)) {
    const int n = 64 - __builtin_clzll(q);
    c.bar_sh = (uint64_t)(n - 2);
    c.bar_mu = (uint64_t)((one << (64 + n - 2)) / q);
  }
  return c;
}

int main() {
  std::mt19937_64 rng(11);
  long tests = 0, bad = 0;
  auto check = [&](uint64_t got, uint64_t want) {
    tests++;
    if (got != want) bad++;
  };
  for (int n = 3; n <= 63; n++) {
    for (int t = 0; t < 300; t++) {
      const uint64_t q = t == 0 ? (1ull << (n - 1)) | 1 : t == 1 ? (1ull << n) - 1
                                                       : (1ull << (n - 1)) | (rng() & ((1ull << (n - 1)) - 1)) | 1;
      const PrimeConst P = constants(q);
      const uint64_t lim = (1ull << n) - 1;
      auto pick = [&](int r) -> uint64_t {
        if (r == 0) return lim;
        if (r == 1) return q - 1;
        if (r < 30) return lim - (rng() & 3) * (lim > 8);
        return rng() & lim;
      };
      for (int r = 0; r < 100; r++) {
        uint64_t a = pick(r), b = pick(r), c = pick(r), d = pick(r);
        if (P.bar_sh) {                                                     // any operands below 2^n
          check(barrett_mul(a, b, q, P.bar_mu, (uint32_t)P.bar_sh), (uint64_t)(((unsigned __int128)a * b) % q));
          if (n <= 61)
            check(barrett_mul_add2(a, b, c, d, q, P.bar_mu, (uint32_t)P.bar_sh),
                  (uint64_t)((((unsigned __int128)a * b) % q + ((unsigned __int128)c * d) % q) % q));
        }
        a %= q;                                                             // the entry point: a, b < q
        b %= q;
        check(mul_mod(a, b, P), (uint64_t)(((unsigned __int128)a * b) % q));
      }
    }
  }
  for (int n = 34; n <= 60; n++) {                                      // q = q1 2^32 + 1
    for (int t = 0; t < 100; t++) {
      const uint64_t hi = t == 0 ? (1ull << (n - 33)) : t == 1 ? (1ull << (n - 32)) - 1
                                                       : (1ull << (n - 33)) | (rng() & ((1ull << (n - 33)) - 1));
      const uint64_t q = (hi << 32) | 1;
      const PrimeConst P = constants(q);
      const uint64_t lim = (1ull << n) - 1;
      for (int r = 0; r < 100; r++) {
        const uint64_t a = r == 0 ? lim : rng() & lim, b = r == 0 ? lim : rng() & lim;
        const uint64_t t64 = rng();
        check(mul_q1(t64, q), t64 * q);
        const unsigned __int128 ab = (unsigned __int128)a * b;
        check(barrett_wide_q1((uint64_t)ab, (uint64_t)(ab >> 64), q, P.bar_mu, (uint32_t)P.bar_sh),
              (uint64_t)(ab % q));
        const uint64_t w = r == 1 ? q - 1 : rng() % q;
        const uint64_t wp = (uint64_t)(((unsigned __int128)w << 64) / q);
        const uint64_t x = r == 2 ? ~0ull : rng();                        // any 64-bit operand
        check(shoup_q1(x, w, wp, q), (uint64_t)(((unsigned __int128)x * w) % q));
      }
    }
  }
  if (bad) {
    printf("bad %ld of %ld\n", bad, tests);
    return 1;
  }
  printf("ok %ld\n", tests);
  return 0;
}
