// Host-side check of the device modular arithmetic (aoa_b200/csrc/modarith.cuh),
// compiled by nvcc as host code: Barrett products for every modulus bit length
// 3..62 (extreme and random operands below 2^n), the Montgomery fallback for
// 63-bit moduli, against exact 128-bit arithmetic.  Prints "ok <count>".
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
  if (q >= 4 && q < (1ull << 62)) {
    const int n = 64 - __builtin_clzll(q);
    c.bar_sh = (uint64_t)(n - 2);
    c.bar_mu = (uint64_t)((one << (64 + n - 2)) / q);
  }
  return c;
}

int main() {
  std::mt19937_64 rng(11);
  long tests = 0, bad = 0;
  for (int n = 3; n <= 63; n++) {
    for (int t = 0; t < 400; t++) {
      uint64_t q = t == 0 ? (1ull << (n - 1)) | 1 : t == 1 ? (n == 64 ? ~0ull : (1ull << n) - 1)
                                                           : (1ull << (n - 1)) | (rng() & ((1ull << (n - 1)) - 1)) | 1;
      const PrimeConst P = constants(q);
      const uint64_t lim = (1ull << n) - 1;
      for (int r = 0; r < 100; r++) {
        uint64_t a, b;
        if (r == 0) a = b = lim;
        else if (r == 1) a = b = q - 1;
        else if (r < 30) { a = lim - (rng() & 3) * (lim > 8); b = lim - (rng() & 3) * (lim > 8); }
        else { a = rng() & lim; b = rng() & lim; }
        const uint64_t want = (uint64_t)(((unsigned __int128)a * b) % q);
        uint64_t got;
        if (n <= 62) {
          got = barrett_mul(a, b, q, P.bar_mu, (uint32_t)P.bar_sh);        // any a, b < 2^n
        } else {
          a %= q;                                                           // Montgomery: a, b < q
          b %= q;
          got = mul_mod(a, b, P);
          if (got != (uint64_t)(((unsigned __int128)a * b) % q)) bad++;
          tests++;
          continue;
        }
        tests++;
        if (got != want) bad++;
        if (a < q && b < q) {                                               // the dispatching entry point
          tests++;
          if (mul_mod(a, b, P) != want) bad++;
        }
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
