// Host-side number theory for engine set-up: primality, primitive roots,
// modular inverses and Shoup companions.  Replaces the NTL ZZ/RR calls of the
// reference precompute (aoa-ntt src/cuda/manager.cu:566-759,
// src/cuda/htrans/common.cu:485-538, src/cuda/htrans/ntt.cu:685-1023).
#include <algorithm>
#include <vector>

#include "aoa_internal.h"

namespace aoa {

typedef unsigned __int128 u128;

uint64_t h_mulmod(uint64_t a, uint64_t b, uint64_t q) { return (uint64_t)((u128)a * b % q); }

uint64_t h_powmod(uint64_t a, uint64_t e, uint64_t q) {
  uint64_t r = 1 % q;
  a %= q;
  for (; e; e >>= 1) {
    if (e & 1) r = h_mulmod(r, a, q);
    a = h_mulmod(a, a, q);
  }
  return r;
}

uint64_t h_invmod(uint64_t a, uint64_t q) {   // q prime
  return h_powmod(a % q, q - 2, q);
}

// floor(w * 2^64 / q), w < q
uint64_t h_shoup_companion(uint64_t w, uint64_t q) { return (uint64_t)(((u128)w << 64) / q); }

bool h_is_prime(uint64_t n) {
  if (n < 2) return false;
  const uint64_t bases[] = {2, 3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37};
  for (uint64_t p : bases)
    if (n % p == 0) return n == p;
  uint64_t d = n - 1;
  int s = 0;
  while (!(d & 1)) { d >>= 1; ++s; }
  for (uint64_t a : bases) {
    uint64_t x = h_powmod(a, d, n);
    if (x == 1 || x == n - 1) continue;
    bool witness = true;
    for (int i = 1; i < s && witness; i++) {
      x = h_mulmod(x, x, n);
      if (x == n - 1) witness = false;
    }
    if (witness) return false;
  }
  return true;
}

static uint64_t gcd_u64(uint64_t a, uint64_t b) {
  while (b) { uint64_t t = a % b; a = b; b = t; }
  return a;
}

// Pollard rho with Floyd cycle detection; n composite and odd.
static uint64_t pollard(uint64_t n) {
  for (uint64_t c = 1;; ++c) {
    uint64_t x = 2, y = 2, d = 1;
    auto f = [&](uint64_t v) { return (uint64_t)(((u128)v * v + c) % n); };
    while (d == 1) {
      x = f(x);
      y = f(f(y));
      d = gcd_u64(x > y ? x - y : y - x, n);
    }
    if (d != n) return d;
  }
}

static void prime_factors(uint64_t n, std::vector<uint64_t>& out) {
  for (uint64_t p = 2; p < 1000 && p * p <= n; ++p)
    while (n % p == 0) { out.push_back(p); n /= p; }
  if (n == 1) return;
  if (h_is_prime(n)) { out.push_back(n); return; }
  uint64_t d = pollard(n);
  prime_factors(d, out);
  prime_factors(n / d, out);
}

// Smallest primitive root modulo the prime q (the reference's PROOTS entries).
uint64_t h_smallest_primitive_root(uint64_t q) {
  std::vector<uint64_t> f;
  prime_factors(q - 1, f);
  std::sort(f.begin(), f.end());
  f.erase(std::unique(f.begin(), f.end()), f.end());
  for (uint64_t g = 2; g < q; ++g) {
    bool ok = true;
    for (uint64_t p : f)
      if (h_powmod(g, (q - 1) / p, q) == 1) { ok = false; break; }
    if (ok) return g;
  }
  return 0;
}

// Primes of exactly `bits` bits with q = 1 mod `modulus`, descending from 2^bits.
int h_search_primes(int bits, uint64_t modulus, int count, uint64_t* out) {
  if (bits < 2 || bits > 63 || modulus == 0) return 0;
  uint64_t top = (1ull << bits) - 1;
  uint64_t q = top / modulus * modulus + 1;
  if (q > top) q -= modulus;
  int n = 0;
  for (; n < count && q > (1ull << (bits - 1)); q -= modulus)
    if (h_is_prime(q)) out[n++] = q;
  return n;
}

}  // namespace aoa
