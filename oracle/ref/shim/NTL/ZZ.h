// A small stand-in for the part of NTL's ZZ interface that the reference's
// CUDA sources use (NTL is absent here), so that the reference's own host
// precompute (CUDAManager::precompute, NTTEngine::init, COMMONEngine::init)
// runs unmodified in the harness of oracle/ref.
//
// Nonnegative integers of any size as little-endian 64-bit limbs: products,
// sums, differences, powers, comparisons, and division / remainder by values
// below 2^64 (the only divisors the reference uses: its primes).  InvMod and
// NumBits follow NTL's definitions.  Anything outside that (a negative
// result, a divisor of 2^64 or more, a number too large for conv) aborts.
// Test infrastructure only.
#pragma once
#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <ostream>
#include <string>
#include <vector>

namespace NTL {

[[noreturn]] inline void stand_in_abort(const char* what) {
  std::fprintf(stderr, "NTL stand-in: %s\n", what);
  std::abort();
}

class ZZ {
 public:
  std::vector<uint64_t> w;    // limbs, little endian, no leading zero limbs

  ZZ() {}
  ZZ(long v) {
    if (v < 0) stand_in_abort("negative value");
    set(uint64_t(v));
  }
  static ZZ of(uint64_t v) {
    ZZ z;
    z.set(v);
    return z;
  }
  void set(uint64_t v) {
    w.clear();
    if (v) w.push_back(v);
  }
  void trim() {
    while (!w.empty() && w.back() == 0) w.pop_back();
  }
  bool fits64() const { return w.size() <= 1; }
  uint64_t low() const { return w.empty() ? 0 : w[0]; }

  ZZ& operator*=(const ZZ& b) { return *this = mul(*this, b); }
  ZZ& operator+=(const ZZ& b) { return *this = add(*this, b); }
  ZZ& operator-=(const ZZ& b) { return *this = sub(*this, b); }
  ZZ& operator/=(const ZZ& b) { return *this = divmod(*this, b, nullptr); }
  ZZ& operator%=(const ZZ& b) {
    uint64_t r;
    divmod(*this, b, &r);
    set(r);
    return *this;
  }

  static ZZ mul(const ZZ& a, const ZZ& b) {
    ZZ c;
    if (a.w.empty() || b.w.empty()) return c;
    c.w.assign(a.w.size() + b.w.size(), 0);
    for (size_t i = 0; i < a.w.size(); i++) {
      unsigned __int128 carry = 0;
      for (size_t j = 0; j < b.w.size(); j++) {
        unsigned __int128 t = (unsigned __int128)a.w[i] * b.w[j] + c.w[i + j] + carry;
        c.w[i + j] = (uint64_t)t;
        carry = t >> 64;
      }
      c.w[i + b.w.size()] = (uint64_t)carry;
    }
    c.trim();
    return c;
  }
  static ZZ add(const ZZ& a, const ZZ& b) {
    ZZ c;
    const size_t n = std::max(a.w.size(), b.w.size());
    c.w.assign(n + 1, 0);
    unsigned __int128 carry = 0;
    for (size_t i = 0; i < n; i++) {
      unsigned __int128 t = carry;
      if (i < a.w.size()) t += a.w[i];
      if (i < b.w.size()) t += b.w[i];
      c.w[i] = (uint64_t)t;
      carry = t >> 64;
    }
    c.w[n] = (uint64_t)carry;
    c.trim();
    return c;
  }
  static int cmp(const ZZ& a, const ZZ& b) {
    if (a.w.size() != b.w.size()) return a.w.size() < b.w.size() ? -1 : 1;
    for (size_t i = a.w.size(); i-- > 0;)
      if (a.w[i] != b.w[i]) return a.w[i] < b.w[i] ? -1 : 1;
    return 0;
  }
  static ZZ sub(const ZZ& a, const ZZ& b) {
    if (cmp(a, b) < 0) stand_in_abort("negative difference");
    ZZ c = a;
    uint64_t borrow = 0;
    for (size_t i = 0; i < c.w.size(); i++) {
      const uint64_t bi = i < b.w.size() ? b.w[i] : 0;
      const uint64_t t = c.w[i] - bi - borrow;
      borrow = (c.w[i] < bi || (c.w[i] == bi && borrow)) ? 1 : 0;
      c.w[i] = t;
    }
    c.trim();
    return c;
  }
  // quotient of a / d for d < 2^64 (remainder in *rem when given)
  static ZZ divmod(const ZZ& a, const ZZ& d, uint64_t* rem) {
    if (!d.fits64() || d.low() == 0) stand_in_abort("division by zero or by a value of 2^64 or more");
    const uint64_t dv = d.low();
    ZZ q;
    q.w.assign(a.w.size(), 0);
    unsigned __int128 r = 0;
    for (size_t i = a.w.size(); i-- > 0;) {
      const unsigned __int128 cur = (r << 64) | a.w[i];
      q.w[i] = (uint64_t)(cur / dv);
      r = cur % dv;
    }
    q.trim();
    if (rem) *rem = (uint64_t)r;
    return q;
  }
  long bits() const {
    if (w.empty()) return 0;
    return 64 * (long)(w.size() - 1) + (64 - __builtin_clzll(w.back()));
  }
};

inline ZZ operator*(const ZZ& a, const ZZ& b) { return ZZ::mul(a, b); }
inline ZZ operator*(uint64_t a, const ZZ& b) { return ZZ::mul(ZZ::of(a), b); }
inline ZZ operator*(const ZZ& a, uint64_t b) { return ZZ::mul(a, ZZ::of(b)); }
inline ZZ operator+(const ZZ& a, const ZZ& b) { return ZZ::add(a, b); }
inline ZZ operator-(const ZZ& a, const ZZ& b) { return ZZ::sub(a, b); }
inline ZZ operator/(const ZZ& a, const ZZ& b) { return ZZ::divmod(a, b, nullptr); }
inline ZZ operator/(const ZZ& a, uint64_t b) { return ZZ::divmod(a, ZZ::of(b), nullptr); }
inline ZZ operator%(const ZZ& a, const ZZ& b) {
  uint64_t r;
  ZZ::divmod(a, b, &r);
  return ZZ::of(r);
}
inline ZZ operator%(const ZZ& a, uint64_t b) { return a % ZZ::of(b); }
inline bool operator==(const ZZ& a, const ZZ& b) { return ZZ::cmp(a, b) == 0; }
inline bool operator!=(const ZZ& a, const ZZ& b) { return ZZ::cmp(a, b) != 0; }
inline bool operator<(const ZZ& a, const ZZ& b) { return ZZ::cmp(a, b) < 0; }
inline bool operator>(const ZZ& a, const ZZ& b) { return ZZ::cmp(a, b) > 0; }
inline bool operator<=(const ZZ& a, const ZZ& b) { return ZZ::cmp(a, b) <= 0; }
inline bool operator>=(const ZZ& a, const ZZ& b) { return ZZ::cmp(a, b) >= 0; }

inline std::ostream& operator<<(std::ostream& o, const ZZ& z) {   // decimal
  if (z.w.empty()) return o << '0';
  std::string s;
  ZZ t = z;
  while (!t.w.empty()) {
    uint64_t r;
    t = ZZ::divmod(t, ZZ::of(10), &r);
    s.push_back(char('0' + r));
  }
  std::reverse(s.begin(), s.end());
  return o << s;
}

inline ZZ to_ZZ(uint64_t v) { return ZZ::of(v); }
inline ZZ to_ZZ(unsigned v) { return ZZ::of(v); }
inline ZZ to_ZZ(long v) { return ZZ(v); }
inline ZZ to_ZZ(long long v) { return ZZ((long)v); }
inline ZZ to_ZZ(int v) { return ZZ((long)v); }
inline ZZ to_ZZ(const char* s) {
  ZZ z;
  for (; *s; s++) {
    if (*s < '0' || *s > '9') stand_in_abort("to_ZZ: not a decimal number");
    z = ZZ::add(ZZ::mul(z, ZZ::of(10)), ZZ::of(uint64_t(*s - '0')));
  }
  return z;
}

template <class T>
inline T conv(const ZZ& z) {
  if (!z.fits64()) stand_in_abort("conv: value does not fit");
  return (T)z.low();
}

inline long NumBits(const ZZ& z) { return z.bits(); }
inline long NumBits(uint64_t v) { return ZZ::of(v).bits(); }
inline long NumBits(long v) { return ZZ(v).bits(); }
inline long NumBits(int v) { return ZZ((long)v).bits(); }

inline ZZ power(const ZZ& a, long e) {
  ZZ r = ZZ::of(1), b = a;
  for (; e > 0; e >>= 1) {
    if (e & 1) r = r * b;
    b = b * b;
  }
  return r;
}

// a^-1 mod n (0 <= a < n < 2^64, gcd 1), as NTL's InvMod
inline ZZ InvMod(const ZZ& a, const ZZ& n) {
  if (!a.fits64() || !n.fits64()) stand_in_abort("InvMod: operands of 2^64 or more");
  const uint64_t m = n.low();
  __int128 t = 0, nt = 1, r = m, nr = a.low() % m;
  while (nr) {
    const __int128 qq = r / nr;
    __int128 x = t - qq * nt;
    t = nt;
    nt = x;
    x = r - qq * nr;
    r = nr;
    nr = x;
  }
  if (r != 1) stand_in_abort("InvMod: not invertible");
  if (t < 0) t += m;
  return ZZ::of((uint64_t)t);
}

inline ZZ PowerMod(const ZZ& a, const ZZ& e, const ZZ& n) {
  if (!a.fits64() || !e.fits64() || !n.fits64()) stand_in_abort("PowerMod: operands of 2^64 or more");
  const uint64_t m = n.low();
  unsigned __int128 r = 1 % m, b = a.low() % m;
  for (uint64_t x = e.low(); x; x >>= 1) {
    if (x & 1) r = r * b % m;
    b = b * b % m;
  }
  return ZZ::of((uint64_t)r);
}
inline ZZ PowerMod(const ZZ& a, long e, const ZZ& n) { return PowerMod(a, ZZ(e), n); }

}  // namespace NTL

// NTL_CLIENT brings both namespaces into scope, as NTL's own definition does
#define NTL_CLIENT using namespace std; using namespace NTL;
