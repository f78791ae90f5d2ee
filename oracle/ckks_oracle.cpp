// CKKS CPU ORACLE — test infrastructure only.
//
// This file checks results and is never the product: only tests/, the smoke check of
// __graft_entry__.py and the cpu_baseline / reference leg of bench.py load it.
// It restates, on the CPU and in plain C++17 (`unsigned __int128`), the
// algorithms of the reference evaluator pdroalves/aoa (aoa-ntt = library
// `newckks`) for the CKKS hot path.  Every function cites the reference
// file:line it follows (paths relative to the reference project root).
//
// Parity pins (see tests/test_oracle_*.py):
//   * modular arithmetic: the reference Barrett `mod` restated below is checked
//     against exact 128-bit `%` on random canonical products for every prime of
//     the reference prime tables (tests/golden/reference_primes.json), which is
//     what the reference's own TestPrimitives.mod/mulmod check against NTL ZZ
//     (aoa-ntt/tests/tests.cpp:300-424);
//   * NTT: the restated hierarchical transform is checked against the closed
//     form a(psi^(2*bitrev(p)+1)) and its products against the schoolbook
//     negacyclic product (the reference's TestNTTArithmetic.Mul/MulAdd/MulInt,
//     aoa-ntt/tests/tests.cpp:564-694), through an independent Python big-int
//     model;
//   * CKKS ops: decrypted error bounds as in the reference's CKKS tests.
//
// Randomness (cuRAND in the reference) is kept out of every function here:
// secrets, uniform polynomials and noise are explicit inputs.
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <cmath>
#include <complex>
#include <vector>
#include <algorithm>
#include <stdexcept>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef unsigned __int128 u128;
typedef __int128 i128;

extern "C" {

// ---------------------------------------------------------------------------
// Exact number theory helpers (restate NTL ZZ InvMod/PowerMod used on the host
// by the reference precompute, aoa-ntt/src/cuda/manager.cu:566-759).
// ---------------------------------------------------------------------------
uint64_t oc_mulmod_exact(uint64_t a, uint64_t b, uint64_t q) {
  return (uint64_t)(((u128)a * b) % q);
}

uint64_t oc_powmod(uint64_t a, uint64_t e, uint64_t q) {
  uint64_t r = 1 % q, s = a % q;
  while (e) {
    if (e & 1) r = oc_mulmod_exact(r, s, q);
    s = oc_mulmod_exact(s, s, q);
    e >>= 1;
  }
  return r;
}

uint64_t oc_invmod(uint64_t a, uint64_t q) {
  // extended Euclid over signed 128-bit
  i128 t = 0, nt = 1, r = q, nr = a % q;
  while (nr) {
    i128 qq = r / nr, tmp;
    tmp = t - qq * nt; t = nt; nt = tmp;
    tmp = r - qq * nr; r = nr; nr = tmp;
  }
  if (r != 1) return 0;
  if (t < 0) t += q;
  return (uint64_t)t;
}

static int nbits64(uint64_t x) { return x ? 64 - __builtin_clzll(x) : 0; }

// Deterministic Miller-Rabin for 64-bit integers (bases valid below 2^64).
int oc_is_prime(uint64_t n) {
  if (n < 2) return 0;
  static const uint64_t small[] = {2, 3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37};
  for (uint64_t p : small) {
    if (n % p == 0) return n == p;
  }
  uint64_t d = n - 1; int s = 0;
  while (!(d & 1)) { d >>= 1; s++; }
  for (uint64_t a : small) {
    uint64_t x = oc_powmod(a, d, n);
    if (x == 1 || x == n - 1) continue;
    bool comp = true;
    for (int r = 1; r < s; r++) {
      x = oc_mulmod_exact(x, x, n);
      if (x == n - 1) { comp = false; break; }
    }
    if (comp) return 0;
  }
  return 1;
}

static uint64_t gcd64(uint64_t a, uint64_t b) { while (b) { uint64_t t = a % b; a = b; b = t; } return a; }

// Pollard-Brent rho: returns a non-trivial factor of composite n.
static uint64_t rho_factor(uint64_t n) {
  if (n % 2 == 0) return 2;
  for (uint64_t c = 1;; c++) {
    uint64_t y = 2, x = 2, g = 1, q = 1, ys = 2;
    uint64_t m = 128, r = 1;
    auto f = [&](uint64_t v) { return (uint64_t)(((u128)v * v + c) % n); };
    do {
      x = y;
      for (uint64_t i = 0; i < r; i++) y = f(y);
      uint64_t k = 0;
      do {
        ys = y;
        for (uint64_t i = 0; i < std::min(m, r - k); i++) {
          y = f(y);
          q = oc_mulmod_exact(q, x > y ? x - y : y - x, n);
        }
        g = gcd64(q, n);
        k += m;
      } while (k < r && g == 1);
      r <<= 1;
    } while (g == 1);
    if (g == n) {
      do { ys = f(ys); g = gcd64(x > ys ? x - ys : ys - x, n); } while (g == 1);
    }
    if (g != n) return g;
  }
}

static void factor_rec(uint64_t n, std::vector<uint64_t>& out) {
  if (n == 1) return;
  if (oc_is_prime(n)) { out.push_back(n); return; }
  for (uint64_t p : {2ull, 3ull, 5ull, 7ull, 11ull, 13ull}) {
    if (n % p == 0) { out.push_back(p); factor_rec(n / p, out); return; }
  }
  uint64_t d = rho_factor(n);
  factor_rec(d, out);
  factor_rec(n / d, out);
}

// Smallest primitive root of the prime q.  The reference's PROOTS table
// (aoa-ntt/src/cuda/htrans/coprimes.cu:24048-24879) was filled by querying
// "primitive root of q" (aoa-ntt/src/cuda/htrans/aux/generate_coprimes.py:
// load_primitiveroots), which answers the smallest primitive root; the
// fixture test checks this function against that table.
uint64_t oc_smallest_primitive_root(uint64_t q) {
  std::vector<uint64_t> f;
  factor_rec(q - 1, f);
  std::sort(f.begin(), f.end());
  f.erase(std::unique(f.begin(), f.end()), f.end());
  for (uint64_t g = 2; g < q; g++) {
    bool ok = true;
    for (uint64_t p : f) {
      if (oc_powmod(g, (q - 1) / p, q) == 1) { ok = false; break; }
    }
    if (ok) return g;
  }
  return 0;
}

// Deterministic downward search for `count` primes of exactly `bits` bits with
// q = 1 mod `modulus` (a power of two), starting from 2^bits.  Used for the
// 60-bit and 52-bit prime sets that the reference's tables do not contain.
int oc_gen_ntt_primes(int bits, uint64_t modulus, int count, uint64_t* out) {
  uint64_t top = (bits == 64) ? ~0ull : ((1ull << bits) - 1);
  uint64_t q = (top / modulus) * modulus + 1;
  if (q > top) q -= modulus;
  int found = 0;
  while (found < count && q > (1ull << (bits - 1))) {
    if (oc_is_prime(q)) out[found++] = q;
    q -= modulus;
  }
  return found;
}

// ---------------------------------------------------------------------------
// The reference's Barrett reduction.
//   mu = floor(4^NumBits(q) / q)          aoa-ntt/src/cuda/htrans/common.cu:489-498
//   mod(u128 a, rid)                      aoa-ntt/src/cuda/htrans/common.cu:257-291
//   mulmod(a, b, rid) = mod(a*b)          aoa-ntt/src/cuda/htrans/common.cu:174-193
// ---------------------------------------------------------------------------
uint64_t oc_ref_barrett_mu(uint64_t q) {
  int n = nbits64(q);
  u128 four = ((u128)1) << (2 * n);
  return (uint64_t)(four / q);
}

static inline uint64_t ref_mod(u128 a, uint64_t p, int numbits, uint64_t MU) {
  uint64_t z = (numbits == 64) ? ~0ull : ((1ull << numbits) - 1);
  uint64_t alo = (uint64_t)a, ahi = (uint64_t)(a >> 64);
  uint64_t m0 = alo & z;
  uint64_t m1 = (ahi << (64 - numbits)) + (alo >> numbits);
  int sh = 2 * numbits - 64;             // rshift(a, 2*numbits-64)
  uint64_t xlo, xhi;
  if (sh == 0) { xlo = alo; xhi = ahi; }
  else { xlo = (alo >> sh) + (ahi << (64 - sh)); xhi = ahi >> sh; }
  uint64_t q = (uint64_t)(((u128)xlo * MU) >> 64) + xhi * MU;
  u128 qp = (u128)q * p;
  uint64_t qplo = (uint64_t)qp, qphi = (uint64_t)(qp >> 64);
  uint64_t q0 = qplo & z;
  uint64_t q1 = (qphi << (64 - numbits)) + (qplo >> numbits);
  uint64_t r0 = m0 - q0;
  uint64_t r1 = (m1 - q1) - (m0 < q0);
  uint64_t r = (r0 - r1 * p) & z;
  return (r >= p) ? r - p : r;           // SEL(r, r-p, r>=p)
}

uint64_t oc_ref_mulmod(uint64_t a, uint64_t b, uint64_t q) {
  return ref_mod((u128)a * b, q, nbits64(q), oc_ref_barrett_mu(q));
}

uint64_t oc_ref_mod128(uint64_t hi, uint64_t lo, uint64_t q) {
  return ref_mod(((u128)hi << 64) | lo, q, nbits64(q), oc_ref_barrett_mu(q));
}

// Scan `count` random canonical products for prime q; returns how many times
// the reference Barrett result differs from the exact residue.
long oc_ref_mulmod_mismatches(uint64_t q, long count, uint64_t seed) {
  uint64_t s = seed ? seed : 0x9E3779B97F4A7C15ull;
  int n = nbits64(q); uint64_t mu = oc_ref_barrett_mu(q);
  long bad = 0;
  for (long i = 0; i < count; i++) {
    s ^= s << 13; s ^= s >> 7; s ^= s << 17; uint64_t a = s % q;
    s ^= s << 13; s ^= s >> 7; s ^= s << 17; uint64_t b = s % q;
    if (i & 1) { a = q - 1 - (a & 0xFFFF); }
    u128 x = (u128)a * b;
    if (ref_mod(x, q, n, mu) != (uint64_t)(x % q)) bad++;
  }
  return bad;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Oracle context: RNS bases, per-prime tables, CRT constants.
// ---------------------------------------------------------------------------
namespace {

enum { ST_COEF = 1, ST_NTT = 2 };             // RNSSTATE / TRANSSTATE (defines.h:56-60)
enum { BASE_Q = 0, BASE_B = 1, BASE_QB = 2 };  // poly_bases (defines.h:62-66)

struct Prime {
  uint64_t q; int nbits; uint64_t mu;
  uint64_t proot;
  // reference hierarchical-NTT tables, one residue (ntt.cu:685-1023, common.cu:314-357)
  std::vector<uint64_t> gjk_a, invgjk_a, gjk_b, invgjk_b;  // [log2 S][S]
  std::vector<uint64_t> nthroot, invnthroot;              // [N]
  std::vector<uint64_t> gN, ginvN;                        // [N]
  inline uint64_t mul(uint64_t a, uint64_t b) const { return ref_mod((u128)a * b, q, nbits, mu); }
  inline uint64_t add(uint64_t a, uint64_t b) const { uint64_t s = a + b; return s >= q ? s - q : s; }
  inline uint64_t sub(uint64_t a, uint64_t b) const { return a < b ? a + (q - b) : a - b; }
};

static int ilog2i(long n) { int l = 0; while ((1L << l) < n) l++; return l; }

static int bitrev(int x, int bits) {
  int r = 0;
  for (int i = 0; i < bits; i++) r |= ((x >> i) & 1) << (bits - 1 - i);
  return r;
}

// NTT factorisations NTTFACT* (aoa-ntt/include/newckks/cuda/htrans/ntt.h:24-44):
// Na = 2^ceil(log N / 2), Nb = 2^floor(log N / 2); hierarchical for N >= 128.
static void fact(int N, int& Na, int& Nb) {
  int l = ilog2i(N);
  Na = 1 << ((l + 1) / 2);
  Nb = 1 << (l / 2);
}

// compute_gjk (aoa-ntt/src/cuda/htrans/common.cu:314-357) for one residue:
// g = proot^((p-1)/(2S)); gjk[s][j] = g^(j*2^(s+1)); invgjk[s][j] = g^((2S-j)*2^(s+1)).
static void compute_gjk(const Prime& P, int S, std::vector<uint64_t>& gjk, std::vector<uint64_t>& inv) {
  int L = ilog2i(S);
  gjk.assign((size_t)L * S, 0);
  inv.assign((size_t)L * S, 0);
  uint64_t g = oc_powmod(P.proot, (P.q - 1) / (2 * (uint64_t)S), P.q);
  for (int st = 0; st < L; st++)
    for (int j = 0; j < S; j++) {
      uint64_t n = (uint64_t)j * ((uint64_t)(S * 2) >> (L - st));
      gjk[(size_t)st * S + j] = oc_powmod(g, n, P.q);
      uint64_t ni = (uint64_t)(S * 2 - j) * ((uint64_t)(S * 2) >> (L - st));
      inv[(size_t)st * S + j] = oc_powmod(g, ni, P.q);
    }
}

struct Ctx {
  int N, k, kl, logN, Na, Nb;
  bool hier;
  std::vector<Prime> P;   // Q primes then B primes (the reference's COPRIMES_BUCKET order)
  // RNS constants (manager.cu:566-671)
  std::vector<uint64_t> InvQqi;   // [l][i]   (Q_l/q_i)^-1 mod q_i
  std::vector<uint64_t> Qqibi;    // [l][i][j] (Q_l/q_i) mod b_j
  std::vector<uint64_t> Bbiqi;    // [i][j]   (B/b_j) mod q_i
  std::vector<uint64_t> InvBbi;   // [j]      ((B/b_j) mod b_j)^-1
  std::vector<uint64_t> InvModBqi;// [i]      (B mod q_i)^-1
  std::vector<uint64_t> Bqi;      // [i]      B mod q_i
  std::vector<uint64_t> Invqlqi;  // [l][i]   q_l^-1 mod q_i
  int nres(int base) const { return base == BASE_Q ? k : (base == BASE_B ? kl : k + kl); }
};

// Product of a subset of 64-bit primes reduced modulo m, computed exactly by
// modular accumulation (equivalent to NTL ZZ products followed by %).
static uint64_t prod_mod(const std::vector<Prime>& P, int a, int b, int except, uint64_t m) {
  uint64_t acc = 1 % m;
  for (int i = a; i < b; i++)
    if (i != except) acc = oc_mulmod_exact(acc, P[i].q % m, m);
  return acc;
}

static void precompute(Ctx& C) {
  const int k = C.k, kl = C.kl;
  C.InvQqi.assign((size_t)k * k, 0);
  C.Qqibi.assign((size_t)k * k * kl, 0);
  C.Bbiqi.assign((size_t)k * kl, 0);
  C.InvBbi.assign(kl, 0);
  C.InvModBqi.assign(k, 0);
  C.Bqi.assign(k, 0);
  C.Invqlqi.assign((size_t)k * k, 0);
  for (int i = 0; i < k; i++) {
    uint64_t qi = C.P[i].q;
    C.Bqi[i] = prod_mod(C.P, k, k + kl, -1, qi);                 // manager.cu:599
    C.InvModBqi[i] = oc_invmod(C.Bqi[i], qi);                    // manager.cu:603-605
  }
  for (int j = 0; j < kl; j++) {
    uint64_t bj = C.P[k + j].q;
    C.InvBbi[j] = oc_invmod(prod_mod(C.P, k, k + kl, k + j, bj), bj);  // manager.cu:615
  }
  for (int l = 0; l < k; l++)                                      // manager.cu:639-644
    for (int i = 0; i < k; i++)
      if (l != i) C.Invqlqi[(size_t)l * k + i] = oc_invmod(C.P[l].q % C.P[i].q, C.P[i].q);
  for (int i = 0; i < k; i++)                                      // manager.cu:650-652
    for (int j = 0; j < kl; j++)
      C.Bbiqi[(size_t)i * kl + j] = prod_mod(C.P, k, k + kl, k + j, C.P[i].q);
  for (int l = 0; l < k; l++)                                      // manager.cu:654-671
    for (int i = 0; i <= l; i++) {
      // only i <= l is ever read (fast_conv_Q_to_B loops rid_Q <= level)
      C.InvQqi[(size_t)l * k + i] = oc_invmod(prod_mod(C.P, 0, l + 1, i, C.P[i].q), C.P[i].q);
      for (int j = 0; j < kl; j++)
        C.Qqibi[((size_t)l * k + i) * kl + j] = prod_mod(C.P, 0, l + 1, i, C.P[k + j].q);
    }
}

// NTTEngine::init tables (aoa-ntt/src/cuda/htrans/ntt.cu:685-1023) for one residue.
static void ntt_tables(Ctx& C, Prime& P) {
  const int N = C.N;
  uint64_t q = P.q;
  if ((q - 1) % (2 * (uint64_t)N) != 0) throw std::runtime_error("2N does not divide q-1");
  // compute_nthroot_ntt (ntt.cu:685-721): psi = proot^((p-1)/(2N))
  uint64_t psi = oc_powmod(P.proot, (q - 1) / (2 * (uint64_t)N), q);
  uint64_t ipsi = oc_invmod(psi, q);
  uint64_t invN = oc_invmod((uint64_t)N % q, q);
  P.nthroot.resize(N); P.invnthroot.resize(N);
  uint64_t pw = 1, ipw = 1;                 // psi^c and psi^-c by running products
  for (int c = 0; c < N; c++) {
    P.nthroot[c] = pw;
    P.invnthroot[c] = C.hier ? ipw : oc_mulmod_exact(ipw, invN, q);   // ntt.cu:714-720
    pw = oc_mulmod_exact(pw, psi, q);
    ipw = oc_mulmod_exact(ipw, ipsi, q);
  }
  if (C.hier) {
    compute_gjk(P, C.Na, P.gjk_a, P.invgjk_a);
    compute_gjk(P, C.Nb, P.gjk_b, P.invgjk_b);
    // 4-step twiddles (ntt.cu:961-1023): g = proot^((p-1)/N)
    int Na = C.Na, Nb = C.Nb, lb = ilog2i(Nb);
    uint64_t g = oc_powmod(P.proot, (q - 1) / (uint64_t)N, q);
    uint64_t gi = oc_invmod(g, q);
    uint64_t invNN = oc_invmod((uint64_t)(Na * Nb) % q, q);
    P.gN.resize(N); P.ginvN.resize(N);
    // gN[c] = g^((c / Nb) * bitrev(c % Nb)): running product down each column
    for (int col = 0; col < Nb; col++) {
      uint64_t step = oc_powmod(g, bitrev(col, lb), q), cur = 1;
      for (int r = 0; r < Na; r++) { P.gN[(size_t)r * Nb + col] = cur; cur = oc_mulmod_exact(cur, step, q); }
    }
    // ginvN[c] = g^-(bitrev(c / Na) * (c % Na)) / N: running product along each row
    for (int u = 0; u < Nb; u++) {
      uint64_t step = oc_powmod(gi, bitrev(u, lb), q), cur = invNN;
      for (int v = 0; v < Na; v++) { P.ginvN[(size_t)u * Na + v] = cur; cur = oc_mulmod_exact(cur, step, q); }
    }
  } else {
    compute_gjk(P, N, P.gjk_a, P.invgjk_a);
  }
}

// doNTT<S> / ntttransform (ntt.cu:128-158, 196-219): Gentleman-Sande DIF over
// an S-point signal held in s[], natural order in, bit-reversed order out.
static void doNTT(const Prime& P, uint64_t* s, int S, const std::vector<uint64_t>& gjk) {
  int L = ilog2i(S);
  for (int st = 0; st < L; st++) {
    int m = S / (2 << st);
    for (int cid = 0; cid < S / 2; cid++) {
      int j = cid * 2 * m / S;
      int i = j + (cid % (S / (2 * m))) * 2 * m;
      uint64_t a = gjk[(size_t)st * S + j];
      uint64_t xi = s[i], xim = s[i + m];
      s[i] = P.add(xi, xim);
      s[i + m] = P.mul(a, P.sub(xi, xim));
    }
  }
}

// doINTT<S> / intttransform (ntt.cu:160-194, 222-246): Cooley-Tukey DIT.
static void doINTT(const Prime& P, uint64_t* s, int S, const std::vector<uint64_t>& inv) {
  int L = ilog2i(S);
  for (int st = L - 1; st >= 0; st--) {
    int m = S / (2 << st);
    for (int cid = 0; cid < S / 2; cid++) {
      int j = cid * 2 * m / S;
      int i = j + (cid % (S / (2 * m))) * 2 * m;
      uint64_t a = inv[(size_t)st * S + j];
      uint64_t xi = s[i], xim = s[i + m];
      uint64_t axim = P.mul(a, xim);
      s[i] = P.add(xi, axim);
      s[i + m] = P.sub(xi, axim);
    }
  }
}

// Forward transform of one residue.  Hierarchical: hntt_tr<Nb> then hntt_tr<Na>
// (ntt.cu:35-50, 321-363); small N: ntt<N> (ntt.cu:251-278).
static void ntt_fwd_one(const Ctx& C, const Prime& P, uint64_t* x) {
  const int N = C.N;
  if (!C.hier) {
    for (int i = 0; i < N; i++) x[i] = P.mul(x[i], P.nthroot[i]);
    doNTT(P, x, N, P.gjk_a);
    return;
  }
  const int Na = C.Na, Nb = C.Nb;
  std::vector<uint64_t> tmp(N), s(std::max(Na, Nb));
  // pass 1: hntt_tr<Nb>, grid Na: block c gathers x[j*Na + c], twist by psi^(j*Na+c)
  for (int c = 0; c < Na; c++) {
    for (int j = 0; j < Nb; j++) s[j] = P.mul(x[(size_t)j * Na + c], P.nthroot[(size_t)j * Na + c]);
    doNTT(P, s.data(), Nb, P.gjk_b);
    for (int t = 0; t < Nb; t++) tmp[(size_t)c * Nb + t] = s[t];   // written transposed
  }
  // pass 2: hntt_tr<Na>, grid Nb: block c' gathers tmp[j*Nb + c'], twist by gN
  for (int c = 0; c < Nb; c++) {
    for (int j = 0; j < Na; j++) s[j] = P.mul(tmp[(size_t)j * Nb + c], P.gN[(size_t)j * Nb + c]);
    doNTT(P, s.data(), Na, P.gjk_a);
    for (int t = 0; t < Na; t++) x[(size_t)c * Na + t] = s[t];
  }
}

// Inverse transform of one residue: hintt<Na> then hintt_tr<Nb>
// (ntt.cu:51-65, 373-460); small N: intt<N> (ntt.cu:282-308).
static void ntt_inv_one(const Ctx& C, const Prime& P, uint64_t* x) {
  const int N = C.N;
  if (!C.hier) {
    doINTT(P, x, N, P.invgjk_a);
    for (int i = 0; i < N; i++) x[i] = P.mul(x[i], P.invnthroot[i]);
    return;
  }
  const int Na = C.Na, Nb = C.Nb;
  std::vector<uint64_t> tmp(N), s(std::max(Na, Nb));
  // hintt<Na>: contiguous rows of Na, untwist by ginvN (1/N folded in)
  for (int r = 0; r < Nb; r++) {
    for (int t = 0; t < Na; t++) s[t] = x[(size_t)r * Na + t];
    doINTT(P, s.data(), Na, P.invgjk_a);
    for (int t = 0; t < Na; t++) tmp[(size_t)r * Na + t] = P.mul(s[t], P.ginvN[(size_t)r * Na + t]);
  }
  // hintt_tr<Nb>: column c gathers tmp[t*Na + c], untwist by psi^-(t*Na+c)
  for (int c = 0; c < Na; c++) {
    for (int t = 0; t < Nb; t++) s[t] = tmp[(size_t)t * Na + c];
    doINTT(P, s.data(), Nb, P.invgjk_b);
    for (int t = 0; t < Nb; t++) x[(size_t)t * Na + c] = P.mul(s[t], P.invnthroot[(size_t)t * Na + c]);
  }
}

// ---------------------------------------------------------------------------
// poly_t restatement (defines.h:66-72, poly_t.cpp): residues [nres][N], a
// domain state and a base.  Operations follow poly_t.cpp's lazy domain rules.
// ---------------------------------------------------------------------------
struct Poly {
  std::vector<uint64_t> d;
  int state = ST_COEF;
  int base = BASE_Q;
};

static void poly_init(const Ctx& C, Poly& p, int base) {
  if (!p.d.empty()) return;
  p.d.assign((size_t)C.nres(base) * C.N, 0);
  p.state = ST_COEF; p.base = base;
}

static void transform(const Ctx& C, Poly& p, int dir) {   // NTTEngine::execute_ntt (ntt.cu:463-475)
  if ((p.state == ST_NTT && dir == ST_NTT) || (p.state == ST_COEF && dir == ST_COEF)) return;
  int n = C.nres(p.base);
  #pragma omp parallel for schedule(static)
  for (int r = 0; r < n; r++) {
    if (dir == ST_NTT) ntt_fwd_one(C, C.P[r], p.d.data() + (size_t)r * C.N);
    else ntt_inv_one(C, C.P[r], p.d.data() + (size_t)r * C.N);
  }
  p.state = dir;
}

enum { OP_ADD, OP_SUB, OP_MUL };

// ntt_vector_op (ntt.cu:479-509) over the residues of `base`
static void vec_op(const Ctx& C, uint64_t* c, const uint64_t* a, const uint64_t* b, int op, int base) {
  long total = (long)C.nres(base) * C.N;
  #pragma omp parallel for schedule(static)
  for (long t = 0; t < total; t++) {
    const Prime& P = C.P[t / C.N];
    switch (op) {
      case OP_ADD: c[t] = P.add(a[t], b[t]); break;
      case OP_SUB: c[t] = P.sub(a[t], b[t]); break;
      default: c[t] = P.mul(a[t], b[t]); break;
    }
  }
}

static void poly_add(const Ctx& C, Poly& c, Poly& a, Poly& b) {      // poly_t.cpp:137-155
  int base = std::min(a.base, b.base);
  poly_init(C, c, base);
  if (a.state != b.state) { transform(C, a, ST_COEF); transform(C, b, ST_COEF); }
  vec_op(C, c.d.data(), a.d.data(), b.d.data(), OP_ADD, base);
  c.state = a.state; c.base = base;
}

static void poly_sub(const Ctx& C, Poly& c, Poly& a, Poly& b) {      // poly_t.cpp:169-187
  int base = std::min(a.base, b.base);
  poly_init(C, c, base);
  if (a.state != b.state) { transform(C, a, ST_COEF); transform(C, b, ST_COEF); }
  vec_op(C, c.d.data(), a.d.data(), b.d.data(), OP_SUB, base);
  c.state = a.state; c.base = base;
}

static void poly_mul(const Ctx& C, Poly& c, Poly& a, Poly& b) {      // poly_t.cpp:201-220
  int base = std::min(a.base, b.base);
  poly_init(C, c, base);
  transform(C, a, ST_NTT);
  transform(C, b, ST_NTT);
  vec_op(C, c.d.data(), a.d.data(), b.d.data(), OP_MUL, base);
  c.state = a.state; c.base = base;
}

static void poly_mul_add(const Ctx& C, Poly& d, Poly& a, Poly& b, Poly& c) {   // poly_t.cpp:274-300
  int base = std::min(std::min(a.base, b.base), c.base);
  poly_init(C, d, base);
  transform(C, a, ST_NTT); transform(C, b, ST_NTT); transform(C, c, ST_NTT);
  long total = (long)C.nres(base) * C.N;
  std::vector<uint64_t> out(total);
  #pragma omp parallel for schedule(static)
  for (long t = 0; t < total; t++) {                                  // ntt_vector_seqop (ntt.cu:625-648)
    const Prime& P = C.P[t / C.N];
    out[t] = P.add(P.mul(a.d[t], b.d[t]), c.d[t]);
  }
  std::copy(out.begin(), out.end(), d.d.begin());
  d.state = a.state; d.base = base;
}

static void poly_add_add(const Ctx& C, Poly& c1, Poly& a1, Poly& b1,
                         Poly& c2, Poly& a2, Poly& b2) {             // poly_t.cpp:237-272
  int base = std::min(std::min(a1.base, b1.base), std::min(a2.base, b2.base));
  poly_init(C, c1, base); poly_init(C, c2, base);
  if (a1.state != b1.state) { transform(C, a1, ST_COEF); transform(C, b1, ST_COEF); }
  if (a2.state != b2.state) { transform(C, a2, ST_COEF); transform(C, b2, ST_COEF); }
  std::vector<uint64_t> o1((size_t)C.nres(base) * C.N), o2(o1.size());
  vec_op(C, o1.data(), a1.d.data(), b1.d.data(), OP_ADD, base);
  vec_op(C, o2.data(), a2.d.data(), b2.d.data(), OP_ADD, base);
  std::copy(o1.begin(), o1.end(), c1.d.begin());
  std::copy(o2.begin(), o2.end(), c2.d.begin());
  c1.state = a1.state; c1.base = base;
  c2.state = a2.state; c2.base = base;
}

// fast_conv_Q_to_B_opt (manager.cu:180-223) writing the B residues of the
// QB-sized array `a` from its Q residues (coefficient domain).
static void conv_Q_to_B(const Ctx& C, uint64_t* a, int level) {
  const int N = C.N, k = C.k, kl = C.kl;
  #pragma omp parallel for schedule(static)
  for (int j = 0; j < kl; j++) {
    const Prime& B = C.P[k + j];
    for (int cid = 0; cid < N; cid++) {
      uint64_t val = 0;
      for (int i = 0; i <= level; i++) {
        uint64_t aux = C.P[i].mul(a[(size_t)i * N + cid], C.InvQqi[(size_t)level * k + i]);
        aux %= B.q;
        uint64_t c = C.Qqibi[((size_t)level * k + i) * kl + j];
        val = B.add(val, B.mul(aux, c));
      }
      a[(size_t)(k + j) * N + cid] = val;
    }
  }
}

// fast_conv_B_to_Q (manager.cu:312-341)
static void conv_B_to_Q(const Ctx& C, uint64_t* out, const uint64_t* a, int level) {
  const int N = C.N, k = C.k, kl = C.kl;
  #pragma omp parallel for schedule(static)
  for (int i = 0; i <= level; i++) {
    const Prime& Q = C.P[i];
    for (int cid = 0; cid < N; cid++) {
      uint64_t val = 0;
      for (int j = 0; j < kl; j++) {
        uint64_t aux = C.P[k + j].mul(a[(size_t)(k + j) * N + cid], C.InvBbi[j]);
        uint64_t tmp = Q.mul(aux, C.Bbiqi[(size_t)i * kl + j]);
        val = Q.add(val, tmp);
      }
      uint64_t t = Q.sub(a[(size_t)i * N + cid], val);
      out[(size_t)i * N + cid] = Q.mul(t, C.InvModBqi[i]);
    }
  }
}

static void poly_copy(const Ctx& C, Poly& b, const Poly& a) {          // poly_t.cpp:102-116
  poly_init(C, b, a.base);
  size_t n = (size_t)C.nres(a.base) * C.N;
  std::copy(a.d.begin(), a.d.begin() + n, b.d.begin());
  b.state = a.state;
}

static void poly_modup(const Ctx& C, Poly& a, Poly& b, int level) {    // poly_t.cpp:345-361
  poly_init(C, a, BASE_QB);
  poly_copy(C, a, b);
  transform(C, a, ST_COEF);
  conv_Q_to_B(C, a.d.data(), level);
}

static void poly_moddown(const Ctx& C, Poly& a, Poly& b, int level) {  // poly_t.cpp:363-378
  poly_init(C, a, BASE_Q);
  transform(C, b, ST_COEF);
  conv_B_to_Q(C, a.d.data(), b.d.data(), level);
  a.state = ST_COEF;
}

// ckks_rescale kernel (manager.cu:90-118): for i < level,
// a_i = (a_i - a_level) * q_level^-1 mod q_i (floor rescale, no rounding).
static void rescale_kernel(const Ctx& C, uint64_t* a, uint64_t* b, int level) {
  const int N = C.N, k = C.k;
  #pragma omp parallel for schedule(static)
  for (int rid = 0; rid < level; rid++) {
    const Prime& P = C.P[rid];
    uint64_t s = C.Invqlqi[(size_t)level * k + rid];
    for (int cid = 0; cid < N; cid++) {
      // submod with an operand a_level < q_level <= q_rid for the reference's
      // descending prime order; reduced first so any order is well defined.
      uint64_t ra = a[(size_t)level * N + cid] % P.q, rb = b[(size_t)level * N + cid] % P.q;
      a[(size_t)rid * N + cid] = P.mul(P.sub(a[(size_t)rid * N + cid], ra), s);
      b[(size_t)rid * N + cid] = P.mul(P.sub(b[(size_t)rid * N + cid], rb), s);
    }
  }
}

static void poly_rescale(const Ctx& C, Poly& a, Poly& b, int level) {  // poly_t.cpp:395-411
  transform(C, a, ST_COEF);
  transform(C, b, ST_COEF);
  rescale_kernel(C, a.d.data(), b.d.data(), level);
}

// execute_rotation (aoa-ntt/src/ckks/encoder.cu:300-322): X -> X^pow (pow odd
// mod 2N) in the coefficient domain, with the negacyclic sign.
static void rotation_kernel(const Ctx& C, uint64_t* b, const uint64_t* a, long pow, int nres) {
  const long N = C.N;
  #pragma omp parallel for schedule(static)
  for (int rid = 0; rid < nres; rid++) {
    uint64_t q = C.P[rid].q;
    for (long cid = 0; cid < N; cid++) {
      long nc = cid * pow % (N << 1);
      int flag = nc >= N;
      if (flag) nc -= N;
      uint64_t v = a[(size_t)rid * N + cid];
      b[(size_t)rid * N + nc] = flag ? C.P[rid].sub(q, v) : v;
    }
  }
}

// rotate_slots_left (encoder.cu:325-353): INTT the input in place, rotate by 5^r mod 2N.
static void rotate_slots_left(const Ctx& C, Poly& b, Poly& a, int r) {
  long M = 2L * C.N;
  long g = (long)oc_powmod(5, (uint64_t)r, (uint64_t)M);
  poly_init(C, b, a.base);
  transform(C, a, ST_COEF);
  rotation_kernel(C, b.d.data(), a.d.data(), g, C.nres(a.base));
  b.state = ST_COEF;
}

// conjugate_slots (encoder.cu:391-427): NTT-domain index reversal, in place.
static void conjugate_slots(const Ctx& C, Poly& a) {
  transform(C, a, ST_NTT);
  int n = C.nres(a.base);
  for (int rid = 0; rid < n; rid++) {
    uint64_t* x = a.d.data() + (size_t)rid * C.N;
    std::reverse(x, x + C.N);
  }
}

struct SwitchKey { Poly a, b; };

// Key switch of `d` (Q base) by `key`, the shared core of ckks_mul_without_rescale
// (ckks.cpp:309-318) and ckks_rotate_left/right, ckks_conjugate (ckks.cpp:965-973,
// 994-1002, 1025-1033): ModUp, multiply by (b, a) over QB, ModDown twice.
static void keyswitch(const Ctx& C, Poly& out0, Poly& out1, Poly& d, SwitchKey& key, int level) {
  Poly d2QB, t0, t1;
  poly_modup(C, d2QB, d, level);
  poly_mul(C, t0, d2QB, key.b);
  poly_mul(C, t1, d2QB, key.a);
  poly_moddown(C, out0, t0, level);
  poly_moddown(C, out1, t1, level);
}

}  // namespace

// ---------------------------------------------------------------------------
// C entry points for the test harness (ctypes).
// ---------------------------------------------------------------------------
extern "C" {

typedef struct oc_ctx oc_ctx;

void oc_set_threads(int n) {
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads(n);
#else
  (void)n;
#endif
}

int oc_get_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

// primes: k Q primes then kl B primes; proots: generators (NULL -> smallest
// primitive root).  Returns NULL when 2N does not divide some q-1.
oc_ctx* oc_create(int N, int k, int kl, const uint64_t* primes, const uint64_t* proots) {
  Ctx* C = new Ctx();
  try {
    C->N = N; C->k = k; C->kl = kl; C->logN = ilog2i(N);
    fact(N, C->Na, C->Nb);
    C->hier = N >= 128;
    C->P.resize(k + kl);
    for (int i = 0; i < k + kl; i++) {
      Prime& P = C->P[i];
      P.q = primes[i]; P.nbits = nbits64(P.q); P.mu = oc_ref_barrett_mu(P.q);
      P.proot = proots ? proots[i] : oc_smallest_primitive_root(P.q);
    }
    #pragma omp parallel for schedule(dynamic)
    for (int i = 0; i < k + kl; i++) ntt_tables(*C, C->P[i]);
    precompute(*C);
  } catch (...) {
    delete C;
    return nullptr;
  }
  return (oc_ctx*)C;
}

void oc_destroy(oc_ctx* c) { delete (Ctx*)c; }

// In-place forward / inverse transform of `nlimbs` residues whose primes start
// at index `first` of the context's Q|B list; data is [nlimbs][N].
void oc_ntt_fwd(oc_ctx* c, uint64_t* data, int first, int nlimbs) {
  Ctx& C = *(Ctx*)c;
  #pragma omp parallel for schedule(static)
  for (int r = 0; r < nlimbs; r++) ntt_fwd_one(C, C.P[first + r], data + (size_t)r * C.N);
}

void oc_ntt_inv(oc_ctx* c, uint64_t* data, int first, int nlimbs) {
  Ctx& C = *(Ctx*)c;
  #pragma omp parallel for schedule(static)
  for (int r = 0; r < nlimbs; r++) ntt_inv_one(C, C.P[first + r], data + (size_t)r * C.N);
}

// Batched forward / inverse over `npolys` polynomials of `nlimbs` limbs each,
// layout [npolys][nlimbs][N], limb r of every poly under prime first+r.
void oc_ntt_fwd_batch(oc_ctx* c, uint64_t* data, int npolys, int first, int nlimbs) {
  Ctx& C = *(Ctx*)c;
  long tot = (long)npolys * nlimbs;
  #pragma omp parallel for schedule(static)
  for (long t = 0; t < tot; t++) ntt_fwd_one(C, C.P[first + (int)(t % nlimbs)], data + (size_t)t * C.N);
}

void oc_ntt_inv_batch(oc_ctx* c, uint64_t* data, int npolys, int first, int nlimbs) {
  Ctx& C = *(Ctx*)c;
  long tot = (long)npolys * nlimbs;
  #pragma omp parallel for schedule(static)
  for (long t = 0; t < tot; t++) ntt_inv_one(C, C.P[first + (int)(t % nlimbs)], data + (size_t)t * C.N);
}

// psi_i = proot_i^((q_i - 1)/(2N)) (ntt.cu:708), for the closed-form pin.
uint64_t oc_psi(oc_ctx* c, int rid) {
  Ctx& C = *(Ctx*)c;
  return oc_powmod(C.P[rid].proot, (C.P[rid].q - 1) / (2 * (uint64_t)C.N), C.P[rid].q);
}

uint64_t oc_prime(oc_ctx* c, int rid) { return ((Ctx*)c)->P[rid].q; }
uint64_t oc_proot(oc_ctx* c, int rid) { return ((Ctx*)c)->P[rid].proot; }

// RNS constant tables, for the GPU precompute pins: which = 0 InvQqi[k*k],
// 1 Qqibi[k*k*kl], 2 Bbiqi[k*kl], 3 InvBbi[kl], 4 InvModBqi[k], 5 Bqi[k], 6 Invqlqi[k*k]
int oc_table(oc_ctx* c, int which, uint64_t* out) {
  Ctx& C = *(Ctx*)c;
  const std::vector<uint64_t>* t = nullptr;
  switch (which) {
    case 0: t = &C.InvQqi; break; case 1: t = &C.Qqibi; break; case 2: t = &C.Bbiqi; break;
    case 3: t = &C.InvBbi; break; case 4: t = &C.InvModBqi; break; case 5: t = &C.Bqi; break;
    case 6: t = &C.Invqlqi; break; default: return -1;
  }
  if (out) std::copy(t->begin(), t->end(), out);
  return (int)t->size();
}

// ModUp of a Q-base coefficient-domain poly `in` ([k][N]) at `level`: writes
// the kl B residues to out_b ([kl][N]).  (fast_conv_Q_to_B_opt)
void oc_modup(oc_ctx* c, const uint64_t* in, int level, uint64_t* out_b) {
  Ctx& C = *(Ctx*)c;
  std::vector<uint64_t> a((size_t)(C.k + C.kl) * C.N, 0);
  std::copy(in, in + (size_t)C.k * C.N, a.begin());
  conv_Q_to_B(C, a.data(), level);
  std::copy(a.begin() + (size_t)C.k * C.N, a.end(), out_b);
}

// ModDown of a QB coefficient-domain poly `in` ([k+kl][N]) at `level`:
// writes limbs 0..level of out ([k][N]).  (fast_conv_B_to_Q)
void oc_moddown(oc_ctx* c, const uint64_t* in, int level, uint64_t* out) {
  conv_B_to_Q(*(Ctx*)c, out, in, level);
}

// Rescale of a ciphertext pair in the coefficient domain at `level` (in place).
void oc_rescale(oc_ctx* c, uint64_t* c0, uint64_t* c1, int level) {
  rescale_kernel(*(Ctx*)c, c0, c1, level);
}

// Coefficient-domain automorphism X -> X^pow over nres residues.
void oc_automorph(oc_ctx* c, const uint64_t* in, uint64_t* out, long pow, int nres) {
  rotation_kernel(*(Ctx*)c, out, in, pow, nres);
}

// Helpers to marshal polys from flat arrays.
static void load_poly(const Ctx& C, Poly& p, const uint64_t* src, int base, int state) {
  p.d.assign(src, src + (size_t)C.nres(base) * C.N);
  p.base = base; p.state = state;
}
static void store_coef(const Ctx& C, Poly& p, uint64_t* dst) {
  transform(C, p, ST_COEF);
  std::copy(p.d.begin(), p.d.begin() + (size_t)C.nres(p.base) * C.N, dst);
}

// Switching key generation with injected randomness, ckks_new_evk
// (ckkskeys.cpp:101-131): b = rho(s1) + e - a*s2 over QB, where rho multiplies
// residue i by B mod q_i (ckks_rho, manager.cu:149-160; zero on B residues).
//   s1, s2: QB-sized coefficient-domain polys; a: QB-sized uniform residues
//   (taken as given, domain `a_state`); e: signed noise, one integer per coefficient.
// Outputs b, a over QB in the NTT domain.
void oc_swk_gen(oc_ctx* c, const uint64_t* s1, const uint64_t* s2, const uint64_t* a_in, int a_state,
                const int64_t* e, uint64_t* out_b, uint64_t* out_a) {
  Ctx& C = *(Ctx*)c;
  const int nqb = C.k + C.kl;
  Poly S1, S2, A, E, B, T;
  load_poly(C, S1, s1, BASE_QB, ST_COEF);
  load_poly(C, S2, s2, BASE_QB, ST_COEF);
  load_poly(C, A, a_in, BASE_QB, a_state);
  poly_init(C, E, BASE_QB);
  for (int r = 0; r < nqb; r++)                       // sample_DG cast (sampler.cu:72-113)
    for (int i = 0; i < C.N; i++) {
      int64_t v = e[i];
      E.d[(size_t)r * C.N + i] = v >= 0 ? (uint64_t)v : C.P[r].q + v;
    }
  // rho(s1): elementwise, domain preserving
  poly_init(C, B, BASE_QB);
  for (int r = 0; r < nqb; r++) {
    uint64_t f = r < C.k ? C.Bqi[r] : 0;
    for (int i = 0; i < C.N; i++) B.d[(size_t)r * C.N + i] = C.P[r].mul(S1.d[(size_t)r * C.N + i], f);
  }
  B.state = S1.state;
  poly_add(C, B, B, E);
  poly_mul(C, T, A, S2);
  poly_sub(C, B, B, T);
  transform(C, B, ST_NTT);
  transform(C, A, ST_NTT);
  std::copy(B.d.begin(), B.d.end(), out_b);
  std::copy(A.d.begin(), A.d.end(), out_a);
}

// s^2 over QB, coefficient domain out (ckks_new_mtk, ckkskeys.cpp:133-144)
void oc_square_secret(oc_ctx* c, const uint64_t* s, uint64_t* out) {
  Ctx& C = *(Ctx*)c;
  Poly S, S2, Sc;
  load_poly(C, S, s, BASE_QB, ST_COEF);
  load_poly(C, Sc, s, BASE_QB, ST_COEF);
  poly_mul(C, S2, S, Sc);
  store_coef(C, S2, out);
}

// rotated secret for rtk_left[r] (ckkskeys.cpp:146-163), QB coefficient domain
void oc_rotate_secret(oc_ctx* c, const uint64_t* s, int r, uint64_t* out) {
  Ctx& C = *(Ctx*)c;
  Poly S, O;
  load_poly(C, S, s, BASE_QB, ST_COEF);
  rotate_slots_left(C, O, S, r);
  store_coef(C, O, out);
}

// conjugated secret for cjk (ckkskeys.cpp:183-191), QB coefficient domain
void oc_conjugate_secret(oc_ctx* c, const uint64_t* s, uint64_t* out) {
  Ctx& C = *(Ctx*)c;
  Poly S;
  load_poly(C, S, s, BASE_QB, ST_COEF);
  conjugate_slots(C, S);
  store_coef(C, S, out);
}

// HMult + relinearisation (ckks_mul_without_rescale, ckks.cpp:273-332) and,
// when do_rescale, the rescale that ckks_mul adds (ckks.cpp:334-347).
// a0,a1,b0,b1: [k][N] residues in domain a_state / b_state; evk: QB NTT domain.
// Returns out0/out1 ([k][N], coefficient domain; limbs above the output level
// are stale as in the reference) and *out_scale.
void oc_hmult(oc_ctx* c, const uint64_t* a0, const uint64_t* a1, int a_state,
              const uint64_t* b0, const uint64_t* b1, int b_state,
              const uint64_t* evk_b, const uint64_t* evk_a,
              int level, uint64_t scale_a, uint64_t scale_b, int do_rescale,
              uint64_t* out0, uint64_t* out1, uint64_t* out_scale) {
  Ctx& C = *(Ctx*)c;
  Poly c10, c11, c20, c21;
  load_poly(C, c10, a0, BASE_Q, a_state); load_poly(C, c11, a1, BASE_Q, a_state);
  load_poly(C, c20, b0, BASE_Q, b_state); load_poly(C, c21, b1, BASE_Q, b_state);
  SwitchKey evk;
  load_poly(C, evk.b, evk_b, BASE_QB, ST_NTT);
  load_poly(C, evk.a, evk_a, BASE_QB, ST_NTT);
  Poly axbx1, axbx2, bxbx, axax, ks0, ks1, o0, o1;
  poly_add_add(C, axbx1, c11, c10, axbx2, c21, c20);
  poly_mul(C, axbx1, axbx1, axbx2);
  poly_mul(C, bxbx, c10, c20);
  poly_mul(C, axax, c11, c21);
  keyswitch(C, ks0, ks1, axax, evk, level);
  poly_add_add(C, o0, bxbx, ks0, o1, axbx1, ks1);
  poly_sub(C, o1, o1, bxbx);
  poly_sub(C, o1, o1, axax);
  *out_scale = (uint64_t)(((u128)scale_a * scale_b) / C.P[level].q);   // ckks.cpp:328-330
  if (do_rescale) poly_rescale(C, o0, o1, level);
  store_coef(C, o0, out0);
  store_coef(C, o1, out1);
}

// ckks_rotate_left (ckks.cpp:982-1009); right rotation by r is left by N/2 - r
// (encoder.cu:356-363).  rtk: QB NTT domain.  Output coefficient domain.
void oc_rotate_left(oc_ctx* c, const uint64_t* in0, const uint64_t* in1, int state, int r,
                    const uint64_t* rtk_b, const uint64_t* rtk_a, int level,
                    uint64_t* out0, uint64_t* out1) {
  Ctx& C = *(Ctx*)c;
  Poly c10, c11, o0, ax, ks0, o1;
  load_poly(C, c10, in0, BASE_Q, state); load_poly(C, c11, in1, BASE_Q, state);
  SwitchKey key;
  load_poly(C, key.b, rtk_b, BASE_QB, ST_NTT);
  load_poly(C, key.a, rtk_a, BASE_QB, ST_NTT);
  rotate_slots_left(C, o0, c10, r);
  rotate_slots_left(C, ax, c11, r);
  keyswitch(C, ks0, o1, ax, key, level);
  poly_add(C, o0, o0, ks0);
  store_coef(C, o0, out0);
  store_coef(C, o1, out1);
}

// ckks_conjugate (ckks.cpp:1011-1040).  cjk: QB NTT domain.
void oc_conjugate(oc_ctx* c, const uint64_t* in0, const uint64_t* in1, int state,
                  const uint64_t* cjk_b, const uint64_t* cjk_a, int level,
                  uint64_t* out0, uint64_t* out1) {
  Ctx& C = *(Ctx*)c;
  Poly c10, c11, o0, ax, ks0, o1;
  load_poly(C, c10, in0, BASE_Q, state); load_poly(C, c11, in1, BASE_Q, state);
  SwitchKey key;
  load_poly(C, key.b, cjk_b, BASE_QB, ST_NTT);
  load_poly(C, key.a, cjk_a, BASE_QB, ST_NTT);
  poly_copy(C, o0, c10);
  poly_copy(C, ax, c11);
  conjugate_slots(C, o0);
  conjugate_slots(C, ax);
  keyswitch(C, ks0, o1, ax, key, level);
  poly_add(C, o0, o0, ks0);
  store_coef(C, o0, out0);
  store_coef(C, o1, out1);
}

// ckks_add / ckks_sub (ckks.cpp:240-271); output in the domain the reference
// leaves it in; returns that domain.
int oc_add(oc_ctx* c, const uint64_t* a0, const uint64_t* a1, int a_state,
           const uint64_t* b0, const uint64_t* b1, int b_state, int subtract,
           uint64_t* out0, uint64_t* out1) {
  Ctx& C = *(Ctx*)c;
  Poly c10, c11, c20, c21, o0, o1;
  load_poly(C, c10, a0, BASE_Q, a_state); load_poly(C, c11, a1, BASE_Q, a_state);
  load_poly(C, c20, b0, BASE_Q, b_state); load_poly(C, c21, b1, BASE_Q, b_state);
  if (subtract) { poly_sub(C, o0, c10, c20); poly_sub(C, o1, c11, c21); }
  else poly_add_add(C, o0, c10, c20, o1, c11, c21);
  std::copy(o0.d.begin(), o0.d.end(), out0);
  std::copy(o1.d.begin(), o1.d.end(), out1);
  return o0.state;
}

// ckks_encrypt_poly (ckks.cpp:87-105) with injected u (ternary, Q coef domain)
// and noise e1, e2 (one signed integer per coefficient).  m: Q coef domain.
// pk_b, pk_a: Q-base residues in domain pk_state.  Output NTT domain.
void oc_encrypt(oc_ctx* c, const uint64_t* m, const uint64_t* u, const int64_t* e1, const int64_t* e2,
                const uint64_t* pk_b, const uint64_t* pk_a, int pk_state,
                uint64_t* out0, uint64_t* out1) {
  Ctx& C = *(Ctx*)c;
  Poly M, U, E, PB, PA, O0, O1;
  load_poly(C, M, m, BASE_Q, ST_COEF);
  load_poly(C, U, u, BASE_Q, ST_COEF);
  load_poly(C, PB, pk_b, BASE_Q, pk_state);
  load_poly(C, PA, pk_a, BASE_Q, pk_state);
  auto noise = [&](Poly& P, const int64_t* e) {
    poly_init(C, P, BASE_Q);
    for (int r = 0; r < C.k; r++)
      for (int i = 0; i < C.N; i++)
        P.d[(size_t)r * C.N + i] = e[i] >= 0 ? (uint64_t)e[i] : C.P[r].q + e[i];
    P.state = ST_COEF;
  };
  noise(E, e1);
  poly_add(C, E, E, M);
  poly_mul_add(C, O0, U, PB, E);
  Poly E2; noise(E2, e2);
  poly_mul_add(C, O1, U, PA, E2);
  std::copy(O0.d.begin(), O0.d.end(), out0);
  std::copy(O1.d.begin(), O1.d.end(), out1);
}

// ckks_decrypt_poly (ckks.cpp:179-192): m = c1*s + c0, coefficient domain out.
void oc_decrypt(oc_ctx* c, const uint64_t* c0, const uint64_t* c1, int state, const uint64_t* s,
                uint64_t* out_m) {
  Ctx& C = *(Ctx*)c;
  Poly C0, C1, S, M;
  load_poly(C, C0, c0, BASE_Q, state);
  load_poly(C, C1, c1, BASE_Q, state);
  load_poly(C, S, s, BASE_Q, ST_COEF);
  poly_mul_add(C, M, C1, S, C0);
  store_coef(C, M, out_m);
}

// ---------------------------------------------------------------------------
// Encoder (aoa-ntt/src/ckks/encoder.cu:12-298), FP64.  Compile with
// -ffp-contract=off: the reference's host FFT rounds every product and sum.
// ---------------------------------------------------------------------------
static void array_bit_reverse(std::complex<double>* v, long size) {   // encoder.cu:12-23
  for (long i = 1, j = 0; i < size; ++i) {
    long bit = size >> 1;
    for (; j >= bit; bit >>= 1) j -= bit;
    j += bit;
    if (i < j) std::swap(v[i], v[j]);
  }
}

static inline std::complex<double> cmul(std::complex<double> a, std::complex<double> b) {
  // (a.re*b.re - a.im*b.im, a.re*b.im + a.im*b.re), each product rounded
  double re = a.real() * b.real() - a.imag() * b.imag();
  double im = a.real() * b.imag() + a.imag() * b.real();
  return std::complex<double>(re, im);
}

// ksiPows[j] = (cos(2 pi j / M), sin(2 pi j / M)), M = 2N (encoder.cu:87-94)
void oc_ksi_pows(int N, double* re, double* im) {
  long M = 2L * N;
  for (long j = 0; j < M; ++j) {
    double angle = 2.0 * M_PI * j / M;
    re[j] = cos(angle); im[j] = sin(angle);
  }
  re[M] = re[0]; im[M] = im[0];
}

static std::vector<long> rot_group(int N, long M) {
  std::vector<long> g(N / 2);
  uint64_t v = 1;
  for (long i = 0; i < N / 2; ++i) { g[i] = (long)v; v = (v * 5) % (uint64_t)M; }
  return g;
}

// fftSpecialInv (encoder.cu:75-124)
static void fft_special_inv(int N, std::complex<double>* vals, long size) {
  long M = 2L * N;
  std::vector<long> rg = rot_group(N, M);
  std::vector<double> kr(M + 1), ki(M + 1);
  oc_ksi_pows(N, kr.data(), ki.data());
  for (long len = size; len >= 1; len >>= 1)
    for (long i = 0; i < size; i += len) {
      long lenh = len >> 1, lenq = len << 2;
      for (long j = 0; j < lenh; ++j) {
        long idx = (lenq - (rg[j] % lenq)) * M / lenq;
        std::complex<double> u = vals[i + j] + vals[i + j + lenh];
        std::complex<double> v = vals[i + j] - vals[i + j + lenh];
        v = cmul(v, std::complex<double>(kr[idx], ki[idx]));
        vals[i + j] = u;
        vals[i + j + lenh] = v;
      }
    }
  array_bit_reverse(vals, size);
  for (long i = 0; i < size; ++i) vals[i] = std::complex<double>(vals[i].real() / size, vals[i].imag() / size);
}

// fftSpecial (encoder.cu:33-73).  The reference builds its tables with M = 4N
// there; the angles 2 pi idx / M are the same doubles as with M = 2N.
static void fft_special(int N, std::complex<double>* vals, long size) {
  long M = 2L * N;
  std::vector<long> rg = rot_group(N, M);
  std::vector<double> kr(M + 1), ki(M + 1);
  oc_ksi_pows(N, kr.data(), ki.data());
  array_bit_reverse(vals, size);
  for (long len = 2; len <= size; len <<= 1)
    for (long i = 0; i < size; i += len) {
      long lenh = len >> 1, lenq = len << 2;
      for (long j = 0; j < lenh; ++j) {
        long idx = (rg[j] % lenq) * M / lenq;
        std::complex<double> u = vals[i + j];
        std::complex<double> v = vals[i + j + lenh];
        v = cmul(v, std::complex<double>(kr[idx], ki[idx]));
        vals[i + j] = u + v;
        vals[i + j + lenh] = u - v;
      }
    }
}

// ckks_encode (encoder.cu:166-221) + ckks_convert_C2PC (encoder.cu:143-164):
// out is [nres][N] coefficient domain over the first `nres` Q primes.
void oc_encode(oc_ctx* c, const double* re, const double* im, int filled, int empty,
               uint64_t scale, int nres, uint64_t* out) {
  Ctx& C = *(Ctx*)c;
  int slots = filled + empty;
  std::vector<std::complex<double>> v(slots);
  for (int i = 0; i < filled; i++) v[i] = std::complex<double>(re[i], im[i]);
  fft_special_inv(C.N, v.data(), slots);
  std::fill(out, out + (size_t)nres * C.N, 0);
  int gap = (C.N >> 1) / slots;
  for (int lid = 0; lid < nres; lid++) {
    uint64_t p = C.P[lid].q;
    for (int sid = 0; sid < slots; sid++) {
      int64_t mir = (int64_t)(v[sid].real() * (double)scale);
      int64_t mii = (int64_t)(v[sid].imag() * (double)scale);
      // ADJUSTNEG(x, p) (encoder.cu:130)
      uint64_t rr = mir >= 0 ? (uint64_t)mir % p : p - ((uint64_t)(-mir) % p);
      uint64_t ri = mii >= 0 ? (uint64_t)mii % p : p - ((uint64_t)(-mii) % p);
      out[(size_t)lid * C.N + (size_t)sid * gap] = rr;
      out[(size_t)lid * C.N + (size_t)sid * gap + (C.N >> 1)] = ri;
    }
  }
}

// ckks_decode (encoder.cu:259-298) + ckks_convert_PC2C (encoder.cu:234-257):
// m0 = residue 0 of the coefficient-domain message.
void oc_decode(oc_ctx* c, const uint64_t* m0, int slots, uint64_t scale, double* re, double* im) {
  Ctx& C = *(Ctx*)c;
  uint64_t p = C.P[0].q;
  int gap = (C.N >> 1) / slots;
  std::vector<std::complex<double>> v(slots);
  for (int sid = 0; sid < slots; sid++) {
    uint64_t x = m0[(size_t)sid * gap], y = m0[(size_t)sid * gap + (C.N >> 1)];
    // ADJUSTSCALE(x, p, factor) (encoder.cu:131)
    double xr = x <= (p >> 1) ? ((double)x) / (double)scale : (((double)x) - ((double)p)) / (double)scale;
    double yr = y <= (p >> 1) ? ((double)y) / (double)scale : (((double)y) - ((double)p)) / (double)scale;
    v[sid] = std::complex<double>(xr, yr);
  }
  fft_special(C.N, v.data(), slots);
  for (int i = 0; i < slots; i++) { re[i] = v[i].real(); im[i] = v[i].imag(); }
}

// The FP64 special FFTs alone (for GPU encoder parity on the transform itself).
void oc_fft_special_inv(int N, double* re, double* im, int size) {
  std::vector<std::complex<double>> v(size);
  for (int i = 0; i < size; i++) v[i] = std::complex<double>(re[i], im[i]);
  fft_special_inv(N, v.data(), size);
  for (int i = 0; i < size; i++) { re[i] = v[i].real(); im[i] = v[i].imag(); }
}

void oc_fft_special(int N, double* re, double* im, int size) {
  std::vector<std::complex<double>> v(size);
  for (int i = 0; i < size; i++) v[i] = std::complex<double>(re[i], im[i]);
  fft_special(N, v.data(), size);
  for (int i = 0; i < size; i++) { re[i] = v[i].real(); im[i] = v[i].imag(); }
}

}  // extern "C"

// ===========================================================================
// DGT variant (aoa-dgt): folded Gaussian-integer transform.
//
// A degree-n polynomial is folded into N = n/2 Gaussian integers
// a_j + i a_{j+N} (poly_copy_to_device, aoa-dgt src/arithmetic/polynomial.cu:
// 92-116), twisted by powers of r, r^N = i (NTHROOT[p][N], aoa-dgt
// src/arithmetic/coprimes.cu), and transformed by a length-N DIF transform
// over GF(p)[i] with Z_p twiddles; N >= 1024 uses the two-kernel hierarchical
// form (Na x Nb, DGTFACT*, aoa-dgt include/AOADGT/cuda/dgt.h:26-35).  Data
// layout as in the reference: [residue][N] of {re, im} (16 bytes).
// ===========================================================================
namespace {

struct GI { uint64_t re, im; };

struct DgtPrime {
  uint64_t q; int nbits; uint64_t mu;
  uint64_t mul(uint64_t a, uint64_t b) const { return ref_mod((u128)a * b, q, nbits, mu); }
  uint64_t add(uint64_t a, uint64_t b) const { uint64_t s = a + b; return s >= q ? s - q : s; }   // addmod
  uint64_t sub(uint64_t a, uint64_t b) const { return a < b ? a + (q - b) : a - b; }             // submod
  GI gadd(GI a, GI b) const { return {add(a.re, b.re), add(a.im, b.im)}; }     // GIAdd, dgt.cu:486-495
  GI gsub(GI a, GI b) const { return {sub(a.re, b.re), sub(a.im, b.im)}; }     // GISub, dgt.cu:498-508
  // GIMul (Karatsuba), aoa-dgt src/cuda/dgt.cu:530-553
  GI gmul(GI a, GI b) const {
    uint64_t s1 = mul(a.re, b.re), s2 = mul(a.im, b.im);
    uint64_t s3 = mul(add(a.re, a.im), add(b.re, b.im));
    return {sub(s1, s2), sub(s3, add(s1, s2))};
  }
  std::vector<uint64_t> gjk_n, inv_n, gjk_a, inv_a, gjk_b, inv_b;   // compute_gjk
  std::vector<GI> nth, invnth;                                      // compute_nthroot
  std::vector<uint64_t> gN, ginvN;                                  // DGTEngine::init, dgt.cu:1918-1941
};

struct DgtCtx {
  int N = 0, Na = 0, Nb = 0;
  bool hier = false;
  std::vector<DgtPrime> P;
};

// DGTFACT* (aoa-dgt include/AOADGT/cuda/dgt.h:26-35): hierarchical from N = 1024.
static void dgt_fact(int N, int& Na, int& Nb) {
  switch (N) {
    case 1024: Na = 32; Nb = 32; break;
    case 2048: Na = 64; Nb = 32; break;
    case 4096: Na = 64; Nb = 64; break;
    case 8192: Na = 128; Nb = 64; break;
    case 16384: Na = 128; Nb = 128; break;
    case 32768: Na = 256; Nb = 128; break;
    default: Na = Nb = 0;
  }
}

// compute_gjk (aoa-dgt src/cuda/dgt.cu:1511-1560), one residue:
// g = proot^((p-1)/(2S)); gjk[s][j] = g^(j 2^(s+1)); inv[s][j] = g^((2S - j) 2^(s+1)).
static void dgt_gjk(const DgtPrime& P, uint64_t proot, int S, std::vector<uint64_t>& gjk, std::vector<uint64_t>& inv) {
  int L = ilog2i(S);
  gjk.assign((size_t)L * S, 0);
  inv.assign((size_t)L * S, 0);
  uint64_t g = oc_powmod(proot, (P.q - 1) / (2 * (uint64_t)S), P.q);
  for (int s = 0; s < L; s++)
    for (int j = 0; j < S; j++) {
      gjk[(size_t)s * S + j] = oc_powmod(g, (uint64_t)j * ((2ull * S) >> (L - s)), P.q);
      inv[(size_t)s * S + j] = oc_powmod(g, (uint64_t)(2 * S - j) * ((2ull * S) >> (L - s)), P.q);
    }
}

// dgttransform (dgt.cu:667-700) over all butterflies of stage s, inside the
// stage loop of doDGT (dgt.cu:741-765): DIF, natural in, bit-reversed out.
static void dgt_do(const DgtPrime& P, GI* d, int S, const std::vector<uint64_t>& gjk) {
  int L = ilog2i(S);
  for (int s = 0; s < L; s++) {
    int m = S / (2 << s);
    for (int cid = 0; cid < S / 2; cid++) {
      int j = cid * 2 * m / S;
      int i = j + (cid % (S / (2 * m))) * 2 * m;
      GI xi = d[i], xim = d[i + m];
      uint64_t a = gjk[(size_t)s * S + j];
      d[i] = P.gadd(xi, xim);
      GI t = P.gsub(xi, xim);
      d[i + m] = {P.mul(a, t.re), P.mul(a, t.im)};
    }
  }
}

// idgttransform (dgt.cu:702-739) + doIDGT (dgt.cu:768-790): DIT, stages L-1..0.
static void dgt_undo(const DgtPrime& P, GI* d, int S, const std::vector<uint64_t>& inv) {
  int L = ilog2i(S);
  for (int s = L - 1; s >= 0; s--) {
    int m = S / (2 << s);
    for (int cid = 0; cid < S / 2; cid++) {
      int j = cid * 2 * m / S;
      int i = j + (cid % (S / (2 * m))) * 2 * m;
      GI xi = d[i], xim = d[i + m];
      uint64_t a = inv[(size_t)s * S + j];
      GI axim = {P.mul(a, xim.re), P.mul(a, xim.im)};
      d[i] = P.gadd(xi, axim);
      d[i + m] = P.gsub(xi, axim);
    }
  }
}

static void dgt_forward(const DgtCtx& D, const DgtPrime& P, GI* x) {
  const int N = D.N;
  if (!D.hier) {                                     // dgt<N> (dgt.cu:995-1024)
    for (int t = 0; t < N; t++) x[t] = P.gmul(x[t], P.nth[t]);
    dgt_do(P, x, N, P.gjk_n);
    return;
  }
  const int Na = D.Na, Nb = D.Nb;
  std::vector<GI> tmp(N), s(std::max(Na, Nb));
  // hdgt_tr<Nb> with the GI twist (dgt.cu:805-848): column c of the Nb x Na
  // matrix, written transposed to row c.
  for (int c = 0; c < Na; c++) {
    for (int t = 0; t < Nb; t++) s[t] = P.gmul(x[t * Na + c], P.nth[t * Na + c]);
    dgt_do(P, s.data(), Nb, P.gjk_b);
    for (int t = 0; t < Nb; t++) tmp[c * Nb + t] = s[t];
  }
  // hdgt_tr<Na> with the integer twist gN (dgt.cu:850-901).
  for (int c = 0; c < Nb; c++) {
    for (int t = 0; t < Na; t++) {
      GI v = tmp[t * Nb + c];
      uint64_t w = P.gN[t * Nb + c];
      s[t] = {P.mul(w, v.re), P.mul(w, v.im)};
    }
    dgt_do(P, s.data(), Na, P.gjk_a);
    for (int t = 0; t < Na; t++) x[c * Na + t] = s[t];
  }
}

static void dgt_inverse(const DgtCtx& D, const DgtPrime& P, GI* x) {
  const int N = D.N;
  if (!D.hier) {                                     // idgt<N> (dgt.cu:1026-1053)
    dgt_undo(P, x, N, P.inv_n);
    for (int t = 0; t < N; t++) x[t] = P.gmul(x[t], P.invnth[t]);
    return;
  }
  const int Na = D.Na, Nb = D.Nb;
  std::vector<GI> tmp(N), s(std::max(Na, Nb));
  // hidgt<Na> (dgt.cu:903-949): rows of Na, untwist by ginvN (N^-1 inside).
  for (int r = 0; r < Nb; r++) {
    for (int t = 0; t < Na; t++) s[t] = x[r * Na + t];
    dgt_undo(P, s.data(), Na, P.inv_a);
    for (int t = 0; t < Na; t++) {
      uint64_t w = P.ginvN[r * Na + t];
      tmp[r * Na + t] = {P.mul(w, s[t].re), P.mul(w, s[t].im)};
    }
  }
  // hidgt_tr<Nb> (dgt.cu:951-993): columns, untwist by r^-n, not transposed.
  for (int c = 0; c < Na; c++) {
    for (int t = 0; t < Nb; t++) s[t] = tmp[t * Na + c];
    dgt_undo(P, s.data(), Nb, P.inv_b);
    for (int t = 0; t < Nb; t++) x[t * Na + c] = P.gmul(s[t], P.invnth[t * Na + c]);
  }
}

}  // namespace

extern "C" {

typedef void* oc_dgt;

// DGTEngine::init (aoa-dgt src/cuda/dgt.cu:1696-1945) for one folded length N:
// primes[i] with generator proots[i] and root roots[2i] + i roots[2i+1]
// (NTHROOT[p][N]); the inverse root is the GF(p)[i] inverse of r (what
// INVNTHROOT[p][N] holds, asserted by compute_nthroot, dgt.cu:1640-1644).
oc_dgt oc_dgt_create(int N, int nprimes, const uint64_t* primes, const uint64_t* proots, const uint64_t* roots) {
  DgtCtx* D = new DgtCtx();
  D->N = N;
  dgt_fact(N, D->Na, D->Nb);
  D->hier = D->Na > 0;
  D->P.resize(nprimes);
  for (int i = 0; i < nprimes; i++) {
    DgtPrime& P = D->P[i];
    P.q = primes[i]; P.nbits = nbits64(P.q); P.mu = oc_ref_barrett_mu(P.q);
    GI r = {roots[2 * i], roots[2 * i + 1]};
    uint64_t norm = (uint64_t)(((u128)r.re * r.re + (u128)r.im * r.im) % P.q);
    uint64_t ninv_norm = oc_invmod(norm, P.q);
    GI rinv = {oc_mulmod_exact(r.re, ninv_norm, P.q), oc_mulmod_exact(r.im ? P.q - r.im : 0, ninv_norm, P.q)};
    P.nth.resize(N); P.invnth.resize(N);
    uint64_t ninv = oc_invmod((uint64_t)N % P.q, P.q);
    GI a = {1, 0}, b = {1, 0};
    for (int t = 0; t < N; t++) {                      // compute_nthroot, dgt.cu:1646-1662
      P.nth[t] = a;
      P.invnth[t] = D->hier ? b : P.gmul(b, GI{ninv, 0});
      a = P.gmul(a, r);
      b = P.gmul(b, rinv);
    }
    if (!D->hier) {
      dgt_gjk(P, proots[i], N, P.gjk_n, P.inv_n);
    } else {
      dgt_gjk(P, proots[i], D->Na, P.gjk_a, P.inv_a);
      dgt_gjk(P, proots[i], D->Nb, P.gjk_b, P.inv_b);
      uint64_t g = oc_powmod(proots[i], (P.q - 1) / (uint64_t)N, P.q), ginv = oc_invmod(g, P.q);
      P.gN.resize(N); P.ginvN.resize(N);
      int lb = ilog2i(D->Nb);
      for (int cid = 0; cid < N; cid++) {
        P.gN[cid] = oc_powmod(g, (uint64_t)(cid / D->Nb) * bitrev(cid % D->Nb, lb), P.q);
        P.ginvN[cid] = oc_mulmod_exact(oc_powmod(ginv, (uint64_t)bitrev(cid / D->Na, lb) * (cid % D->Na), P.q), ninv,
                                       P.q);
      }
    }
  }
  return D;
}

void oc_dgt_destroy(oc_dgt h) { delete (DgtCtx*)h; }

// execute_dgt (dgt.cu:1055-1096) on residues first..first+nres-1 of x
// ([nres][N] Gaussian integers, interleaved re/im), in place.
void oc_dgt_fwd(oc_dgt h, uint64_t* x, int first, int nres) {
  DgtCtx& D = *(DgtCtx*)h;
  #pragma omp parallel for schedule(static)
  for (int r = 0; r < nres; r++) dgt_forward(D, D.P[first + r], (GI*)x + (size_t)r * D.N);
}

void oc_dgt_inv(oc_dgt h, uint64_t* x, int first, int nres) {
  DgtCtx& D = *(DgtCtx*)h;
  #pragma omp parallel for schedule(static)
  for (int r = 0; r < nres; r++) dgt_inverse(D, D.P[first + r], (GI*)x + (size_t)r * D.N);
}

// Element-wise GI product (mul_dgt<GaussianInteger>, dgt.cu:1327-1341): c = a * b.
void oc_gi_mul(oc_dgt h, const uint64_t* a, const uint64_t* b, uint64_t* c, int first, int nres) {
  DgtCtx& D = *(DgtCtx*)h;
  for (int r = 0; r < nres; r++) {
    const DgtPrime& P = D.P[first + r];
    for (int t = 0; t < D.N; t++) {
      size_t i = (size_t)r * D.N + t;
      ((GI*)c)[i] = P.gmul(((const GI*)a)[i], ((const GI*)b)[i]);
    }
  }
}

// The twist tables, for inspection by the tests: nth[t] = r^t, invnth[t].
void oc_dgt_twist(oc_dgt h, int rid, uint64_t* nth, uint64_t* invnth) {
  DgtCtx& D = *(DgtCtx*)h;
  std::memcpy(nth, D.P[rid].nth.data(), (size_t)D.N * 16);
  std::memcpy(invnth, D.P[rid].invnth.data(), (size_t)D.N * 16);
}

}  // extern "C"
