// Binary wire format for ciphertexts and switching keys: the serving
// boundary's request / response payload.  The reference exchanges JSON with
// decimal residues (cipher_export / cipher_import, aoa-ntt src/ckks/
// cipher_t.cpp:42-81; CKKSContext::export_keys / load_keys, ckkscontext.cpp:
// 50-100; the JSON form is in the Python package); this format carries the
// same state in binary, little-endian:
//   header (64 bytes): magic "AOACKKS1" | kind u32 (1 ciphertext, 2 switching
//   key) | log_n u32 | nprimes u32 (primes of the engine) | nlimbs u32 (limbs
//   per poly that follow) | level i32 | slots i32 | domain i32 | reserved u32
//   | scale u64 | primes fingerprint u64 (FNV-1a over k and the engine's primes) | 8
//   reserved bytes
//   body: 2 polys x nlimbs x N residues, u64
// A ciphertext carries its live limbs 0..level in its current domain (no
// transform on either side); a switching key carries both (k + kl)-limb polys
// in its transform domain.  Reading checks the magic, kind, ring, fingerprint,
// length, level and slot count, and that every residue is below its prime,
// and rejects anything else.
#include <cstring>

#include "aoa_internal.h"

using namespace aoa;

namespace {

constexpr char kMagic[8] = {'A', 'O', 'A', 'C', 'K', 'K', 'S', '1'};
constexpr uint32_t kKindCt = 1, kKindKey = 2;

struct WireHeader {
  char magic[8];
  uint32_t kind, log_n, nprimes, nlimbs;
  int32_t level, slots, domain;
  uint32_t reserved;
  uint64_t scale, fingerprint;
  uint64_t pad;
};
static_assert(sizeof(WireHeader) == 64, "wire header is 64 bytes");

// FNV-1a over the Q prime count and the Q | B primes: buffers move only
// between engines with the same primes and the same Q / B split
uint64_t fingerprint(const Engine& E) {
  uint64_t h = 0xcbf29ce484222325ull;
  for (int b = 0; b < 4; b++) {
    h ^= ((uint32_t)E.k >> (8 * b)) & 0xff;
    h *= 0x100000001b3ull;
  }
  for (uint64_t q : E.primes)
    for (int b = 0; b < 8; b++) {
      h ^= (q >> (8 * b)) & 0xff;
      h *= 0x100000001b3ull;
    }
  return h;
}

WireHeader make_header(const Engine& E, uint32_t kind, int nlimbs) {
  WireHeader h{};
  memcpy(h.magic, kMagic, 8);
  h.kind = kind;
  h.log_n = (uint32_t)E.log_n;
  h.nprimes = (uint32_t)E.nprimes;
  h.nlimbs = (uint32_t)nlimbs;
  h.fingerprint = fingerprint(E);
  return h;
}

WireHeader read_header(const Engine& E, const uint8_t* buf, size_t len, uint32_t kind) {
  if (!buf || len < sizeof(WireHeader)) throw AoaError(AOA_ERR_BAD_PARAM, "wire buffer shorter than its header");
  WireHeader h;
  memcpy(&h, buf, sizeof h);
  if (memcmp(h.magic, kMagic, 8) != 0) throw AoaError(AOA_ERR_BAD_PARAM, "not an aoa wire buffer");
  if (h.kind != kind) throw AoaError(AOA_ERR_BAD_PARAM, "wire buffer holds another kind of object");
  if (h.log_n != (uint32_t)E.log_n || h.nprimes != (uint32_t)E.nprimes || h.fingerprint != fingerprint(E))
    throw AoaError(AOA_ERR_BAD_PARAM, "wire buffer was written for other parameters");
  if (h.domain != AOA_COEF && h.domain != AOA_NTT && h.domain != AOA_DGT)
    throw AoaError(AOA_ERR_BAD_PARAM, "wire buffer has a bad domain");
  const size_t body = (size_t)2 * h.nlimbs * E.N * 8;
  if (len != sizeof(WireHeader) + body) throw AoaError(AOA_ERR_BAD_PARAM, "wire buffer length does not match");
  return h;
}

// Every word of the body must be a canonical residue of its limb's prime:
// the kernels' lazy bounds assume inputs below q, so a corrupted or foreign
// buffer is rejected here instead of giving wrong results later.
void check_residues(const Engine& E, const uint8_t* body, int npolys, int nlimbs) {
  const size_t N = (size_t)E.N;
  for (int p = 0; p < npolys; p++)
    for (int i = 0; i < nlimbs; i++) {
      const uint64_t q = E.primes[i];
      const uint8_t* limb = body + ((size_t)p * nlimbs + i) * N * 8;
      for (size_t j = 0; j < N; j++) {
        uint64_t v;
        memcpy(&v, limb + j * 8, 8);
        if (v >= q)
          throw AoaError(AOA_ERR_BAD_PARAM, "wire buffer holds a residue >= its prime (poly " + std::to_string(p) +
                                                ", limb " + std::to_string(i) + ", word " + std::to_string(j) + ")");
      }
    }
}

}  // namespace

extern "C" {

size_t aoa_ct_wire_size(const aoa_ctx* c, const aoa_ct* ct) {
  if (!c || !ct) return 0;
  const Engine& E = *c->c.E;
  return sizeof(WireHeader) + (size_t)2 * (ct->level + 1) * E.N * 8;
}

int aoa_ct_serialize(aoa_ctx* c, const aoa_ct* ct, uint8_t* buf, size_t cap, size_t* len) {
  if (!c || !ct || !buf || !len) return fail(AOA_ERR_BAD_PARAM, "null argument");
  return guarded([&] {
    const Engine& E = *c->c.E;
    const int nl = ct->level + 1;
    const size_t need = aoa_ct_wire_size(c, ct);
    if (cap < need) throw AoaError(AOA_ERR_BAD_PARAM, "wire buffer too small");
    WireHeader h = make_header(E, kKindCt, nl);
    h.level = ct->level;
    h.slots = ct->slots;
    h.domain = ct->domain;
    h.scale = ct->scale;
    memcpy(buf, &h, sizeof h);
    const size_t poly = (size_t)nl * E.N * 8;
    for (int p = 0; p < 2; p++)
      AOA_CUDA(cudaMemcpyAsync(buf + sizeof h + p * poly, ct->d + (size_t)p * E.k * E.N, poly, cudaMemcpyDeviceToHost,
                               c->c.stream));
    AOA_CUDA(cudaStreamSynchronize(c->c.stream));
    *len = need;
  });
}

int aoa_ct_deserialize(aoa_ctx* c, aoa_ct* ct, const uint8_t* buf, size_t len) {
  if (!c || !ct || !buf) return fail(AOA_ERR_BAD_PARAM, "null argument");
  return guarded([&] {
    const Engine& E = *c->c.E;
    const WireHeader h = read_header(E, buf, len, kKindCt);
    if (h.nlimbs < 1 || h.nlimbs > (uint32_t)E.k || h.level != (int32_t)h.nlimbs - 1)
      throw AoaError(AOA_ERR_BAD_PARAM, "wire ciphertext has a bad level");
    if (h.slots < 0 || h.slots > E.N / 2 || (h.slots & (h.slots - 1)) != 0)
      throw AoaError(AOA_ERR_BAD_PARAM, "wire ciphertext has a bad slot count (0 or a power of two <= N/2)");
    check_residues(E, buf + sizeof h, 2, (int)h.nlimbs);
    const size_t poly = (size_t)h.nlimbs * E.N * 8;
    for (int p = 0; p < 2; p++)
      AOA_CUDA(cudaMemcpyAsync(ct->d + (size_t)p * E.k * E.N, buf + sizeof h + p * poly, poly, cudaMemcpyHostToDevice,
                               c->c.stream));
    AOA_CUDA(cudaStreamSynchronize(c->c.stream));     // the caller may reuse buf on return
    ct->level = h.level;
    ct->slots = h.slots;
    ct->scale = h.scale;
    ct->domain = h.domain;
  });
}

size_t aoa_swk_wire_size(const aoa_ctx* c) {
  if (!c) return 0;
  const Engine& E = *c->c.E;
  return sizeof(WireHeader) + (size_t)2 * E.nprimes * E.N * 8;
}

int aoa_swk_serialize(aoa_ctx* c, const aoa_swk* k, uint8_t* buf, size_t cap, size_t* len) {
  if (!c || !k || !buf || !len) return fail(AOA_ERR_BAD_PARAM, "null argument");
  return guarded([&] {
    const Engine& E = *c->c.E;
    const size_t need = aoa_swk_wire_size(c);
    if (cap < need) throw AoaError(AOA_ERR_BAD_PARAM, "wire buffer too small");
    WireHeader h = make_header(E, kKindKey, E.nprimes);
    h.level = E.k - 1;
    h.domain = k->domain;
    memcpy(buf, &h, sizeof h);
    AOA_CUDA(cudaMemcpyAsync(buf + sizeof h, k->d, need - sizeof h, cudaMemcpyDeviceToHost, c->c.stream));
    AOA_CUDA(cudaStreamSynchronize(c->c.stream));
    *len = need;
  });
}

int aoa_swk_deserialize(aoa_ctx* c, const uint8_t* buf, size_t len, aoa_swk** out) {
  if (!c || !buf || !out) return fail(AOA_ERR_BAD_PARAM, "null argument");
  return guarded([&] {
    const Engine& E = *c->c.E;
    const WireHeader h = read_header(E, buf, len, kKindKey);
    if (h.nlimbs != (uint32_t)E.nprimes || h.domain == AOA_COEF)
      throw AoaError(AOA_ERR_BAD_PARAM, "wire key has a bad shape or domain");
    if (h.domain != c->c.transform)
      throw AoaError(AOA_ERR_BAD_PARAM, "the switching key is in another transform domain");
    check_residues(E, buf + sizeof h, 2, E.nprimes);
    aoa_swk* k = new aoa_swk();
    if (cudaMallocAsync(&k->d, len - sizeof h, c->c.stream) != cudaSuccess) {
      cudaGetLastError();
      delete k;
      throw AoaError(AOA_ERR_OOM, "key allocation failed");
    }
    AOA_CUDA(cudaMemcpyAsync(k->d, buf + sizeof h, len - sizeof h, cudaMemcpyHostToDevice, c->c.stream));
    AOA_CUDA(cudaStreamSynchronize(c->c.stream));
    k->domain = h.domain;
    *out = k;
  });
}

}  // extern "C"
