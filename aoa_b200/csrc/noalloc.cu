// HMult + relinearise + rescale without any device allocation.
//
// Who needs this: callers that are not allowed to allocate device memory
// while they evaluate.  Typical cases are a host application that reserves
// the whole GPU memory budget for its own allocator and forbids libraries to
// call cudaMalloc behind its back, and a latency-critical serving thread for
// which cudaMalloc / cudaFree are off limits because they can synchronise the
// device and serialise on the driver's allocation lock.  The regular entry
// point (aoa_hmult_relin_rescale) allocates its key-switch workspace on the
// context's stream the first time it needs it; this one instead runs the same
// kernels on a fixed scratch array that is part of the library's device image.
//
// Contract:
//  - scratch: one file-scope device array of kScratchBytes (32 MiB), created
//    when the library is loaded on a device and held by every device that
//    loads the library until the process exits;
//  - the parameter set must need at most that much workspace, otherwise the
//    call fails with AOA_ERR_BAD_PARAM and says how much it would need;
//  - the array's device address is looked up once per device on the first call
//    made on that device (with the engine's device current); make that first
//    call before any stream capture;
//  - every call on a device shares the one array and leaves its contents
//    behind: calls whose work overlaps on the GPU (other streams, other
//    contexts, other threads) race on it and must be serialised by the caller;
//  - no part of the scratch has to start at zero: the pipeline writes every
//    scratch word it reads earlier in the same call.
#include <mutex>

#include "aoa_internal.h"

namespace aoa {
size_t workspace_words(const Engine& E);
void hmult_with_scratch(Ctx& C, aoa_ct* out, aoa_ct* a, aoa_ct* b, const aoa_swk* evk, bool do_rescale,
                        uint64_t* scratch);
}  // namespace aoa

using namespace aoa;

namespace {

constexpr size_t kScratchWords = size_t(4) << 20;            // 4 Mi words
constexpr size_t kScratchBytes = kScratchWords * sizeof(uint64_t);   // 32 MiB

static __device__ __align__(256) uint64_t g_noalloc_scratch[kScratchWords];

constexpr int kMaxDevices = 64;
std::mutex g_setup_mu;
uint64_t* g_scratch_addr[kMaxDevices] = {};

// Device address of the scratch array on `device` (which must be current).
uint64_t* scratch_on(int device) {
  if (device < 0 || device >= kMaxDevices) throw AoaError(AOA_ERR_BAD_PARAM, "device ordinal out of range");
  std::lock_guard<std::mutex> lock(g_setup_mu);
  if (!g_scratch_addr[device]) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p)
      throw AoaError(AOA_ERR_CUDA, std::string("no-alloc scratch address lookup failed: ") + cudaGetErrorString(e));
    g_scratch_addr[device] = (uint64_t*)p;
  }
  return g_scratch_addr[device];
}

}  // namespace

extern "C" {

int aoa_hmult_relin_rescale_noalloc(aoa_ctx* c, aoa_ct* out, aoa_ct* a, aoa_ct* b, const aoa_swk* evk) {
  if (!c || !out || !a || !b) return fail(AOA_ERR_BAD_PARAM, "null argument");
  return guarded([&] {
    const Engine& E = *c->c.E;
    const size_t need = workspace_words(E) * sizeof(uint64_t);
    if (need > kScratchBytes)
      throw AoaError(AOA_ERR_BAD_PARAM, "parameters need " + std::to_string(need >> 20) + " MiB of scratch; the "
                                        "allocation-free HMult is limited to " +
                                            std::to_string(kScratchBytes >> 20) + " MiB");
    int cur = -1;
    AOA_CUDA(cudaGetDevice(&cur));
    if (cur != E.device)
      throw AoaError(AOA_ERR_BAD_PARAM, "make the engine's device current before calling the no-alloc HMult");
    hmult_with_scratch(c->c, out, a, b, evk, true, scratch_on(cur));
  });
}

}  // extern "C"
