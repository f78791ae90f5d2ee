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
//  - the array's device address is looked up once per CUDA context on the
//    first call made in that context (with the engine's device current) and
//    cached under the context's handle, so a caller that switches between the
//    primary context and contexts of its own gets the address that belongs to
//    the current one; make that first call before any stream capture.  After
//    cudaDeviceReset the next call looks the address up again only if the new
//    primary context has a new handle, so do not reset a device between calls;
//  - every call on a device shares the one array and leaves its contents
//    behind: calls whose work overlaps on the GPU (other streams, other
//    contexts, other threads) race on it and must be serialised by the caller;
//  - no part of the scratch has to start at zero: the pipeline writes every
//    scratch word it reads earlier in the same call.
#include <cuda.h>   // CUcontext and CUresult (types only: the driver call is fetched through the runtime)

#include <mutex>
#include <vector>

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

struct ScratchSlot {
  CUcontext ctx;
  uint64_t* addr;
};
std::mutex g_setup_mu;
std::vector<ScratchSlot> g_slots;     // one entry per CUDA context that has made a call

// The calling thread's current CUDA context (cuCtxGetCurrent, fetched once
// through the runtime so the library needs no link against libcuda).
CUcontext current_context() {
  using Fn = CUresult (*)(CUcontext*);
  static Fn fn = [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      return (Fn) nullptr;
    return (Fn)p;
  }();
  if (!fn) throw AoaError(AOA_ERR_CUDA, "cuCtxGetCurrent is not available from the driver");
  CUcontext ctx = nullptr;
  if (fn(&ctx) != CUDA_SUCCESS) throw AoaError(AOA_ERR_CUDA, "cuCtxGetCurrent failed");
  return ctx;
}

// Device address of the scratch array in the current context (whose device
// is the engine's, `device`).
uint64_t* scratch_here(int device) {
  CUcontext ctx = current_context();
  if (!ctx) {                         // a thread without a current context: bind the device's primary one
    AOA_CUDA(cudaSetDevice(device));
    ctx = current_context();
    if (!ctx) throw AoaError(AOA_ERR_CUDA, "no current CUDA context");
  }
  std::lock_guard<std::mutex> lock(g_setup_mu);
  for (const ScratchSlot& s : g_slots)
    if (s.ctx == ctx) return s.addr;
  void* p = nullptr;
  const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
  if (e != cudaSuccess || !p)
    throw AoaError(AOA_ERR_CUDA, std::string("no-alloc scratch address lookup failed: ") + cudaGetErrorString(e));
  g_slots.push_back({ctx, (uint64_t*)p});
  return (uint64_t*)p;
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
    hmult_with_scratch(c->c, out, a, b, evk, true, scratch_here(cur));
  });
}

}  // extern "C"
