// Asynchronous-copy and mbarrier helpers (sm_100a), shared by the transform
// and basis-conversion kernels.  Every wait is bounded: a wait that runs out
// returns false and the caller records an error instead of hanging.
#pragma once
#include <cstdint>

namespace aoa {

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

constexpr int kSpinLimit = 1 << 20;     // bounded mbarrier waits (default; engine knob "spin_limit")

__device__ __forceinline__ void mbar_init(uint64_t* mb, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(mb)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_init_fence() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t* mb) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(mb)) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* mb, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(mb)), "r"(bytes)
               : "memory");
}

// global -> shared bulk copy; bytes % 16 == 0, both addresses 16-byte aligned
__device__ __forceinline__ void bulk_g2s(uint32_t dst, const void* src, unsigned bytes, uint64_t* mb) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
      "l"(src), "r"(bytes), "r"(smem_u32(mb))
      : "memory");
}

// 4-D tensor-map tile load into shared memory (no multicast); the tensor map
// is a __grid_constant__ kernel parameter, x * element size a multiple of 16
__device__ __forceinline__ void tma_load_4d(uint32_t dst, const void* tmap, int x, int y, int z, int w,
                                            uint64_t* mb) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}],"
      " [%6];" ::"r"(dst),
      "l"((uint64_t)tmap), "r"(x), "r"(y), "r"(z), "r"(w), "r"(smem_u32(mb))
      : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* mb, unsigned parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(mb)), "r"(parity)
      : "memory");
  return ok != 0;
}

// Waits for phase `parity` of the barrier; gives up after `limit` tries.
// The waits for a kernel's own work use the engine's limit (a kernel
// argument); the drain after an expired wait, which lets copies and MMAs in
// flight land before the CTA exits, always uses the default bound.
__device__ __forceinline__ bool mbar_wait(uint64_t* mb, unsigned parity, int limit = kSpinLimit) {
  for (int i = 0; i < limit; i++)
    if (mbar_try_wait(mb, parity)) return true;
  return false;
}

__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

}  // namespace aoa
