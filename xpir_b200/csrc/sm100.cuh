// sm_100a building blocks: shared-memory mbarriers with bounded waits, TMA tiled loads
// (no multicast), and host-side tensor-map encoding through the driver entry point.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace xpir {

// Each try_wait poll may suspend the thread for up to kSuspendNs (it wakes as soon as the
// phase completes), so a waiting warp costs almost no issue slots.  kSpinLimit polls bound
// one wait to about kSpinLimit * kSuspendNs (~2.6 s); past it the kernel records an error
// and returns instead of spinning forever.
constexpr uint32_t kSuspendNs = 20000;
constexpr uint32_t kSpinLimit = 1u << 17;

// Error codes a kernel can leave in its status word.
enum KernelStatus : int { kStatusOk = 0, kStatusWaitTimeout = 1 };

__device__ __forceinline__ uint32_t smem_addr(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}

// Makes barrier initialisation visible to the async (TMA) proxy.
__device__ __forceinline__ void mbar_fence_init() { asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory"); }

__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
  asm volatile("{\n .reg .b64 st;\n mbarrier.arrive.shared::cta.b64 st, [%0];\n}\n" ::"r"(smem_addr(bar)) : "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, uint32_t bytes) {
  asm volatile("{\n .reg .b64 st;\n mbarrier.arrive.expect_tx.shared::cta.b64 st, [%0], %1;\n}\n" ::"r"(smem_addr(bar)),
               "r"(bytes)
               : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_addr(bar)), "r"(parity), "n"(kSuspendNs)
      : "memory");
  return ok != 0;
}

// Waits for the phase with the given parity to complete; false after `limit` polls.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity, uint32_t limit = kSpinLimit) {
  for (uint32_t i = 0; i < limit; ++i)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}

// TMA tiled loads into this CTA's shared memory, completion signalled on `bar`.
__device__ __forceinline__ void tma_load_4d(void *dst, const CUtensorMap *map, int c0, int c1, int c2, int c3,
                                            uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], "
      "[%6];\n" ::"r"(smem_addr(dst)),
      "l"((uint64_t)map), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(smem_addr(bar))
      : "memory");
}

__device__ __forceinline__ void tma_prefetch_desc(const CUtensorMap *map) {
  asm volatile("prefetch.tensormap [%0];\n" ::"l"((uint64_t)map) : "memory");
}

// Host: cuTensorMapEncodeTiled for a u64 tensor of rank 4 (dims innermost first, byte
// strides of dims 1..3).  Returns false if the driver rejects the description.
bool encode_tensor_map_u64_4d(CUtensorMap *map, const void *base, const uint64_t dims[4], const uint64_t strides[3],
                              const uint32_t box[4]);


}  // namespace xpir
