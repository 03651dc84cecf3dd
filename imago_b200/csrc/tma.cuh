// tma.cuh -- TMA tensor copies into shared memory with mbarrier completion
// (sm_90 and later PTX), bounded waits, and the host-side tensor-map
// encoder reached through the runtime's driver entry point.
//
// No copy here uses cluster multicast: every load reads this GPU's own
// memory into this CTA's shared memory.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <cstdint>

#include "common.cuh"

namespace imago {

__device__ __forceinline__ unsigned smem_addr(const void *p) {
  return (unsigned)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_addr(bar)), "r"(count)
               : "memory");
}

// Make initialised barriers visible to the async proxy before any copy
// names them.
__device__ __forceinline__ void mbar_init_fence() {
  asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
}

// Order this CTA's earlier generic-proxy accesses of shared memory before
// the async-proxy writes of a copy issued after it.
__device__ __forceinline__ void fence_proxy_async() {
  asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(
                   smem_addr(bar)),
               "r"(bytes)
               : "memory");
}

// One tiled 3-D tensor copy global -> shared, completing `bar`'s
// transaction count.  Coordinates are in elements, innermost first; the
// innermost one is always 0 here (16-byte aligned by construction).
__device__ __forceinline__ void tma_load_3d(void *dst, const CUtensorMap *map, uint64_t *bar,
                                            int x, int y, int z) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3, %4}], [%5];\n" ::"r"(smem_addr(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(smem_addr(bar))
      : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, unsigned parity) {
  unsigned ok = 0;
  asm volatile(
      "{\n .reg .pred p;\n"
      " mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
      " selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_addr(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;\n" : "=l"(t));
  return t;
}

// Wait for phase `parity` of `bar` to complete, for at most about limit_ns
// (kWaitLimitNs unless given, and never more than kWaitPolls polls).
// False when the bound ran out.
constexpr unsigned long long kWaitLimitNs = 1000000000ULL;  // 1 s
constexpr unsigned kWaitPolls = 1u << 26;

__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar, unsigned parity,
                                                  unsigned long long limit_ns = kWaitLimitNs) {
  if (mbar_try_wait(bar, parity)) return true;
  const unsigned long long t0 = global_ns();
  for (unsigned it = 1; it < kWaitPolls; ++it) {
    if (mbar_try_wait(bar, parity)) return true;
    if ((it & 255u) == 0 && global_ns() - t0 > limit_ns) return false;
  }
  return false;
}

// Record a device-side failure for the host (first one wins).
__device__ __forceinline__ void report_status(int *flag, int status) {
  if (flag) atomicCAS(flag, 0, status);
}

// Host: encode a 3-D FP64 tiled tensor map (dims innermost first, strides
// in bytes of dims 1 and 2), no interleave, no swizzle, out-of-range
// elements zero-filled.  Returns false when the driver refuses the map.
bool encode_tensor_map_f64_3d(CUtensorMap *map, const void *base, const uint64_t dims[3],
                              const uint64_t strides[2], const uint32_t box[3]);

}  // namespace imago
