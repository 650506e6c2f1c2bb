// TMA (2-D tiled tensor loads) and mbarrier helpers in inline PTX, shared by
// the tile kernels that stage their windows through the TMA unit.
#pragma once
#include <cuda.h>
#include <cstdint>

namespace h266 {
namespace tile_dev {

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(unsigned long long *bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_expect_tx(unsigned long long *bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}

// 2-D tiled tensor load of the box at (x, y) (elements) into shared memory,
// completing on `bar`.  Every call site keeps x * 2 bytes a multiple of 16.
__device__ __forceinline__ void tma_load_2d(void *dst, const CUtensorMap *map, int x, int y, unsigned long long *bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(
          smem_u32(dst)),
      "l"(map), "r"(x), "r"(y), "r"(smem_u32(bar))
      : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(unsigned long long *bar, uint32_t phase) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(phase)
      : "memory");
  return ok != 0;
}

__device__ __forceinline__ uint64_t global_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Polls the barrier's phase `phase` for at most `limit_ns` (default 20 ms).
__device__ __forceinline__ bool mbar_wait_bounded(unsigned long long *bar, uint32_t phase,
                                                  uint64_t limit_ns = 20000000) {
  if (mbar_try_wait(bar, phase)) return true;
  const uint64_t t0 = global_ns();
  for (;;) {
    if (mbar_try_wait(bar, phase)) return true;
    if (global_ns() - t0 > limit_ns) return false;
  }
}

// A tensor map written to global memory before the launch, made visible to
// the tensor-map proxy.
__device__ __forceinline__ void tmap_acquire(const CUtensorMap *m) {
  asm volatile("fence.proxy.tensormap::generic.acquire.gpu [%0], 128;" ::"l"(m) : "memory");
}

}  // namespace tile_dev
}  // namespace h266
