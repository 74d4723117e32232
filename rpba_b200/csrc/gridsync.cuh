// gridsync.cuh -- bounded grid-wide barrier for cooperative launches.
#pragma once

#include <cuda_runtime.h>

namespace rpba {

constexpr unsigned long long BAR_TIMEOUT_NS = 2000000000ull;  // 2 s

__device__ __forceinline__ unsigned long long gtimer() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Barrier over all CTAs of a cooperative launch (co-residency guaranteed).
// bar[0] counts arrivals, bar[1] is the generation.  The wait is bounded:
// after timeout_ns (BAR_TIMEOUT_NS unless a caller shortens it) it sets err
// bit 2 and returns false; every caller then leaves the kernel.
__device__ __forceinline__ bool grid_barrier(unsigned *bar, unsigned nblocks, int *err,
                                             unsigned long long timeout_ns = BAR_TIMEOUT_NS) {
  __syncthreads();
  if (threadIdx.x == 0) {
    volatile unsigned *vgen = bar + 1;
    const unsigned gen = *vgen;
    __threadfence();
    const unsigned arrived = atomicAdd(bar, 1u);
    if (arrived == nblocks - 1) {
      atomicExch(bar, 0u);
      __threadfence();
      atomicAdd(bar + 1, 1u);
    } else {
      const unsigned long long t0 = gtimer();
      while (*vgen == gen) {
        if (*(volatile int *)err) break;
        if (gtimer() - t0 > timeout_ns) {
          atomicOr(err, 2);
          break;
        }
        __nanosleep(40);
      }
    }
    __threadfence();
  }
  __syncthreads();
  return *(volatile int *)err == 0;
}

}  // namespace rpba
