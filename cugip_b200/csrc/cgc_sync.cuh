// Grid-wide barrier for cooperative (co-resident) launches.
#pragma once
#include <cstdint>
#include "cgc.h"

namespace cgc {

__device__ __forceinline__ uint64_t sync_globaltimer_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// bar[0] counts arrivals, bar[1] is the generation.  Waits are bounded: after
// `limit_ns` the waiting CTA records CGC_ERR_TIMEOUT in *err and every CTA
// leaves at its next barrier.  Returns false once an error was recorded.
__device__ __forceinline__ bool grid_barrier(uint32_t* bar, int32_t* err, uint64_t limit_ns) {
  __syncthreads();
  if (threadIdx.x == 0) {
    volatile uint32_t* gen = bar + 1;
    const uint32_t g0 = *gen;
    __threadfence();
    const uint32_t arrived = atomicAdd(bar, 1u) + 1u;
    if (arrived == gridDim.x) {
      atomicExch(bar, 0u);
      __threadfence();
      atomicAdd(bar + 1, 1u);
    } else {
      const uint64_t t0 = sync_globaltimer_ns();
      while (*gen == g0) {
        __nanosleep(64);
        if (sync_globaltimer_ns() - t0 > limit_ns) {
          atomicCAS(err, 0, CGC_ERR_TIMEOUT);
          break;
        }
      }
    }
    __threadfence();
  }
  __syncthreads();
  return *(volatile int32_t*)err == 0;
}

}  // namespace cgc
