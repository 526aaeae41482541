// cb_sync.cuh -- the lane barrier of the persistent ensemble kernel: CTAs
// of one lane meet on a monotone counter in global memory.  Every wait is
// bounded in time (%globaltimer), so a missing CTA ends in an error flag the
// host reads, never in a hang.
#pragma once

#include "cb_tma.cuh"

namespace cb {

constexpr unsigned long long LANE_SYNC_LIMIT_NS = 2000000000ull; // a lane barrier gives up after 2 s

// Barrier over the w CTAs of a lane, with release/acquire at GPU scope so
// that each CTA's writes of the phase are visible to the lane's next phase,
// and proxy fences so that bulk tensor copies (the async proxy) of the next
// phase see them too.  Bounded: gives up after limit_ns (setting the abort
// flag) or when another lane has given up, and then returns false in every
// thread.
__device__ __forceinline__ bool lane_sync(unsigned *ctr, int w, int *abort, unsigned long long limit_ns = LANE_SYNC_LIMIT_NS) {
  __shared__ int s_ok;
  asm volatile("fence.proxy.async.global;" ::: "memory");
  __syncthreads();
  if (threadIdx.x == 0 && threadIdx.y == 0) {
    int ok = 1;
    if (w > 1) {
      __threadfence();
      const unsigned old = atomicAdd(ctr, 1u);
      const unsigned target = (old / (unsigned)w + 1u) * (unsigned)w;
      const unsigned long long t0 = global_ns();
      while (true) {
        unsigned v;
        asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(ctr) : "memory");
        if ((int)(v - target) >= 0) break;
        if (*(volatile int *)abort) {
          ok = 0;
          break;
        }
        if (global_ns() - t0 > limit_ns) {
          atomicExch(abort, 1);
          ok = 0;
          break;
        }
        __nanosleep(64);
      }
      __threadfence();
      asm volatile("fence.proxy.async.global;" ::: "memory");
    }
    s_ok = ok;
  }
  __syncthreads();
  return s_ok != 0;
}

} // namespace cb
