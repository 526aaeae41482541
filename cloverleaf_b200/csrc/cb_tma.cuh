// cb_tma.cuh -- TMA staging of halo-padded mesh tiles into shared memory.
//
// A kernel block owns an output tile of 64 columns x TY rows whose first
// element is (x0, y0).  Each input field it reads is copied, with a 4-deep
// halo on every side, from HBM into shared memory by one bulk tensor copy
// (cp.async.bulk.tensor.2d, no multicast: single CTA, this GPU's memory)
// that completes on a shared-memory mbarrier.  Element (i, j) of a staged
// field then sits at box[(j - y0 + 4) * BOX_X + (i - x0 + 4)], so every
// stencil neighbour is a shared-memory load at a constant offset.
//
// Tensor-map coordinates: the map's base is the raw allocation, whose
// element (i, j) is at x = off + i, y = j.  With off = 30 (FP64) or 62
// (FP32) and x0 = 2 + 64k, a box starting at x = off + x0 - 4 begins on a
// 16-byte boundary, as TMA requires.
#pragma once

#include <cuda.h>
#include <cstdint>

namespace cb {

constexpr int TILE_X = 64;  // output columns per block
constexpr int HALO = 4;     // staged halo on every side
constexpr int BOX_X = TILE_X + 2 * HALO;
constexpr unsigned long long TMA_WAIT_LIMIT_NS = 1000000000ull; // a staging wait gives up after 1 s

// Up to eight tensor maps passed by value as one __grid_constant__ parameter.
struct Maps {
  CUtensorMap m[8];
};

__device__ __forceinline__ uint32_t smem_addr(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes) : "memory");
}

__device__ __forceinline__ void tma_load_2d(void *dst, const CUtensorMap *map, int x, int y, uint64_t *bar) {
  asm volatile("cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(
                   smem_addr(dst)),
               "l"(map), "r"(x), "r"(y), "r"(smem_addr(bar))
               : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, unsigned phase) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_addr(bar)), "r"(phase)
      : "memory");
  return ok != 0;
}

// Waits for the barrier's phase for at most limit_ns (the clock read every
// 64 polls); on give-up it records an error for the host and reports
// failure.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, unsigned phase, int *err, unsigned long long limit_ns = TMA_WAIT_LIMIT_NS) {
  if (mbar_try_wait(bar, phase)) return true;
  const unsigned long long t0 = global_ns();
  do {
    for (int it = 0; it < 64; ++it)
      if (mbar_try_wait(bar, phase)) return true;
  } while (global_ns() - t0 <= limit_ns);
  if (err) atomicExch(err, 1);
  return false;
}

} // namespace cb
