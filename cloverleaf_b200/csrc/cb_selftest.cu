// cb_selftest.cu -- diagnostics the test suite calls:
// cb_selftest_width_ratio checks width_ratio (cb_mesh.cuh), the FP64
// kernels' quotient of two mesh widths with a precomputed reciprocal, against
// the division operator on the device, bit for bit; cb_selftest_wait_limits
// runs the kernels' two bounded waits (a tile's staging wait, cb_tma.cuh,
// and the ensemble's lane barrier, cb_sync.cuh) to their limit on purpose,
// on a barrier nothing completes, and reports that each gave up and set its
// error flag.
#include <cuda_runtime.h>

#include <string>

#include "../../include/cloverb200.h"
#include "cb_mesh.cuh"
#include "cb_sync.cuh"

namespace cb {
int set_last_error(int code, const std::string &msg);
} // namespace cb

namespace {

// splitmix64 (S. Vigna), the pseudo-random stream of the test.
__device__ __forceinline__ unsigned long long mix(unsigned long long z) {
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

// Operands: positive, a random significand with an exponent drawn over
// [2^-40, 2^40] for x and over [2^-20, 2^4] for w, or x and w widths
// 10 / n of meshes up to 65536 cells.
__global__ void k_width_ratio(unsigned long long n, unsigned long long seed, unsigned long long *bad, double *example) {
  const unsigned long long stride = (unsigned long long)gridDim.x * blockDim.x;
  unsigned long long local = 0;
  for (unsigned long long k = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; k < n; k += stride) {
    const unsigned long long a = mix(seed ^ (2 * k)), b = mix(seed ^ (2 * k + 1));
    const double sx = __longlong_as_double((long long)((a & 0x000FFFFFFFFFFFFFull) | (1023ull << 52))); // [1, 2)
    const double sw = __longlong_as_double((long long)((b & 0x000FFFFFFFFFFFFFull) | (1023ull << 52)));
    const int ex = (int)((a >> 52) % 81) - 40;
    double x = ldexp(sx, ex), w = ldexp(sw, (int)((b >> 52) % 25) - 20);
    if ((b >> 60) & 1) {
      x = 10.0 / (double)(1 + ((a >> 20) % 65536));
      w = 10.0 / (double)(1 + ((b >> 20) % 65536));
    }
    const double r = 1.0 / w;
    const double q = cb::width_ratio(x, w, r), ref = x / w;
    if (__double_as_longlong(q) != __double_as_longlong(ref)) {
      ++local;
      example[0] = x;
      example[1] = w;
    }
  }
  if (local) atomicAdd(bad, local);
}

// A staging wait on a barrier that needs two arrivals and gets one: no copy
// is in flight, nothing will complete the phase, and mbar_wait gives up
// after limit_ns with the error flag set.
__global__ void k_stage_wait_limit(unsigned long long limit_ns, int *err, unsigned long long *elapsed, int *returned) {
  __shared__ uint64_t bar;
  if (threadIdx.x != 0) return;
  cb::mbar_init(&bar, 2);
  asm volatile("{\n .reg .b64 st;\n mbarrier.arrive.shared::cta.b64 st, [%0];\n}\n" ::"r"(cb::smem_addr(&bar)) : "memory");
  const unsigned long long t0 = cb::global_ns();
  const bool ok = cb::mbar_wait(&bar, 0, err, limit_ns);
  elapsed[0] = cb::global_ns() - t0;
  returned[0] = ok ? 1 : 0;
}

// A lane of two CTAs whose second CTA exits without arriving: the first
// gives up after limit_ns, sets the abort flag and returns false.
__global__ void k_lane_wait_limit(unsigned *ctr, int *abort, unsigned long long limit_ns, unsigned long long *elapsed, int *returned) {
  if (blockIdx.x == 1) return;
  const unsigned long long t0 = cb::global_ns();
  const bool ok = cb::lane_sync(ctr, 2, abort, limit_ns);
  if (threadIdx.x == 0) {
    elapsed[1] = cb::global_ns() - t0;
    returned[1] = ok ? 1 : 0;
  }
}

} // namespace

extern "C" int cb_selftest_wait_limits(double limit_ms, int *stage_flag, int *stage_returned, double *stage_ms, int *lane_abort,
                                       int *lane_returned, double *lane_ms) {
  if (!(limit_ms > 0.0 && limit_ms <= 1000.0) || !stage_flag || !stage_returned || !stage_ms || !lane_abort || !lane_returned || !lane_ms)
    return cb::set_last_error(CB_EINVAL, "cb_selftest_wait_limits: bad argument (limit_ms in (0, 1000])");
  const unsigned long long limit_ns = (unsigned long long)(limit_ms * 1e6);
  // words: [0] staging error flag, [1] lane counter, [2] abort flag, [3..4] returned flags; then two elapsed times
  int *d_w = nullptr;
  unsigned long long *d_t = nullptr;
  cudaError_t e = cudaMalloc(&d_w, 8 * sizeof(int));
  if (e == cudaSuccess) e = cudaMalloc(&d_t, 2 * sizeof(unsigned long long));
  if (e == cudaSuccess) e = cudaMemset(d_w, 0, 8 * sizeof(int));
  if (e == cudaSuccess) e = cudaMemset(d_t, 0, 2 * sizeof(unsigned long long));
  if (e == cudaSuccess) {
    k_stage_wait_limit<<<1, 32>>>(limit_ns, d_w, d_t, d_w + 3);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) {
    k_lane_wait_limit<<<2, 64>>>(reinterpret_cast<unsigned *>(d_w + 1), d_w + 2, limit_ns, d_t, d_w + 3);
    e = cudaGetLastError();
  }
  int w[8] = {0};
  unsigned long long t[2] = {0, 0};
  if (e == cudaSuccess) e = cudaMemcpy(w, d_w, sizeof(w), cudaMemcpyDeviceToHost);
  if (e == cudaSuccess) e = cudaMemcpy(t, d_t, sizeof(t), cudaMemcpyDeviceToHost);
  cudaFree(d_w);
  cudaFree(d_t);
  if (e != cudaSuccess) return cb::set_last_error(CB_ECUDA, std::string("cb_selftest_wait_limits: ") + cudaGetErrorString(e));
  *stage_flag = w[0];
  *stage_returned = w[3];
  *stage_ms = (double)t[0] / 1e6;
  *lane_abort = w[2];
  *lane_returned = w[4];
  *lane_ms = (double)t[1] / 1e6;
  return CB_OK;
}

extern "C" int cb_selftest_width_ratio(long long samples, unsigned long long seed, long long *mismatches) {
  if (samples < 0 || !mismatches) return cb::set_last_error(CB_EINVAL, "cb_selftest_width_ratio: bad argument");
  unsigned long long *d_bad = nullptr;
  double *d_ex = nullptr;
  cudaError_t e = cudaMalloc(&d_bad, sizeof(unsigned long long));
  if (e == cudaSuccess) e = cudaMalloc(&d_ex, 2 * sizeof(double));
  if (e == cudaSuccess) e = cudaMemset(d_bad, 0, sizeof(unsigned long long));
  if (e == cudaSuccess) {
    k_width_ratio<<<1184, 256>>>((unsigned long long)samples, seed, d_bad, d_ex);
    e = cudaGetLastError();
  }
  unsigned long long bad = 0;
  if (e == cudaSuccess) e = cudaMemcpy(&bad, d_bad, sizeof(bad), cudaMemcpyDeviceToHost);
  cudaFree(d_bad);
  cudaFree(d_ex);
  if (e != cudaSuccess) return cb::set_last_error(CB_ECUDA, std::string("cb_selftest_width_ratio: ") + cudaGetErrorString(e));
  *mismatches = (long long)bad;
  return CB_OK;
}
