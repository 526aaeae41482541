// cb_selftest.cu -- cb_selftest_width_ratio: checks width_ratio (cb_mesh.cuh),
// the FP64 kernels' quotient of two mesh widths with a precomputed
// reciprocal, against the division operator on the device, bit for bit.
#include <cuda_runtime.h>

#include <string>

#include "../../include/cloverb200.h"
#include "cb_mesh.cuh"

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

} // namespace

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
