// cb_dual.cuh -- forward-mode dual numbers for the tangent-linear run and the
// local Jacobians of the adjoint kernels.
//
// Dual<N> carries a value and N tangent components.  Every operation forms
// the value exactly as the double operation does (same operation, same
// rounding), so a phase function evaluated on Dual<N> returns bit for bit
// the value the FP64 kernels compute, plus the derivatives of that value
// with respect to whatever the N components were seeded with.  At the
// non-smooth points of the hydro scheme (|x| at 0, min/max ties, branches)
// the derivative of the branch the value takes is used; d|x| at x = 0 is 0,
// the central difference's value there.
#pragma once

#include <cuda_runtime.h>

namespace cb {

// The double overloads stay visible next to the Dual ones declared below.
using ::fabs;
using ::fmax;
using ::fmin;
using ::sqrt;

template <int N> struct Dual {
  double v;
  double d[N];
  __host__ __device__ Dual() : v(0.0) {
    for (int k = 0; k < N; ++k) d[k] = 0.0;
  }
  __host__ __device__ Dual(double x) : v(x) {
    for (int k = 0; k < N; ++k) d[k] = 0.0;
  }
  // the variable x seeded on component k
  __host__ __device__ static Dual var(double x, int k) {
    Dual r(x);
    if (k >= 0 && k < N) r.d[k] = 1.0;
    return r;
  }
};

template <int N> __host__ __device__ inline Dual<N> operator+(const Dual<N> &a, const Dual<N> &b) {
  Dual<N> r;
  r.v = a.v + b.v;
  for (int k = 0; k < N; ++k) r.d[k] = a.d[k] + b.d[k];
  return r;
}
template <int N> __host__ __device__ inline Dual<N> operator-(const Dual<N> &a, const Dual<N> &b) {
  Dual<N> r;
  r.v = a.v - b.v;
  for (int k = 0; k < N; ++k) r.d[k] = a.d[k] - b.d[k];
  return r;
}
template <int N> __host__ __device__ inline Dual<N> operator-(const Dual<N> &a) {
  Dual<N> r;
  r.v = -a.v;
  for (int k = 0; k < N; ++k) r.d[k] = -a.d[k];
  return r;
}
template <int N> __host__ __device__ inline Dual<N> operator*(const Dual<N> &a, const Dual<N> &b) {
  Dual<N> r;
  r.v = a.v * b.v;
  for (int k = 0; k < N; ++k) r.d[k] = a.d[k] * b.v + a.v * b.d[k];
  return r;
}
template <int N> __host__ __device__ inline Dual<N> operator/(const Dual<N> &a, const Dual<N> &b) {
  Dual<N> r;
  r.v = a.v / b.v;
  const double inv = 1.0 / b.v;
  for (int k = 0; k < N; ++k) r.d[k] = (a.d[k] - r.v * b.d[k]) * inv;
  return r;
}
template <int N> __host__ __device__ inline Dual<N> operator+(const Dual<N> &a, double b) { return a + Dual<N>(b); }
template <int N> __host__ __device__ inline Dual<N> operator+(double a, const Dual<N> &b) { return Dual<N>(a) + b; }
template <int N> __host__ __device__ inline Dual<N> operator-(const Dual<N> &a, double b) { return a - Dual<N>(b); }
template <int N> __host__ __device__ inline Dual<N> operator-(double a, const Dual<N> &b) { return Dual<N>(a) - b; }
template <int N> __host__ __device__ inline Dual<N> operator*(const Dual<N> &a, double b) { return a * Dual<N>(b); }
template <int N> __host__ __device__ inline Dual<N> operator*(double a, const Dual<N> &b) { return Dual<N>(a) * b; }
template <int N> __host__ __device__ inline Dual<N> operator/(const Dual<N> &a, double b) { return a / Dual<N>(b); }
template <int N> __host__ __device__ inline Dual<N> operator/(double a, const Dual<N> &b) { return Dual<N>(a) / b; }

template <int N> __host__ __device__ inline bool operator<(const Dual<N> &a, const Dual<N> &b) { return a.v < b.v; }
template <int N> __host__ __device__ inline bool operator>(const Dual<N> &a, const Dual<N> &b) { return a.v > b.v; }
template <int N> __host__ __device__ inline bool operator<=(const Dual<N> &a, const Dual<N> &b) { return a.v <= b.v; }
template <int N> __host__ __device__ inline bool operator>=(const Dual<N> &a, const Dual<N> &b) { return a.v >= b.v; }

template <int N> __host__ __device__ inline Dual<N> fabs(const Dual<N> &a) {
  if (a.v > 0.0) return a;
  if (a.v < 0.0) return -a;
  Dual<N> r(0.0 * a.v); // keeps the sign of a zero as fabs does
  r.v = ::fabs(a.v);
  return r;
}
template <int N> __host__ __device__ inline Dual<N> fmin(const Dual<N> &a, const Dual<N> &b) {
  Dual<N> r = (b.v < a.v) ? b : a;
  r.v = ::fmin(a.v, b.v);
  return r;
}
template <int N> __host__ __device__ inline Dual<N> fmax(const Dual<N> &a, const Dual<N> &b) {
  Dual<N> r = (b.v > a.v) ? b : a;
  r.v = ::fmax(a.v, b.v);
  return r;
}
template <int N> __host__ __device__ inline Dual<N> sqrt(const Dual<N> &a) {
  Dual<N> r;
  r.v = ::sqrt(a.v);
  const double s = r.v > 0.0 ? 0.5 / r.v : 0.0;
  for (int k = 0; k < N; ++k) r.d[k] = a.d[k] * s;
  return r;
}

// Value and derivative access that also works on plain doubles.
__host__ __device__ inline double val(double x) { return x; }
template <int N> __host__ __device__ inline double val(const Dual<N> &x) { return x.v; }

} // namespace cb
