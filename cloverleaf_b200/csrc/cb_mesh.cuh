// cb_mesh.cuh -- device-side layout of one mesh chunk and the reflective
// halo rules, shared by every kernel of the library.
//
// Index convention (same as the reference's serial/CUDA models): interior
// cell (j, k) of the Fortran original is (i, j) = (j + 1, k + 1); x_min =
// y_min = 1, x_max = nx, y_max = ny; every 2-D array carries a 2-deep halo.
// Every 2-D field is stored x-fastest with a common row pitch, padded so
// that the first interior column (i = 2) of every row starts on a 256-byte
// boundary: element (i, j) lives at base[j * pitch + i].
#pragma once

#include <type_traits>

#include <cstdint>
#include <cuda_runtime.h>

namespace cb {

// Field ids 0..14 are driver/definitions.h:61-77 (field_parameter); 15..21
// are work_array1..7 and 22..24 the 2-D geometry arrays.
enum Field : int {
  DENSITY0 = 0, DENSITY1 = 1, ENERGY0 = 2, ENERGY1 = 3, PRESSURE = 4, VISCOSITY = 5, SOUNDSPEED = 6,
  XVEL0 = 7, XVEL1 = 8, YVEL0 = 9, YVEL1 = 10, VOL_FLUX_X = 11, VOL_FLUX_Y = 12, MASS_FLUX_X = 13,
  MASS_FLUX_Y = 14, WORK1 = 15, WORK7 = 21, VOLUME = 22, XAREA = 23, YAREA = 24, NUM_FIELDS = 25
};

enum Geom : int { CELLX = 0, CELLY, CELLDX, CELLDY, VERTEXX, VERTEXY, VERTEXDX, VERTEXDY, NUM_GEOM };

constexpr double g_small = 1.0e-16; // driver/definitions.h:34
constexpr double g_big = 1.0e+21;   // driver/definitions.h:35

// Array classes of driver/definitions.cpp:4-41.
enum Kind : int { CELL = 0, VERTEX = 1, XFACE = 2, YFACE = 3 };

__host__ __device__ constexpr Kind kind_of(int f) {
  return (f == XVEL0 || f == XVEL1 || f == YVEL0 || f == YVEL1 || (f >= WORK1 && f <= WORK7)) ? VERTEX
         : (f == VOL_FLUX_X || f == MASS_FLUX_X || f == XAREA)                                 ? XFACE
         : (f == VOL_FLUX_Y || f == MASS_FLUX_Y || f == YAREA)                                 ? YFACE
                                                                                                : CELL;
}

// The reflective fill of src/serial/update_halo.cpp:33-684 for one field,
// written as "destination index <- source index" per face:
//   bottom (i, 1-k)         <- sign_bt * (i, bot_src + k)
//   top    (i, ny+top_dst+k) <- sign_bt * (i, ny+top_src-k)
//   left   (1-k, j)         <- sign_lr * (left_src + k, j)
//   right  (nx+right_dst+k, j) <- sign_lr * (nx+right_src-k, j)
// Bottom/top run over columns [2-d, nx+2+xe+d), left/right over rows
// [2-d, ny+2+ye+d), in that order.  The face-array rows/columns that look
// shifted by one (x faces top_src = 0, y faces right_src = 0) are the
// reference's own and are kept.
struct HaloRule {
  int xe, ye;
  int bot_src, top_dst, top_src, left_src, right_dst, right_src;
  double sign_bt, sign_lr;
  bool soundspeed_bottom_quirk; // src/serial/update_halo.cpp:273 reads row k
};

__host__ __device__ inline HaloRule halo_rule(int f) {
  HaloRule r{};
  switch (kind_of(f)) {
    case VERTEX:
      r = {1, 1, 3, 3, 1, 3, 3, 1, 1.0, 1.0, false};
      if (f == XVEL0 || f == XVEL1) r.sign_lr = -1.0;
      if (f == YVEL0 || f == YVEL1) r.sign_bt = -1.0;
      break;
    case XFACE: r = {1, 0, 3, 2, 0, 3, 3, 1, 1.0, -1.0, false}; break;
    case YFACE: r = {0, 1, 3, 3, 1, 3, 2, 0, -1.0, 1.0, false}; break;
    default: r = {0, 0, 2, 2, 1, 2, 2, 1, 1.0, 1.0, f == SOUNDSPEED}; break;
  }
  return r;
}

// Quotient for terms that every step recomputes from the state (flux
// limiters, the artificial viscosity, CFL bounds, the sound speed): the
// exact IEEE quotient in FP64; in the FP32 form the approximate hardware
// quotient (within 2 ulp), whose error does not build up from step to step.
// The conservative updates (PdV, accelerate, the advection updates) always
// use the exact operator.
template <typename T> __device__ __forceinline__ T lim_div(T a, T b) { return a / b; }
template <> __device__ __forceinline__ float lim_div<float>(float a, float b) { return __fdividef(a, b); }

// a / b where a is often exactly zero (the fluxes of faces and nodes the
// flow has not reached): for a zero and b positive the quotient is a itself,
// its sign included.  When that holds on every active lane of the warp the
// division is skipped (a branch the warp takes together); otherwise each
// lane takes a or the division operator's quotient, the same bits.  For
// arithmetic types only: the tangent-linear number types divide with their
// own operator.
template <typename T> __device__ __forceinline__ T div_zero_num(T a, T b) {
  if constexpr (std::is_floating_point<T>::value) {
    const bool zero = a == T(0.0) && b > T(0.0);
    if (__all_sync(__activemask(), zero)) return a; // a branch the warp takes together
    return zero ? a : a / b;
  }
  return a / b;
}

// x / w for positive mesh widths x and w, given r = 1 / w rounded to nearest
// (computed on the host), by correction steps q <- RN(q + (x - q w) r) with
// the remainder formed exactly by a fused multiply-add.  q0 = RN(x r) lies
// within 1.5 ulp of x / w; one step brings it within an ulp; then
// Markstein's theorem (P. W. Markstein, "Computation of elementary functions
// on the IBM RISC System/6000 processor", IBM J. Res. Develop. 34(1), 1990:
// with r within half an ulp of 1 / w and q within an ulp of x / w,
// RN(q + (x - q w) r) = RN(x / w)) makes the second step the correctly
// rounded quotient, the value of x / w.  Valid for normal operands whose
// quotient and remainders stay normal, as ratios of mesh widths do.
__device__ __forceinline__ double width_ratio(double x, double w, double r) {
  double q = x * r;
  q = fma(fma(-q, w, x), r, q);
  return fma(fma(-q, w, x), r, q);
}

template <typename T> struct Mesh {
  int nx, ny;
  long long pitch;           // elements per row
  const double *celldx, *celldy, *vertexdx, *vertexdy; // 1-D geometry (FP64 always)
  const T *celldx_t, *celldy_t;                        // the same widths in the storage type
  const double *rcelldx, *rcelldy, *rvertexdx, *rvertexdy; // their reciprocals, rounded to nearest

  __device__ __forceinline__ long long at(int i, int j) const { return (long long)j * pitch + i; }
};

// Mirror positions of an interior source index s along one axis for a fold
// of depth d: writes up to 2 halo indices into out[] and returns how many.
// lo = left/bottom rule (1 - k <- src0 + k), hi = right/top rule
// (n + dst + k <- n + src - k).
__device__ __forceinline__ int mirrors(int s, int n, int d, int src0, int hdst, int hsrc, int out[2]) {
  int m = 0;
  int k = s - src0;
  if (k >= 0 && k < d) out[m++] = 1 - k;
  k = (n + hsrc) - s;
  if (k >= 0 && k < d) out[m++] = n + hdst + k;
  return m;
}

// Writes value v of interior element (i, j) of field `a` into every halo
// element that update_halo(depth d) would fill from it (corners included).
// Valid when the mesh is large enough that every source lies inside the
// interior (the library only folds when nx, ny >= 8).
template <typename T>
__device__ __forceinline__ void fold_halo(T *a, const Mesh<T> &m, const HaloRule &r, int d, int i, int j, T v) {
  int xm[2], ym[2];
  int nxm = mirrors(i, m.nx, d, r.left_src, r.right_dst, r.right_src, xm);
  int nym = mirrors(j, m.ny, d, r.bot_src, r.top_dst, r.top_src, ym);
  for (int a1 = 0; a1 < nxm; ++a1) a[m.at(xm[a1], j)] = (T)(r.sign_lr * (double)v);
  for (int b1 = 0; b1 < nym; ++b1) {
    a[m.at(i, ym[b1])] = (T)(r.sign_bt * (double)v);
    for (int a1 = 0; a1 < nxm; ++a1) a[m.at(xm[a1], ym[b1])] = (T)(r.sign_lr * (r.sign_bt * (double)v));
  }
}

} // namespace cb
