// cb_adj.cuh -- tangent-linear and adjoint kernels of the hydro step (FP64).
//
// The step is differentiated with the dt sequence held fixed, as a map of
// the level-0 state (density0, energy0, xvel0, yvel0) and gamma; the other
// fields are recomputed inside every step, and calc_dt is not part of the
// map.  Every phase has
//  * tangent-linear kernels: the phase's arithmetic on Dual<1> numbers (value
//    and one tangent), through the same value functions the FP64 tile
//    kernels use, so the values are bit-identical to the plain path's.  The
//    same kernels instantiated on double compute the primal work arrays the
//    adjoint kernels read.
//  * adjoint kernels: one thread per output element re-evaluates the
//    element's function on Dual<N> numbers seeded on its N inputs (its local
//    Jacobian row), multiplies by the output's adjoint and adds the products
//    into the inputs' adjoints (atomically where neighbouring outputs share
//    an input).
// Halos: a producer's fold (the reflective update_halo) is a linear copy
// with signs; its tangent is the same copy, its adjoint moves each halo
// element's adjoint back onto the interior element it was copied from
// (k_adj_unfold, the two passes of update_halo in reverse order).
//
// Index ranges follow the FP64 tile kernels (cb_tile.cuh), which follow
// src/serial/*.cpp; element (i, j) of a slab is at base[j * pitch + i].
#pragma once

#include "cb_dual.cuh"
#include "cb_phase.cuh"
#include "cb_tile.cuh"

namespace cb {
namespace adj {

using D1 = Dual<1>;

struct Grid {
  int nx, ny, pitch;
  const double *cdx, *cdy, *vdx, *vdy; // celldx, celldy, vertexdx, vertexdy
  __device__ __forceinline__ int at(int i, int j) const { return j * pitch + i; }
};

// A field slab pair: values and tangents (tangents unused for S = double).
struct VD {
  double *v, *d;
};

template <typename S> struct IO;
template <> struct IO<double> {
  __device__ static double ld(const VD &a, int g) { return a.v[g]; }
  __device__ static void st(const VD &a, int g, double x) { a.v[g] = x; }
};
template <> struct IO<D1> {
  __device__ static D1 ld(const VD &a, int g) {
    D1 r(a.v[g]);
    r.d[0] = a.d[g];
    return r;
  }
  __device__ static void st(const VD &a, int g, const D1 &x) {
    a.v[g] = x.v;
    a.d[g] = x.d[0];
  }
};

// 2-D launch over [i0, i0 + w) x [j0, j0 + h).
#define ADJ_IJ(i0, j0, w, h)                                                                                                                 \
  const int i = (i0) + (int)(blockIdx.x * blockDim.x + threadIdx.x);                                                                       \
  const int j = (j0) + (int)(blockIdx.y * blockDim.y + threadIdx.y);                                                                       \
  if (i >= (i0) + (w) || j >= (j0) + (h)) return;

__device__ __forceinline__ void aadd(double *p, double v) {
  if (v != 0.0) atomicAdd(p, v);
}

// ===========================================================================
// Tangent-linear / primal kernels (S = D1 or double)
// ===========================================================================

// ideal_gas pressure p = gm1 * rho * e (src/serial/ideal_gas.cpp:40-45) on interior cells.
template <typename S> __global__ void k_tl_ideal_gas(Grid g, VD rho, VD e, VD p, double gm1, double gm1_dot) {
  ADJ_IJ(2, 2, g.nx, g.ny);
  S gm(gm1);
  if constexpr (sizeof(S) != sizeof(double)) gm.d[0] = gm1_dot;
  const int c = g.at(i, j);
  const S pr = gm * IO<S>::ld(rho, c) * IO<S>::ld(e, c);
  IO<S>::st(p, c, pr);
}

// viscosity (src/serial/viscosity.cpp:30-68) on interior cells.
template <typename S> __global__ void k_tl_viscosity(Grid g, VD u, VD v, VD p, VD rho, VD q) {
  ADJ_IJ(2, 2, g.nx, g.ny);
  auto L = [&](const VD &a, int ii, int jj) { return IO<S>::ld(a, g.at(ii, jj)); };
  const S r = viscosity_value<S>(L(u, i, j), L(u, i + 1, j), L(u, i, j + 1), L(u, i + 1, j + 1), L(v, i, j), L(v, i + 1, j), L(v, i, j + 1),
                                 L(v, i + 1, j + 1), L(p, i - 1, j), L(p, i + 1, j), L(p, i, j - 1), L(p, i, j + 1), L(rho, i, j), S(g.cdx[i]),
                                 S(g.cdx[i + 1]), S(g.cdy[j]), S(g.cdy[j + 2]));
  IO<S>::st(q, g.at(i, j), r);
}

// PdV (src/serial/PdV.cpp:36-87) on interior cells.  predict: the
// predictor, whose ideal_gas pressure goes to p_out (and density1, energy1
// take the reverted level-0 values); else the corrector into d1, e1.
template <typename S>
__global__ void k_tl_pdv(Grid g, int predict, double dt, VD u0, VD v0, VD u1, VD v1, VD rho0, VD e0, VD p, VD q, VD d1, VD e1, VD p_out,
                         double gm1, double gm1_dot) {
  ADJ_IJ(2, 2, g.nx, g.ny);
  auto L = [&](const VD &a, int ii, int jj) { return IO<S>::ld(a, g.at(ii, jj)); };
  const S cdx(g.cdx[i]), cdy(g.cdy[j]);
  const S vol = cdx * cdy;
  S w00(0.0), w01(0.0), w10(0.0), w11(0.0), z00(0.0), z10(0.0), z01(0.0), z11(0.0);
  if (!predict) {
    w00 = L(u1, i, j), w01 = L(u1, i, j + 1), w10 = L(u1, i + 1, j), w11 = L(u1, i + 1, j + 1);
    z00 = L(v1, i, j), z10 = L(v1, i + 1, j), z01 = L(v1, i, j + 1), z11 = L(v1, i + 1, j + 1);
  }
  const S r0 = L(rho0, i, j), en0 = L(e0, i, j);
  S dn, en;
  pdv_value<S>(predict != 0, S(dt), cdy, cdx, vol, L(u0, i, j), L(u0, i, j + 1), L(u0, i + 1, j), L(u0, i + 1, j + 1), L(v0, i, j),
               L(v0, i + 1, j), L(v0, i, j + 1), L(v0, i + 1, j + 1), w00, w01, w10, w11, z00, z10, z01, z11, r0, en0, L(p, i, j),
               L(q, i, j), dn, en);
  const int c = g.at(i, j);
  if (predict) {
    S gm(gm1);
    if constexpr (sizeof(S) != sizeof(double)) gm.d[0] = gm1_dot;
    IO<S>::st(p_out, c, gm * dn * en);
    IO<S>::st(d1, c, r0);
    IO<S>::st(e1, c, en0);
  } else {
    IO<S>::st(d1, c, dn);
    IO<S>::st(e1, c, en);
  }
}

// accelerate (src/serial/accelerate.cpp:28-56) on nodes [2, nx+2] x [2, ny+2].
template <typename S> __global__ void k_tl_accelerate(Grid g, double dt, VD rho0, VD p, VD q, VD u0, VD v0, VD u1, VD v1) {
  ADJ_IJ(2, 2, g.nx + 1, g.ny + 1);
  auto L = [&](const VD &a, int ii, int jj) { return IO<S>::ld(a, g.at(ii, jj)); };
  const double cdx = g.cdx[i], cdxm = g.cdx[i - 1], cdy = g.cdy[j], cdym = g.cdy[j - 1];
  S u, v;
  accel_value<S>(S(0.5 * dt), S(cdxm * cdym), S(cdxm * cdy), S(cdx * cdy), S(cdx * cdym), S(cdy), S(cdym), S(cdx), S(cdxm), L(rho0, i - 1, j - 1),
                 L(rho0, i - 1, j), L(rho0, i, j), L(rho0, i, j - 1), L(p, i, j), L(p, i - 1, j), L(p, i, j - 1), L(p, i - 1, j - 1), L(q, i, j),
                 L(q, i - 1, j), L(q, i, j - 1), L(q, i - 1, j - 1), L(u0, i, j), L(v0, i, j), u, v);
  IO<S>::st(u1, g.at(i, j), u);
  IO<S>::st(v1, g.at(i, j), v);
}

// flux_calc (src/serial/flux_calc.cpp:27-43): x faces [2, nx+2] x [2, ny+1],
// y faces [2, nx+1] x [2, ny+2].
template <typename S> __global__ void k_tl_flux(Grid g, double dt, VD u0, VD v0, VD u1, VD v1, VD fx, VD fy) {
  ADJ_IJ(2, 2, g.nx + 1, g.ny + 1);
  auto L = [&](const VD &a, int ii, int jj) { return IO<S>::ld(a, g.at(ii, jj)); };
  if (j <= g.ny + 1) IO<S>::st(fx, g.at(i, j), flux_value<S>(S(dt), S(g.cdy[j]), L(u0, i, j), L(u0, i, j + 1), L(u1, i, j), L(u1, i, j + 1)));
  if (i <= g.nx + 1) IO<S>::st(fy, g.at(i, j), flux_value<S>(S(dt), S(g.cdx[i]), L(v0, i, j), L(v0, i + 1, j), L(v1, i, j), L(v1, i + 1, j)));
}

// Coordinates along (a) and across (l) a sweep of direction dir.
__device__ __forceinline__ int ci(int dir, int a, int l) { return dir == 1 ? a : l; }
__device__ __forceinline__ int cj(int dir, int a, int l) { return dir == 1 ? l : a; }

// advec_cell (src/serial/advec_cell.cpp:28-220), one sweep in three kernels.
// (1) pre_vol of cells a in [1, na+2] on lines [2, nl+1].
template <typename S> __global__ void k_tl_cell_pv(Grid g, int dir, int sweep, VD fx, VD fy, VD pv) {
  const int na = dir == 1 ? g.nx : g.ny, nl = dir == 1 ? g.ny : g.nx;
  ADJ_IJ(1, 2, na + 2, nl);
  const int a = i, l = j, x = ci(dir, a, l), y = cj(dir, a, l);
  auto L = [&](const VD &f, int ii, int jj) { return IO<S>::ld(f, g.at(ii, jj)); };
  const S vol = S(g.cdx[x] * g.cdy[y]);
  S r;
  if (dir == 1)
    r = sweep == 1 ? cell_pre_vol1<S>(vol, L(fx, x, y), L(fx, x + 1, y), L(fy, x, y), L(fy, x, y + 1)) : cell_pre_vol2<S>(vol, L(fx, x, y), L(fx, x + 1, y));
  else
    r = sweep == 1 ? cell_pre_vol1<S>(vol, L(fy, x, y), L(fy, x, y + 1), L(fx, x, y), L(fx, x + 1, y)) : cell_pre_vol2<S>(vol, L(fy, x, y), L(fy, x, y + 1));
  IO<S>::st(pv, g.at(x, y), r);
}

// The donor, upwind, downwind cells and the limiter's dif cell of face f
// (:70-80 / :162-172).
__device__ __forceinline__ void cell_stencil(bool pos, int f, int na, int &donor, int &upwind, int &downwind, int &dif) {
  if (pos) {
    upwind = f - 2; donor = f - 1; downwind = f; dif = donor;
  } else {
    upwind = (f + 1 < na + 2) ? f + 1 : na + 2;
    donor = f; downwind = f - 1; dif = upwind;
  }
}

// (2) mass and energy fluxes of faces f in [2, na+2] on lines [2, nl+1].
template <typename S> __global__ void k_tl_cell_face(Grid g, int dir, VD vf, VD pv, VD rho, VD e, VD mf, VD ef) {
  const int na = dir == 1 ? g.nx : g.ny, nl = dir == 1 ? g.ny : g.nx;
  ADJ_IJ(2, 2, na + 1, nl);
  const int f = i, l = j;
  auto A = [&](const VD &a, int pos) { return IO<S>::ld(a, g.at(ci(dir, pos, l), cj(dir, pos, l))); };
  const S flux = A(vf, f);
  int donor, upwind, downwind, dif;
  cell_stencil(flux > S(0.0), f, na, donor, upwind, downwind, dif);
  const double *vd = dir == 1 ? g.vdx : g.vdy;
  S mflux, eadv;
  cell_face_value<S>(flux, A(pv, donor), S(vd[f] / vd[dif]), A(rho, donor), A(rho, upwind), A(rho, downwind), A(e, donor), A(e, upwind),
                     A(e, downwind), mflux, eadv);
  const int c = g.at(ci(dir, f, l), cj(dir, f, l));
  IO<S>::st(mf, c, mflux);
  IO<S>::st(ef, c, mflux * eadv);
}

// (3) the update of cells a in [2, na+1] on lines [2, nl+1] into (dn, en).
template <typename S> __global__ void k_tl_cell_update(Grid g, int dir, VD vf, VD pv, VD rho, VD e, VD mf, VD ef, VD dn, VD en) {
  const int na = dir == 1 ? g.nx : g.ny, nl = dir == 1 ? g.ny : g.nx;
  ADJ_IJ(2, 2, na, nl);
  const int a = i, l = j;
  auto A = [&](const VD &f, int pos) { return IO<S>::ld(f, g.at(ci(dir, pos, l), cj(dir, pos, l))); };
  S d, en_;
  cell_update_value<S>(A(rho, a), A(e, a), A(pv, a), A(mf, a), A(mf, a + 1), A(ef, a), A(ef, a + 1), A(vf, a), A(vf, a + 1), d, en_);
  const int c = g.at(ci(dir, a, l), cj(dir, a, l));
  IO<S>::st(dn, c, d);
  IO<S>::st(en, c, en_);
}

// advec_mom (src/serial/advec_mom.cpp:30-225), both velocities, in five kernels.
// (1) node fluxes of positions a in [0, na+3] on lines [2, nl+2].
template <typename S> __global__ void k_tl_mom_nf(Grid g, int dir, VD mf, VD nf) {
  const int na = dir == 1 ? g.nx : g.ny, nl = dir == 1 ? g.ny : g.nx;
  ADJ_IJ(0, 2, na + 4, nl + 1);
  const int a = i, l = j;
  auto M = [&](int pa, int pl) { return IO<S>::ld(mf, g.at(ci(dir, pa, pl), cj(dir, pa, pl))); };
  IO<S>::st(nf, g.at(ci(dir, a, l), cj(dir, a, l)), quarter_sum<S>(M(a, l - 1), M(a, l), M(a + 1, l - 1), M(a + 1, l)));
}

// (2) cell masses density1 * post_vol of cells a in [0, na+3] on lines [1, nl+2].
template <typename S> __global__ void k_tl_mom_cm(Grid g, int dir, int mom_sweep, VD rho, VD fx, VD fy, VD cm) {
  const int na = dir == 1 ? g.nx : g.ny, nl = dir == 1 ? g.ny : g.nx;
  ADJ_IJ(0, 1, na + 4, nl + 2);
  const int x = ci(dir, i, j), y = cj(dir, i, j);
  auto L = [&](const VD &f, int ii, int jj) { return IO<S>::ld(f, g.at(ii, jj)); };
  const S vol = S(g.cdx[x] * g.cdy[y]);
  S pvv = vol;
  if (mom_sweep == 1) pvv = mom_post_vol<S>(1, vol, L(fy, x, y), L(fy, x, y + 1));
  if (mom_sweep == 2) pvv = mom_post_vol<S>(2, vol, L(fx, x, y), L(fx, x + 1, y));
  IO<S>::st(cm, g.at(x, y), L(rho, x, y) * pvv);
}

// (3) node_mass_post and node_mass_pre of positions a in [1, na+3] on lines [2, nl+2].
template <typename S> __global__ void k_tl_mom_nm(Grid g, int dir, VD cm, VD nf, VD post, VD pre) {
  const int na = dir == 1 ? g.nx : g.ny, nl = dir == 1 ? g.ny : g.nx;
  ADJ_IJ(1, 2, na + 3, nl + 1);
  const int a = i, l = j, x = ci(dir, a, l), y = cj(dir, a, l);
  auto L = [&](const VD &f, int ii, int jj) { return IO<S>::ld(f, g.at(ii, jj)); };
  const S np = quarter_sum<S>(L(cm, x, y - 1), L(cm, x, y), L(cm, x - 1, y - 1), L(cm, x - 1, y));
  const int pa = ci(dir, a - 1, l), pb = cj(dir, a - 1, l);
  IO<S>::st(post, g.at(x, y), np);
  IO<S>::st(pre, g.at(x, y), mom_node_mass_pre<S>(np, L(nf, pa, pb), L(nf, x, y)));
}

// Donor, upwind, downwind and dif nodes of a node flux (:110-118 / :182-190).
__device__ __forceinline__ void mom_stencil(bool neg, int a, int &donor, int &upwind, int &downwind, int &dif) {
  if (neg) {
    upwind = a + 2; donor = a + 1; downwind = a; dif = donor;
  } else {
    upwind = a - 1; donor = a; downwind = a + 1; dif = upwind;
  }
}

// (4) momentum fluxes of positions a in [1, na+2] on lines [2, nl+2].
template <typename S> __global__ void k_tl_mom_flux(Grid g, int dir, VD nf, VD pre, VD u, VD v, VD fu, VD fv) {
  const int na = dir == 1 ? g.nx : g.ny, nl = dir == 1 ? g.ny : g.nx;
  ADJ_IJ(1, 2, na + 2, nl + 1);
  const int a = i, l = j;
  auto A = [&](const VD &f, int pos) { return IO<S>::ld(f, g.at(ci(dir, pos, l), cj(dir, pos, l))); };
  const S nfv = A(nf, a);
  int donor, upwind, downwind, dif;
  mom_stencil(nfv < S(0.0), a, donor, upwind, downwind, dif);
  const double *cd = dir == 1 ? g.cdx : g.cdy;
  const S sigma = mom_sigma<S>(nfv, A(pre, donor));
  const int c = g.at(ci(dir, a, l), cj(dir, a, l));
  IO<S>::st(fu, c, mom_flux_value<S>(sigma, nfv, S(cd[a]), S(cd[dif]), A(u, donor), A(u, upwind), A(u, downwind)));
  IO<S>::st(fv, c, mom_flux_value<S>(sigma, nfv, S(cd[a]), S(cd[dif]), A(v, donor), A(v, upwind), A(v, downwind)));
}

// (5) velocities of nodes a in [2, na+2] on lines [2, nl+2].
template <typename S> __global__ void k_tl_mom_update(Grid g, int dir, VD pre, VD post, VD fu, VD fv, VD u, VD v, VD un, VD vn) {
  const int na = dir == 1 ? g.nx : g.ny, nl = dir == 1 ? g.ny : g.nx;
  ADJ_IJ(2, 2, na + 1, nl + 1);
  const int a = i, l = j;
  auto A = [&](const VD &f, int pos) { return IO<S>::ld(f, g.at(ci(dir, pos, l), cj(dir, pos, l))); };
  const S npre = A(pre, a), npost = A(post, a);
  const int c = g.at(ci(dir, a, l), cj(dir, a, l));
  IO<S>::st(un, c, mom_update_value<S>(A(u, a), npre, npost, A(fu, a - 1), A(fu, a)));
  IO<S>::st(vn, c, mom_update_value<S>(A(v, a), npre, npost, A(fv, a - 1), A(fv, a)));
}

// Copies src to dst over [i0, i0+w) x [j0, j0+h) (reset_field's interior copies, ring copies).
template <typename S> __global__ void k_tl_copy(Grid g, VD src, VD dst, int i0, int j0, int w, int h) {
  ADJ_IJ(i0, j0, w, h);
  const int c = g.at(i, j);
  IO<S>::st(dst, c, IO<S>::ld(src, c));
}

// Elements of the (ex x ey) extent outside [lo, hi] x [lo, hiy]: src to dst.
template <typename S> __global__ void k_tl_ring(Grid g, VD src, VD dst, int ex, int ey, int lo, int hix, int hiy) {
  ADJ_IJ(0, 0, ex, ey);
  if (i >= lo && i <= hix && j >= lo && j <= hiy) return;
  const int c = g.at(i, j);
  IO<S>::st(dst, c, IO<S>::ld(src, c));
}

// The update_halo fill of one field on values and tangents (two passes).
__global__ void k_tl_halo(Grid g, VD a, int field, int depth, int pass) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  Mesh<double> m{};
  m.nx = g.nx;
  m.ny = g.ny;
  m.pitch = g.pitch;
  Fields<double> F{};
  F.f[field] = a.v;
  halo_fill(F, m, field, depth, pass, t);
  if (a.d) {
    F.f[field] = a.d;
    halo_fill(F, m, field, depth, pass, t);
  }
}

// Kinetic-energy term of every interior cell (src/serial/field_summary.cpp:
// 60-90): cell_vol * density0 * 0.5 * (the 4-node average of u^2 + v^2),
// written per cell (tangent) for a fixed-order sum.
template <typename S> __device__ __forceinline__ S ke_term(const Grid &g, const S &d0, const S *u, const S *v, int i, int j) {
  S vsqrd(0.0);
  for (int k = 0; k < 4; ++k) vsqrd = vsqrd + S(0.25) * (u[k] * u[k] + v[k] * v[k]);
  const double cell_vol = g.cdx[i] * g.cdy[j];
  const S cell_mass = S(cell_vol) * d0;
  return cell_mass * S(0.5) * vsqrd;
}

__global__ void k_tl_ke(Grid g, VD rho, VD u, VD v, double *term_v, double *term_d) {
  ADJ_IJ(2, 2, g.nx, g.ny);
  D1 uu[4], vv[4];
  int k = 0;
  for (int kv = j; kv <= j + 1; ++kv)
    for (int jv = i; jv <= i + 1; ++jv, ++k) {
      uu[k] = IO<D1>::ld(u, g.at(jv, kv));
      vv[k] = IO<D1>::ld(v, g.at(jv, kv));
    }
  const D1 t = ke_term<D1>(g, IO<D1>::ld(rho, g.at(i, j)), uu, vv, i, j);
  const int c = (j - 2) * g.nx + (i - 2);
  term_v[c] = t.v;
  term_d[c] = t.d[0];
}

// Fixed-order sum of n terms (one block of 256 threads).
__global__ void k_sum_fixed(const double *x, int n, double *out) {
  __shared__ double red[256];
  double s = 0.0;
  for (int k = threadIdx.x; k < n; k += 256) s += x[k];
  red[threadIdx.x] = s;
  __syncthreads();
  for (int h = 128; h > 0; h >>= 1) {
    if ((int)threadIdx.x < h) red[threadIdx.x] += red[threadIdx.x + h];
    __syncthreads();
  }
  if (threadIdx.x == 0) *out = red[0];
}

// ===========================================================================
// Adjoint kernels.  Primal inputs are double slabs (the step's tape and the
// recomputed work arrays); b* are adjoint slabs.
// ===========================================================================

template <int N> using DN = Dual<N>;

// Adjoint of update_halo(depth) on one field: pass 1 (left/right rows) then
// pass 0 (bottom/top columns), the fill's passes in reverse; each halo
// element's adjoint goes to its source with the fill's sign and is cleared.
__global__ void k_adj_unfold(Grid g, double *b, int field, int depth, int pass) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const HaloRule r = halo_rule(field);
  const int d = depth;
  auto A = [&](int ii, int jj) -> double & { return b[g.at(ii, jj)]; };
  if (pass == 0) {
    const int jcol = 2 - d + t;
    if (jcol >= g.nx + r.xe + d + 2) return;
    for (int k = d - 1; k >= 0; --k) {
      double &dst = A(jcol, g.ny + r.top_dst + k);
      A(jcol, g.ny + r.top_src - k) += r.sign_bt * dst;
      dst = 0.0;
    }
    for (int k = d - 1; k >= 0; --k) {
      const int src = r.soundspeed_bottom_quirk ? k : r.bot_src + k;
      double &dst = A(jcol, 1 - k);
      A(jcol, src) += r.sign_bt * dst;
      dst = 0.0;
    }
  } else {
    const int krow = 2 - d + t;
    if (krow >= g.ny + r.ye + d + 2) return;
    for (int k = d - 1; k >= 0; --k) {
      double &dst = A(g.nx + r.right_dst + k, krow);
      A(g.nx + r.right_src - k, krow) += r.sign_lr * dst;
      dst = 0.0;
    }
    for (int k = d - 1; k >= 0; --k) {
      double &dst = A(1 - k, krow);
      A(r.left_src + k, krow) += r.sign_lr * dst;
      dst = 0.0;
    }
  }
}

// Adjoint of the final kinetic energy (the objective): seeds the level-0 adjoints.
__global__ void k_adj_ke(Grid g, const double *rho, const double *u, const double *v, double *brho, double *bu, double *bv) {
  ADJ_IJ(2, 2, g.nx, g.ny);
  using X = DN<9>;
  X uu[4], vv[4];
  int k = 0;
  for (int kv = j; kv <= j + 1; ++kv)
    for (int jv = i; jv <= i + 1; ++jv, ++k) {
      uu[k] = X::var(u[g.at(jv, kv)], 1 + k);
      vv[k] = X::var(v[g.at(jv, kv)], 5 + k);
    }
  const X t = ke_term<X>(g, X::var(rho[g.at(i, j)], 0), uu, vv, i, j);
  brho[g.at(i, j)] += t.d[0];
  k = 0;
  for (int kv = j; kv <= j + 1; ++kv)
    for (int jv = i; jv <= i + 1; ++jv, ++k) {
      aadd(&bu[g.at(jv, kv)], t.d[1 + k]);
      aadd(&bv[g.at(jv, kv)], t.d[5 + k]);
    }
}

// Block-wide sum of v folded into *out with one atomic add (gamma's adjoint).
__device__ __forceinline__ void block_add(double v, double *out) {
  __shared__ double red[256];
  const int tid = threadIdx.y * blockDim.x + threadIdx.x;
  red[tid] = v;
  __syncthreads();
  for (int h = (blockDim.x * blockDim.y) / 2; h > 0; h >>= 1) {
    if (tid < h) red[tid] += red[tid + h];
    __syncthreads();
  }
  if (tid == 0 && red[0] != 0.0) atomicAdd(out, red[0]);
}

// ideal_gas: p = gm1 * rho * e.
__global__ void k_adj_ideal_gas(Grid g, const double *rho, const double *e, const double *bp, double *brho, double *be, double gm1,
                                double *bgamma) {
  const int i = 2 + (int)(blockIdx.x * blockDim.x + threadIdx.x);
  const int j = 2 + (int)(blockIdx.y * blockDim.y + threadIdx.y);
  double gb = 0.0;
  if (i < g.nx + 2 && j < g.ny + 2) {
    const int c = g.at(i, j);
    using X = DN<3>;
    const X p = X::var(gm1, 2) * X::var(rho[c], 0) * X::var(e[c], 1);
    const double pb = bp[c];
    brho[c] += pb * p.d[0];
    be[c] += pb * p.d[1];
    gb = pb * p.d[2];
  }
  block_add(gb, bgamma);
}

// viscosity: q(u 4 nodes, v 4 nodes, p 4 neighbours, rho).
__global__ void k_adj_viscosity(Grid g, const double *u, const double *v, const double *p, const double *rho, const double *bq, double *bu,
                                double *bv, double *bp, double *brho) {
  ADJ_IJ(2, 2, g.nx, g.ny);
  const double qb = bq[g.at(i, j)];
  if (qb == 0.0) return;
  using X = DN<13>;
  const int nu[4][2] = {{i, j}, {i + 1, j}, {i, j + 1}, {i + 1, j + 1}};
  const int np[4][2] = {{i - 1, j}, {i + 1, j}, {i, j - 1}, {i, j + 1}};
  X U[4], V[4], P[4];
  for (int k = 0; k < 4; ++k) {
    U[k] = X::var(u[g.at(nu[k][0], nu[k][1])], k);
    V[k] = X::var(v[g.at(nu[k][0], nu[k][1])], 4 + k);
    P[k] = X::var(p[g.at(np[k][0], np[k][1])], 8 + k);
  }
  const X q = viscosity_value<X>(U[0], U[1], U[2], U[3], V[0], V[1], V[2], V[3], P[0], P[1], P[2], P[3], X::var(rho[g.at(i, j)], 12),
                                 X(g.cdx[i]), X(g.cdx[i + 1]), X(g.cdy[j]), X(g.cdy[j + 2]));
  for (int k = 0; k < 4; ++k) {
    aadd(&bu[g.at(nu[k][0], nu[k][1])], qb * q.d[k]);
    aadd(&bv[g.at(nu[k][0], nu[k][1])], qb * q.d[4 + k]);
    aadd(&bp[g.at(np[k][0], np[k][1])], qb * q.d[8 + k]);
  }
  aadd(&brho[g.at(i, j)], qb * q.d[12]);
}

// PdV.  Inputs (local index): u0 0-3, v0 4-7, [u1 8-11, v1 12-15], rho0,
// e0, p, q, gamma.  Predictor: the output is the ideal-gas pressure of the
// predicted state (adjoint in bp_out); corrector: density1, energy1.
template <int PRED>
__global__ void k_adj_pdv(Grid g, double dt, const double *u0, const double *v0, const double *u1, const double *v1, const double *rho0,
                          const double *e0, const double *p, const double *q, const double *bd1, const double *be1, const double *bp_out,
                          double *bu0, double *bv0, double *bu1, double *bv1, double *brho0, double *be0, double *bp, double *bq, double gm1,
                          double *bgamma) {
  const int i = 2 + (int)(blockIdx.x * blockDim.x + threadIdx.x);
  const int j = 2 + (int)(blockIdx.y * blockDim.y + threadIdx.y);
  double gb = 0.0;
  if (i < g.nx + 2 && j < g.ny + 2) {
    constexpr int NV = PRED ? 8 : 16; // velocity inputs
    constexpr int N = NV + 5;
    using X = DN<N>;
    const int c = g.at(i, j);
    const int nn[4][2] = {{i, j}, {i, j + 1}, {i + 1, j}, {i + 1, j + 1}}; // u00, u01, u10, u11 order of pdv_value's u arguments
    X U0[4], W[4], Z[4], V0[4];
    // pdv_value's v argument order is v00, v10, v01, v11
    const int nv[4][2] = {{i, j}, {i + 1, j}, {i, j + 1}, {i + 1, j + 1}};
    for (int k = 0; k < 4; ++k) {
      U0[k] = X::var(u0[g.at(nn[k][0], nn[k][1])], k);
      V0[k] = X::var(v0[g.at(nv[k][0], nv[k][1])], 4 + k);
      if (!PRED) {
        W[k] = X::var(u1[g.at(nn[k][0], nn[k][1])], 8 + k);
        Z[k] = X::var(v1[g.at(nv[k][0], nv[k][1])], 12 + k);
      } else {
        W[k] = X(0.0);
        Z[k] = X(0.0);
      }
    }
    const X r0 = X::var(rho0[c], NV), en0 = X::var(e0[c], NV + 1), pp = X::var(p[c], NV + 2), qq = X::var(q[c], NV + 3);
    const X cdx(g.cdx[i]), cdy(g.cdy[j]);
    const X vol = cdx * cdy;
    X dn, en;
    pdv_value<X>(PRED != 0, X(dt), cdy, cdx, vol, U0[0], U0[1], U0[2], U0[3], V0[0], V0[1], V0[2], V0[3], W[0], W[1], W[2], W[3], Z[0], Z[1],
                 Z[2], Z[3], r0, en0, pp, qq, dn, en);
    double gr[N];
    if (PRED) {
      const X out = X::var(gm1, NV + 4) * dn * en;
      const double b = bp_out[c];
      for (int k = 0; k < N; ++k) gr[k] = b * out.d[k];
    } else {
      const double b1 = bd1[c], b2 = be1[c];
      for (int k = 0; k < N; ++k) gr[k] = b1 * dn.d[k] + b2 * en.d[k];
    }
    for (int k = 0; k < 4; ++k) {
      aadd(&bu0[g.at(nn[k][0], nn[k][1])], gr[k]);
      aadd(&bv0[g.at(nv[k][0], nv[k][1])], gr[4 + k]);
      if (!PRED) {
        aadd(&bu1[g.at(nn[k][0], nn[k][1])], gr[8 + k]);
        aadd(&bv1[g.at(nv[k][0], nv[k][1])], gr[12 + k]);
      }
    }
    brho0[c] += gr[NV];
    be0[c] += gr[NV + 1];
    bp[c] += gr[NV + 2];
    bq[c] += gr[NV + 3];
    if (PRED) gb = gr[NV + 4];
  }
  block_add(gb, bgamma);
}

// accelerate.  Inputs: rho0, p, q of cells mm, m0, 00, 0m (0-11), u0, v0 (12, 13).
__global__ void k_adj_accelerate(Grid g, double dt, const double *rho0, const double *p, const double *q, const double *u0, const double *v0,
                                 const double *bu1, const double *bv1, double *brho0, double *bp, double *bq, double *bu0, double *bv0) {
  ADJ_IJ(2, 2, g.nx + 1, g.ny + 1);
  const int n = g.at(i, j);
  const double ub = bu1[n], vb = bv1[n];
  if (ub == 0.0 && vb == 0.0) return;
  using X = DN<14>;
  const int cc[4][2] = {{i - 1, j - 1}, {i - 1, j}, {i, j}, {i, j - 1}}; // mm, m0, 00, 0m
  X R[4], P[4], Q[4];
  for (int k = 0; k < 4; ++k) {
    const int c = g.at(cc[k][0], cc[k][1]);
    R[k] = X::var(rho0[c], k);
    P[k] = X::var(p[c], 4 + k);
    Q[k] = X::var(q[c], 8 + k);
  }
  const double cdx = g.cdx[i], cdxm = g.cdx[i - 1], cdy = g.cdy[j], cdym = g.cdy[j - 1];
  X u, v;
  // accel_value's pressure / viscosity order is 00, m0, 0m, mm
  accel_value<X>(X(0.5 * dt), X(cdxm * cdym), X(cdxm * cdy), X(cdx * cdy), X(cdx * cdym), X(cdy), X(cdym), X(cdx), X(cdxm), R[0], R[1], R[2],
                 R[3], P[2], P[1], P[3], P[0], Q[2], Q[1], Q[3], Q[0], X::var(u0[n], 12), X::var(v0[n], 13), u, v);
  for (int k = 0; k < 4; ++k) {
    const int c = g.at(cc[k][0], cc[k][1]);
    aadd(&brho0[c], ub * u.d[k] + vb * v.d[k]);
    aadd(&bp[c], ub * u.d[4 + k] + vb * v.d[4 + k]);
    aadd(&bq[c], ub * u.d[8 + k] + vb * v.d[8 + k]);
  }
  bu0[n] += ub * u.d[12] + vb * v.d[12];
  bv0[n] += ub * u.d[13] + vb * v.d[13];
}

// flux_calc: each face's flux is linear in its four node velocities.
__global__ void k_adj_flux(Grid g, double dt, const double *bfx, const double *bfy, double *bu0, double *bv0, double *bu1, double *bv1) {
  ADJ_IJ(2, 2, g.nx + 1, g.ny + 1);
  using X = DN<4>;
  if (j <= g.ny + 1) {
    const double b = bfx[g.at(i, j)];
    if (b != 0.0) {
      const X f = flux_value<X>(X(dt), X(g.cdy[j]), X::var(0.0, 0), X::var(0.0, 1), X::var(0.0, 2), X::var(0.0, 3));
      aadd(&bu0[g.at(i, j)], b * f.d[0]);
      aadd(&bu0[g.at(i, j + 1)], b * f.d[1]);
      aadd(&bu1[g.at(i, j)], b * f.d[2]);
      aadd(&bu1[g.at(i, j + 1)], b * f.d[3]);
    }
  }
  if (i <= g.nx + 1) {
    const double b = bfy[g.at(i, j)];
    if (b != 0.0) {
      const X f = flux_value<X>(X(dt), X(g.cdx[i]), X::var(0.0, 0), X::var(0.0, 1), X::var(0.0, 2), X::var(0.0, 3));
      aadd(&bv0[g.at(i, j)], b * f.d[0]);
      aadd(&bv0[g.at(i + 1, j)], b * f.d[1]);
      aadd(&bv1[g.at(i, j)], b * f.d[2]);
      aadd(&bv1[g.at(i + 1, j)], b * f.d[3]);
    }
  }
}

// advec_cell update.  Inputs: rho, e, pv, mf_lo, mf_hi, ef_lo, ef_hi, vf_lo, vf_hi.
__global__ void k_adj_cell_update(Grid g, int dir, const double *vf, const double *pv, const double *rho, const double *e, const double *mf,
                                  const double *ef, const double *bdn, const double *ben, double *bvf, double *bpv, double *brho,
                                  double *be, double *bmf, double *bef) {
  const int na = dir == 1 ? g.nx : g.ny, nl = dir == 1 ? g.ny : g.nx;
  ADJ_IJ(2, 2, na, nl);
  const int a = i, l = j;
  auto G = [&](int pos) { return g.at(ci(dir, pos, l), cj(dir, pos, l)); };
  const int c = G(a), c1 = G(a + 1);
  const double db = bdn[c], eb = ben[c];
  if (db == 0.0 && eb == 0.0) return;
  using X = DN<9>;
  X d, en;
  cell_update_value<X>(X::var(rho[c], 0), X::var(e[c], 1), X::var(pv[c], 2), X::var(mf[c], 3), X::var(mf[c1], 4), X::var(ef[c], 5),
                       X::var(ef[c1], 6), X::var(vf[c], 7), X::var(vf[c1], 8), d, en);
  double gr[9];
  for (int k = 0; k < 9; ++k) gr[k] = db * d.d[k] + eb * en.d[k];
  aadd(&brho[c], gr[0]);
  aadd(&be[c], gr[1]);
  aadd(&bpv[c], gr[2]);
  aadd(&bmf[c], gr[3]);
  aadd(&bmf[c1], gr[4]);
  aadd(&bef[c], gr[5]);
  aadd(&bef[c1], gr[6]);
  aadd(&bvf[c], gr[7]);
  aadd(&bvf[c1], gr[8]);
}

// advec_cell face fluxes.  Inputs: flux, pv(donor), rho and e of donor, upwind, downwind.
__global__ void k_adj_cell_face(Grid g, int dir, const double *vf, const double *pv, const double *rho, const double *e, const double *bmf,
                                const double *bef, double *bvf, double *bpv, double *brho, double *be) {
  const int na = dir == 1 ? g.nx : g.ny, nl = dir == 1 ? g.ny : g.nx;
  ADJ_IJ(2, 2, na + 1, nl);
  const int f = i, l = j;
  auto G = [&](int pos) { return g.at(ci(dir, pos, l), cj(dir, pos, l)); };
  const int cf = G(f);
  const double mb = bmf[cf], eb = bef[cf];
  if (mb == 0.0 && eb == 0.0) return;
  using X = DN<8>;
  const X flux = X::var(vf[cf], 0);
  int donor, upwind, downwind, dif;
  cell_stencil(flux > X(0.0), f, na, donor, upwind, downwind, dif);
  const double *vd = dir == 1 ? g.vdx : g.vdy;
  const int cd = G(donor), cu = G(upwind), cw = G(downwind);
  X mflux, eadv;
  cell_face_value<X>(flux, X::var(pv[cd], 1), X(vd[f] / vd[dif]), X::var(rho[cd], 2), X::var(rho[cu], 3), X::var(rho[cw], 4),
                     X::var(e[cd], 5), X::var(e[cu], 6), X::var(e[cw], 7), mflux, eadv);
  const X eflux = mflux * eadv;
  double gr[8];
  for (int k = 0; k < 8; ++k) gr[k] = mb * mflux.d[k] + eb * eflux.d[k];
  aadd(&bvf[cf], gr[0]);
  aadd(&bpv[cd], gr[1]);
  aadd(&brho[cd], gr[2]);
  aadd(&brho[cu], gr[3]);
  aadd(&brho[cw], gr[4]);
  aadd(&be[cd], gr[5]);
  aadd(&be[cu], gr[6]);
  aadd(&be[cw], gr[7]);
}

// advec_cell pre_vol: linear in the flux differences.
__global__ void k_adj_cell_pv(Grid g, int dir, int sweep, const double *bpv, double *bfx, double *bfy) {
  const int na = dir == 1 ? g.nx : g.ny, nl = dir == 1 ? g.ny : g.nx;
  ADJ_IJ(1, 2, na + 2, nl);
  const int x = ci(dir, i, j), y = cj(dir, i, j);
  const double b = bpv[g.at(x, y)];
  if (b == 0.0) return;
  double *ba = dir == 1 ? bfx : bfy, *bb = dir == 1 ? bfy : bfx;
  const int a_lo = g.at(x, y), a_hi = dir == 1 ? g.at(x + 1, y) : g.at(x, y + 1);
  const int b_lo = g.at(x, y), b_hi = dir == 1 ? g.at(x, y + 1) : g.at(x + 1, y);
  using X = DN<4>;
  if (sweep == 1) {
    const X r = cell_pre_vol1<X>(X(0.0), X::var(0.0, 0), X::var(0.0, 1), X::var(0.0, 2), X::var(0.0, 3));
    aadd(&ba[a_lo], b * r.d[0]);
    aadd(&ba[a_hi], b * r.d[1]);
    aadd(&bb[b_lo], b * r.d[2]);
    aadd(&bb[b_hi], b * r.d[3]);
  } else {
    const X r = cell_pre_vol2<X>(X(0.0), X::var(0.0, 0), X::var(0.0, 1));
    aadd(&ba[a_lo], b * r.d[0]);
    aadd(&ba[a_hi], b * r.d[1]);
  }
}

// advec_mom update.  Inputs: u, v, pre, post, fu_lo, fu_hi, fv_lo, fv_hi.
__global__ void k_adj_mom_update(Grid g, int dir, const double *pre, const double *post, const double *fu, const double *fv, const double *u,
                                 const double *v, const double *bun, const double *bvn, double *bu, double *bv, double *bpre, double *bpost,
                                 double *bfu, double *bfv) {
  const int na = dir == 1 ? g.nx : g.ny, nl = dir == 1 ? g.ny : g.nx;
  ADJ_IJ(2, 2, na + 1, nl + 1);
  const int a = i, l = j;
  auto G = [&](int pos) { return g.at(ci(dir, pos, l), cj(dir, pos, l)); };
  const int c = G(a), cl = G(a - 1);
  const double ub = bun[c], vb = bvn[c];
  if (ub == 0.0 && vb == 0.0) return;
  using X = DN<8>;
  const X npre = X::var(pre[c], 2), npost = X::var(post[c], 3);
  const X un = mom_update_value<X>(X::var(u[c], 0), npre, npost, X::var(fu[cl], 4), X::var(fu[c], 5));
  const X vn = mom_update_value<X>(X::var(v[c], 1), npre, npost, X::var(fv[cl], 6), X::var(fv[c], 7));
  aadd(&bu[c], ub * un.d[0]);
  aadd(&bv[c], vb * vn.d[1]);
  aadd(&bpre[c], ub * un.d[2] + vb * vn.d[2]);
  aadd(&bpost[c], ub * un.d[3] + vb * vn.d[3]);
  aadd(&bfu[cl], ub * un.d[4]);
  aadd(&bfu[c], ub * un.d[5]);
  aadd(&bfv[cl], vb * vn.d[6]);
  aadd(&bfv[c], vb * vn.d[7]);
}

// advec_mom momentum fluxes.  Inputs: nf, pre(donor), u and v of donor, upwind, downwind.
__global__ void k_adj_mom_flux(Grid g, int dir, const double *nf, const double *pre, const double *u, const double *v, const double *bfu,
                               const double *bfv, double *bnf, double *bpre, double *bu, double *bv) {
  const int na = dir == 1 ? g.nx : g.ny, nl = dir == 1 ? g.ny : g.nx;
  ADJ_IJ(1, 2, na + 2, nl + 1);
  const int a = i, l = j;
  auto G = [&](int pos) { return g.at(ci(dir, pos, l), cj(dir, pos, l)); };
  const int c = G(a);
  const double ub = bfu[c], vb = bfv[c];
  if (ub == 0.0 && vb == 0.0) return;
  using X = DN<8>;
  const X nfv = X::var(nf[c], 0);
  int donor, upwind, downwind, dif;
  mom_stencil(nfv < X(0.0), a, donor, upwind, downwind, dif);
  const double *cdd = dir == 1 ? g.cdx : g.cdy;
  const int cd = G(donor), cu = G(upwind), cw = G(downwind);
  const X sigma = mom_sigma<X>(nfv, X::var(pre[cd], 1));
  const X fu = mom_flux_value<X>(sigma, nfv, X(cdd[a]), X(cdd[dif]), X::var(u[cd], 2), X::var(u[cu], 3), X::var(u[cw], 4));
  const X fv = mom_flux_value<X>(sigma, nfv, X(cdd[a]), X(cdd[dif]), X::var(v[cd], 5), X::var(v[cu], 6), X::var(v[cw], 7));
  aadd(&bnf[c], ub * fu.d[0] + vb * fv.d[0]);
  aadd(&bpre[cd], ub * fu.d[1] + vb * fv.d[1]);
  aadd(&bu[cd], ub * fu.d[2]);
  aadd(&bu[cu], ub * fu.d[3]);
  aadd(&bu[cw], ub * fu.d[4]);
  aadd(&bv[cd], vb * fv.d[5]);
  aadd(&bv[cu], vb * fv.d[6]);
  aadd(&bv[cw], vb * fv.d[7]);
}

// advec_mom node masses: pre = post - nf(a-1) + nf(a); post = 0.25 * (4 cell masses).
__global__ void k_adj_mom_nm(Grid g, int dir, const double *bpre, double *bpost, double *bnf, double *bcm) {
  const int na = dir == 1 ? g.nx : g.ny, nl = dir == 1 ? g.ny : g.nx;
  ADJ_IJ(1, 2, na + 3, nl + 1);
  const int a = i, l = j, x = ci(dir, a, l), y = cj(dir, a, l);
  const int c = g.at(x, y);
  const double pb = bpre[c];
  using X = DN<4>;
  const X r = mom_node_mass_pre<X>(X::var(0.0, 0), X::var(0.0, 1), X::var(0.0, 2));
  const double postb = bpost[c] + pb * r.d[0];
  aadd(&bnf[g.at(ci(dir, a - 1, l), cj(dir, a - 1, l))], pb * r.d[1]);
  aadd(&bnf[c], pb * r.d[2]);
  if (postb == 0.0) return;
  const X s = quarter_sum<X>(X::var(0.0, 0), X::var(0.0, 1), X::var(0.0, 2), X::var(0.0, 3));
  aadd(&bcm[g.at(x, y - 1)], postb * s.d[0]);
  aadd(&bcm[g.at(x, y)], postb * s.d[1]);
  aadd(&bcm[g.at(x - 1, y - 1)], postb * s.d[2]);
  aadd(&bcm[g.at(x - 1, y)], postb * s.d[3]);
}

// advec_mom cell masses: cm = rho * post_vol.
__global__ void k_adj_mom_cm(Grid g, int dir, int mom_sweep, const double *rho, const double *fx, const double *fy, const double *bcm,
                             double *brho, double *bfx, double *bfy) {
  const int na = dir == 1 ? g.nx : g.ny, nl = dir == 1 ? g.ny : g.nx;
  ADJ_IJ(0, 1, na + 4, nl + 2);
  const int x = ci(dir, i, j), y = cj(dir, i, j);
  const int c = g.at(x, y);
  const double b = bcm[c];
  if (b == 0.0) return;
  using X = DN<3>;
  const X vol = X(g.cdx[x] * g.cdy[y]);
  X pvv = vol;
  int lo = -1, hi = -1;
  double *bf = nullptr;
  if (mom_sweep == 1) {
    lo = g.at(x, y), hi = g.at(x, y + 1), bf = bfy;
    pvv = mom_post_vol<X>(1, vol, X::var(fy[lo], 1), X::var(fy[hi], 2));
  } else if (mom_sweep == 2) {
    lo = g.at(x, y), hi = g.at(x + 1, y), bf = bfx;
    pvv = mom_post_vol<X>(2, vol, X::var(fx[lo], 1), X::var(fx[hi], 2));
  }
  const X cmv = X::var(rho[c], 0) * pvv;
  aadd(&brho[c], b * cmv.d[0]);
  if (bf) {
    aadd(&bf[lo], b * cmv.d[1]);
    aadd(&bf[hi], b * cmv.d[2]);
  }
}

// advec_mom node flux: 0.25 * (four mass fluxes).
__global__ void k_adj_mom_nf(Grid g, int dir, const double *bnf, double *bmf) {
  const int na = dir == 1 ? g.nx : g.ny, nl = dir == 1 ? g.ny : g.nx;
  ADJ_IJ(0, 2, na + 4, nl + 1);
  const int a = i, l = j;
  const double b = bnf[g.at(ci(dir, a, l), cj(dir, a, l))];
  if (b == 0.0) return;
  using X = DN<4>;
  const X s = quarter_sum<X>(X::var(0.0, 0), X::var(0.0, 1), X::var(0.0, 2), X::var(0.0, 3));
  const int pos[4][2] = {{a, l - 1}, {a, l}, {a + 1, l - 1}, {a + 1, l}};
  for (int k = 0; k < 4; ++k) aadd(&bmf[g.at(ci(dir, pos[k][0], pos[k][1]), cj(dir, pos[k][0], pos[k][1]))], b * s.d[k]);
}

// Adds src into dst over [i0, i0+w) x [j0, j0+h) (reset_field, ring copies).
__global__ void k_adj_add(Grid g, const double *src, double *dst, int i0, int j0, int w, int h) {
  ADJ_IJ(i0, j0, w, h);
  const int c = g.at(i, j);
  dst[c] += src[c];
}

__global__ void k_adj_add_ring(Grid g, const double *src, double *dst, int ex, int ey, int lo, int hix, int hiy) {
  ADJ_IJ(0, 0, ex, ey);
  if (i >= lo && i <= hix && j >= lo && j <= hiy) return;
  const int c = g.at(i, j);
  dst[c] += src[c];
}

#undef ADJ_IJ

} // namespace adj
} // namespace cb
