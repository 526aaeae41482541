// cb_phase.cuh -- one CUDA kernel per hydro phase (the "phase" path).
//
// Each kernel is one pass over the mesh that does the whole of the
// reference routine it replaces (all of its loops fused, intermediate work
// arrays kept on chip) and, when asked, also writes the reflective halo of
// its outputs so that the update_halo call that follows becomes a no-op.
// The arithmetic of every expression keeps the reference's operation order;
// built with -fmad=false the FP64 instantiation is bit-identical to the
// reference serial model.
//
// Kernels are templated on the storage type T (double, or float for the
// FP32 form).  Where the FP32 form keeps FP64 (calc_dt's minimum, the
// summary sums, cell-advection mass/energy accumulation) the code says
// `double` explicitly.
#pragma once

#include "cb_mesh.cuh"
#include "cb_ops.h"

namespace cb {

// Fields of one chunk as seen by a kernel launch.
template <typename T> struct Fields {
  T *f[NUM_FIELDS];
};

// ---------------------------------------------------------------------------
// generate_chunk: src/serial/generate_chunk.cpp:31-131.  Later states
// overwrite earlier ones; a node takes the velocity of the last state that
// paints any of the (up to four) cells whose loop iteration writes it.
template <typename T>
__device__ __forceinline__ bool state_hits(const DevState &s, const Mesh<T> &m, const double *cellx, const double *celly,
                                           const double *vertexx, const double *vertexy, int i, int j) {
  if (s.geometry == 1) {
    return (vertexx[i + 1] >= s.xmin && vertexx[i] < s.xmax) && (vertexy[j + 1] >= s.ymin && vertexy[j] < s.ymax);
  } else if (s.geometry == 2) {
    double x_cent = s.xmin, y_cent = s.ymin;
    double radius = sqrt((cellx[i] - x_cent) * (cellx[i] - x_cent) + (celly[j] - y_cent) * (celly[j] - y_cent));
    return radius <= s.radius;
  } else if (s.geometry == 3) {
    return vertexx[i] == s.xmin && vertexy[j] == s.ymin;
  }
  return false;
}

template <typename T>
__global__ void k_generate_chunk(Fields<T> F, Mesh<T> m, const DevState *st, int nstates, const double *cellx,
                                 const double *celly, const double *vertexx, const double *vertexy) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int xr = m.nx + 4, yr = m.ny + 4;
  if (i > xr || j > yr) return;
  // cell part (cells cover [0, xr) x [0, yr))
  if (i < xr && j < yr) {
    double e = st[0].energy, d = st[0].density;
    for (int s = 1; s < nstates; ++s) {
      if (state_hits(st[s], m, cellx, celly, vertexx, vertexy, i, j)) {
        e = st[s].energy;
        d = st[s].density;
      }
    }
    F.f[ENERGY0][m.at(i, j)] = (T)e;
    F.f[DENSITY0][m.at(i, j)] = (T)d;
  }
  // node part: node (i, j) is written by cells (i-1..i, j-1..j)
  bool painted = false;
  double u = 0.0, v = 0.0;
  if (i < xr && j < yr) {
    u = st[0].xvel;
    v = st[0].yvel;
    painted = true;
  }
  for (int s = 1; s < nstates; ++s) {
    bool hit = false;
    for (int cj = j - 1; cj <= j; ++cj)
      for (int ci = i - 1; ci <= i; ++ci)
        if (ci >= 0 && cj >= 0 && ci < xr && cj < yr && state_hits(st[s], m, cellx, celly, vertexx, vertexy, ci, cj)) hit = true;
    if (hit) {
      u = st[s].xvel;
      v = st[s].yvel;
      painted = true;
    }
  }
  if (painted) {
    F.f[XVEL0][m.at(i, j)] = (T)u;
    F.f[YVEL0][m.at(i, j)] = (T)v;
  }
}

// ---------------------------------------------------------------------------
// ideal_gas: src/serial/ideal_gas.cpp:28-48.  gm1 = gamma - 1 (0.4 at the
// reference's hard-coded gamma = 1.4).
template <typename T>
__device__ __forceinline__ void eos(T density, T energy, T gm1, T &pressure, T &soundspeed) {
  T v = T(1.0) / density;
  pressure = gm1 * density * energy;
  T pressurebyenergy = gm1 * density;
  T pressurebyvolume = -density * pressure;
  T sound_speed_squared = v * v * (pressure * pressurebyenergy - pressurebyvolume);
  soundspeed = sqrt(sound_speed_squared);
}

template <typename T>
__global__ void k_ideal_gas(Fields<T> F, Mesh<T> m, int predict, T gm1, int fold) {
  const int i = 2 + blockIdx.x * blockDim.x + threadIdx.x;
  const int j = 2 + blockIdx.y * blockDim.y + threadIdx.y;
  if (i >= m.nx + 2 || j >= m.ny + 2) return;
  const long long id = m.at(i, j);
  T p, c;
  eos(F.f[predict ? DENSITY1 : DENSITY0][id], F.f[predict ? ENERGY1 : ENERGY0][id], gm1, p, c);
  F.f[PRESSURE][id] = p;
  F.f[SOUNDSPEED][id] = c;
  if (fold) fold_halo(F.f[PRESSURE], m, halo_rule(PRESSURE), fold, i, j, p);
}

// ---------------------------------------------------------------------------
// viscosity: src/serial/viscosity.cpp:30-68 including the diry quirk (:57).
template <typename T>
__device__ __forceinline__ T viscosity_at(const T *xvel0, const T *yvel0, const T *pressure, T density0, const Mesh<T> &m,
                                          int i, int j) {
  const T cdx = m.celldx_t[i], cdy = m.celldy_t[j], cdx1 = m.celldx_t[i + 1], cdy2 = m.celldy_t[j + 2];
  const T u00 = xvel0[m.at(i, j)], u10 = xvel0[m.at(i + 1, j)], u01 = xvel0[m.at(i, j + 1)], u11 = xvel0[m.at(i + 1, j + 1)];
  const T v00 = yvel0[m.at(i, j)], v10 = yvel0[m.at(i + 1, j)], v01 = yvel0[m.at(i, j + 1)], v11 = yvel0[m.at(i + 1, j + 1)];
  T ugrad = (u10 + u11) - (u00 + u01);
  T vgrad = (v01 + v11) - (v00 + v10);
  T div = (cdx * (ugrad) + cdy * (vgrad));
  T strain2 = T(0.5) * (u01 + u11 - u00 - u10) / cdy + T(0.5) * (v10 + v11 - v00 - v01) / cdx;
  T pgradx = (pressure[m.at(i + 1, j)] - pressure[m.at(i - 1, j)]) / (cdx + cdx1);
  T pgrady = (pressure[m.at(i, j + 1)] - pressure[m.at(i, j - 1)]) / (cdy + cdy2);
  T pgradx2 = pgradx * pgradx;
  T pgrady2 = pgrady * pgrady;
  T limiter = ((T(0.5) * (ugrad) / cdx) * pgradx2 + (T(0.5) * (vgrad) / cdy) * pgrady2 + strain2 * pgradx * pgrady) /
              fmax(pgradx2 + pgrady2, T(g_small));
  if ((limiter > T(0.0)) || (div >= T(0.0))) return T(0.0);
  T dirx = T(1.0);
  if (pgradx < T(0.0)) dirx = T(-1.0);
  pgradx = dirx * fmax(T(g_small), fabs(pgradx));
  T diry = T(1.0);
  if (pgradx < T(0.0)) diry = T(-1.0);
  pgrady = diry * fmax(T(g_small), fabs(pgrady));
  T pgrad = sqrt(pgradx * pgradx + pgrady * pgrady);
  T xgrad = fabs(cdx * pgrad / pgradx);
  T ygrad = fabs(cdy * pgrad / pgrady);
  T grad = fmin(xgrad, ygrad);
  T grad2 = grad * grad;
  return T(2.0) * density0 * grad2 * limiter * limiter;
}

template <typename T>
__global__ void k_viscosity(Fields<T> F, Mesh<T> m, int fold) {
  const int i = 2 + blockIdx.x * blockDim.x + threadIdx.x;
  const int j = 2 + blockIdx.y * blockDim.y + threadIdx.y;
  if (i >= m.nx + 2 || j >= m.ny + 2) return;
  T q = viscosity_at(F.f[XVEL0], F.f[YVEL0], F.f[PRESSURE], F.f[DENSITY0][m.at(i, j)], m, i, j);
  F.f[VISCOSITY][m.at(i, j)] = q;
  if (fold) fold_halo(F.f[VISCOSITY], m, halo_rule(VISCOSITY), fold, i, j, q);
}

// ---------------------------------------------------------------------------
// calc_dt: src/serial/calc_dt.cpp:30-79.  Every cell's candidate is formed
// in T; the minimum is taken in FP64 on the device: a warp/block min, then
// one atomicMin per block on the bit pattern (all candidates are >= 0 and
// NaN candidates lose, as std::fmin ignores them).
template <typename T>
__device__ __forceinline__ T dt_candidate(const Fields<T> &F, const Mesh<T> &m, const DtConsts &k, int i, int j) {
  const T dsx = m.celldx_t[i], dsy = m.celldy_t[j];
  const T vol = dsx * dsy;                     // volume(i, j) = dx * dy
  const T xa0 = m.celldy_t[j], xa1 = xa0;      // xarea(i, j) = xarea(i+1, j) = celldy[j]
  const T ya0 = m.celldx_t[i], ya1 = ya0;      // yarea(i, j) = yarea(i, j+1) = celldx[i]
  const long long id = m.at(i, j);
  const T *xvel0 = F.f[XVEL0], *yvel0 = F.f[YVEL0];
  T ss = F.f[SOUNDSPEED][id];
  T cc = ss * ss;
  cc = cc + T(2.0) * F.f[VISCOSITY][id] / F.f[DENSITY0][id];
  cc = fmax(sqrt(cc), T(g_small));
  T dtct = T(k.dtc_safe) * fmin(dsx, dsy) / cc;
  T div = T(0.0);
  T dv1 = (xvel0[id] + xvel0[m.at(i, j + 1)]) * xa0;
  T dv2 = (xvel0[m.at(i + 1, j)] + xvel0[m.at(i + 1, j + 1)]) * xa1;
  div = div + dv2 - dv1;
  T dtut = T(k.dtu_safe) * T(2.0) * vol / fmax(fmax(fabs(dv1), fabs(dv2)), T(g_small) * vol);
  dv1 = (yvel0[id] + yvel0[m.at(i + 1, j)]) * ya0;
  dv2 = (yvel0[m.at(i, j + 1)] + yvel0[m.at(i + 1, j + 1)]) * ya1;
  div = div + dv2 - dv1;
  T dtvt = T(k.dtv_safe) * T(2.0) * vol / fmax(fmax(fabs(dv1), fabs(dv2)), T(g_small) * vol);
  div = div / (T(2.0) * vol);
  T dtdivt;
  if (div < T(-g_small)) {
    dtdivt = T(k.dtdiv_safe) * (T(-1.0) / div);
  } else {
    dtdivt = T(g_big);
  }
  return fmin(dtct, fmin(dtut, fmin(dtvt, fmin(dtdivt, T(g_big)))));
}

__device__ __forceinline__ double warp_min(double v) {
  for (int o = 16; o > 0; o >>= 1) v = fmin(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

// Block-wide min of v (any block size that is a multiple of 32, <= 1024);
// thread 0 then folds it into *out with one 64-bit atomicMin.
__device__ __forceinline__ void block_min_to(double v, unsigned long long *out) {
  __shared__ double wmin[32];
  v = warp_min(v);
  const int lane = (threadIdx.y * blockDim.x + threadIdx.x) & 31;
  const int warp = (threadIdx.y * blockDim.x + threadIdx.x) >> 5;
  const int nw = (blockDim.x * blockDim.y) >> 5;
  if (lane == 0) wmin[warp] = v;
  __syncthreads();
  if (warp == 0) {
    v = lane < nw ? wmin[lane] : g_big;
    v = warp_min(v);
    if (lane == 0 && v >= 0.0) atomicMin(out, (unsigned long long)__double_as_longlong(v));
  }
}

template <typename T>
__global__ void k_calc_dt(Fields<T> F, Mesh<T> m, DtConsts k, unsigned long long *dt_bits, int tiles_x, int ntiles) {
  double v = g_big;
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const int i = 2 + (t % tiles_x) * blockDim.x + threadIdx.x;
    const int j = 2 + (t / tiles_x) * blockDim.y + threadIdx.y;
    if (i < m.nx + 2 && j < m.ny + 2) {
      double c = (double)dt_candidate(F, m, k, i, j);
      v = fmin(c, v); // fmin drops a NaN candidate, as the reference's fmin does
    }
  }
  block_min_to(v, dt_bits);
}

// ---------------------------------------------------------------------------
// PdV: src/serial/PdV.cpp:36-87.  mode 0 = the kernel alone (writes
// density1, energy1); mode 1 = the whole predictor step of the model's PdV
// driver (:92-133): kernel, ideal_gas on level 1, the depth-1 pressure halo
// (folded) and revert, whose net effect on level 1 is density1 = density0,
// energy1 = energy0.
template <typename T>
__device__ __forceinline__ void pdv_cell(const Fields<T> &F, const Mesh<T> &m, bool predict, T dt, int i, int j,
                                         T &density1, T &energy1) {
  const T *xvel0 = F.f[XVEL0], *yvel0 = F.f[YVEL0], *xvel1 = F.f[XVEL1], *yvel1 = F.f[YVEL1];
  const T xa_l = m.celldy_t[j], xa_r = xa_l;  // xarea(i, j), xarea(i+1, j)
  const T ya_b = m.celldx_t[i], ya_t = ya_b;  // yarea(i, j), yarea(i, j+1)
  const T vol = m.celldx_t[i] * m.celldy_t[j];
  const long long id = m.at(i, j);
  const T u00 = xvel0[id], u01 = xvel0[m.at(i, j + 1)], u10 = xvel0[m.at(i + 1, j)], u11 = xvel0[m.at(i + 1, j + 1)];
  const T v00 = yvel0[id], v10 = yvel0[m.at(i + 1, j)], v01 = yvel0[m.at(i, j + 1)], v11 = yvel0[m.at(i + 1, j + 1)];
  T left_flux, right_flux, bottom_flux, top_flux;
  if (predict) {
    left_flux = (xa_l * (u00 + u01 + u00 + u01)) * T(0.25) * dt * T(0.5);
    right_flux = (xa_r * (u10 + u11 + u10 + u11)) * T(0.25) * dt * T(0.5);
    bottom_flux = (ya_b * (v00 + v10 + v00 + v10)) * T(0.25) * dt * T(0.5);
    top_flux = (ya_t * (v01 + v11 + v01 + v11)) * T(0.25) * dt * T(0.5);
  } else {
    const T w00 = xvel1[id], w01 = xvel1[m.at(i, j + 1)], w10 = xvel1[m.at(i + 1, j)], w11 = xvel1[m.at(i + 1, j + 1)];
    const T z00 = yvel1[id], z10 = yvel1[m.at(i + 1, j)], z01 = yvel1[m.at(i, j + 1)], z11 = yvel1[m.at(i + 1, j + 1)];
    left_flux = (xa_l * (u00 + u01 + w00 + w01)) * T(0.25) * dt;
    right_flux = (xa_r * (u10 + u11 + w10 + w11)) * T(0.25) * dt;
    bottom_flux = (ya_b * (v00 + v10 + z00 + z10)) * T(0.25) * dt;
    top_flux = (ya_t * (v01 + v11 + z01 + z11)) * T(0.25) * dt;
  }
  T total_flux = right_flux - left_flux + top_flux - bottom_flux;
  T volume_change_s = vol / (vol + total_flux);
  T recip_volume = T(1.0) / vol;
  const T d0 = F.f[DENSITY0][id];
  T energy_change = (F.f[PRESSURE][id] / d0 + F.f[VISCOSITY][id] / d0) * total_flux * recip_volume;
  energy1 = F.f[ENERGY0][id] - energy_change;
  density1 = d0 * volume_change_s;
}

template <typename T>
__global__ void k_pdv(Fields<T> F, Mesh<T> m, int predict, T dt, int mode, T gm1, int fold) {
  const int i = 2 + blockIdx.x * blockDim.x + threadIdx.x;
  const int j = 2 + blockIdx.y * blockDim.y + threadIdx.y;
  if (i >= m.nx + 2 || j >= m.ny + 2) return;
  T d1, e1;
  pdv_cell(F, m, predict != 0, dt, i, j, d1, e1);
  const long long id = m.at(i, j);
  if (mode == 0) {
    F.f[DENSITY1][id] = d1;
    F.f[ENERGY1][id] = e1;
    if (fold) {
      fold_halo(F.f[DENSITY1], m, halo_rule(DENSITY1), fold, i, j, d1);
      fold_halo(F.f[ENERGY1], m, halo_rule(ENERGY1), fold, i, j, e1);
    }
  } else {
    T p, c;
    eos(d1, e1, gm1, p, c);
    F.f[PRESSURE][id] = p;
    F.f[SOUNDSPEED][id] = c;
    if (fold) fold_halo(F.f[PRESSURE], m, halo_rule(PRESSURE), fold, i, j, p);
    F.f[DENSITY1][id] = F.f[DENSITY0][id];
    F.f[ENERGY1][id] = F.f[ENERGY0][id];
  }
}

// revert: src/serial/revert.cpp:29-41.
template <typename T>
__global__ void k_revert(Fields<T> F, Mesh<T> m) {
  const int i = 2 + blockIdx.x * blockDim.x + threadIdx.x;
  const int j = 2 + blockIdx.y * blockDim.y + threadIdx.y;
  if (i >= m.nx + 2 || j >= m.ny + 2) return;
  const long long id = m.at(i, j);
  F.f[DENSITY1][id] = F.f[DENSITY0][id];
  F.f[ENERGY1][id] = F.f[ENERGY0][id];
}

// ---------------------------------------------------------------------------
// accelerate: src/serial/accelerate.cpp:28-56 over nodes [2, nx+3) x [2, ny+3).
template <typename T>
__device__ __forceinline__ void accelerate_node(const Fields<T> &F, const Mesh<T> &m, T halfdt, int i, int j, T &u1, T &v1) {
  const T *d0 = F.f[DENSITY0], *p = F.f[PRESSURE], *q = F.f[VISCOSITY];
  const T vol_mm = m.celldx_t[i - 1] * m.celldy_t[j - 1], vol_m0 = m.celldx_t[i - 1] * m.celldy_t[j];
  const T vol_00 = m.celldx_t[i] * m.celldy_t[j], vol_0m = m.celldx_t[i] * m.celldy_t[j - 1];
  const long long c00 = m.at(i, j), cm0 = m.at(i - 1, j), c0m = m.at(i, j - 1), cmm = m.at(i - 1, j - 1);
  T stepbymass_s = halfdt / ((d0[cmm] * vol_mm + d0[cm0] * vol_m0 + d0[c00] * vol_00 + d0[c0m] * vol_0m) * T(0.25));
  const T xa = m.celldy_t[j], xa_m = m.celldy_t[j - 1]; // xarea(i, j), xarea(i, j-1)
  const T ya = m.celldx_t[i], ya_m = m.celldx_t[i - 1]; // yarea(i, j), yarea(i-1, j)
  T u = F.f[XVEL0][c00] - stepbymass_s * (xa * (p[c00] - p[cm0]) + xa_m * (p[c0m] - p[cmm]));
  T v = F.f[YVEL0][c00] - stepbymass_s * (ya * (p[c00] - p[c0m]) + ya_m * (p[cm0] - p[cmm]));
  u = u - stepbymass_s * (xa * (q[c00] - q[cm0]) + xa_m * (q[c0m] - q[cmm]));
  v = v - stepbymass_s * (ya * (q[c00] - q[c0m]) + ya_m * (q[cm0] - q[cmm]));
  u1 = u;
  v1 = v;
}

template <typename T>
__global__ void k_accelerate(Fields<T> F, Mesh<T> m, T dt, int fold) {
  const int i = 2 + blockIdx.x * blockDim.x + threadIdx.x;
  const int j = 2 + blockIdx.y * blockDim.y + threadIdx.y;
  if (i >= m.nx + 3 || j >= m.ny + 3) return;
  T halfdt = T(0.5) * dt;
  T u, v;
  accelerate_node(F, m, halfdt, i, j, u, v);
  F.f[XVEL1][m.at(i, j)] = u;
  F.f[YVEL1][m.at(i, j)] = v;
  if (fold) {
    fold_halo(F.f[XVEL1], m, halo_rule(XVEL1), fold, i, j, u);
    fold_halo(F.f[YVEL1], m, halo_rule(YVEL1), fold, i, j, v);
  }
}

// ---------------------------------------------------------------------------
// flux_calc: src/serial/flux_calc.cpp:27-43 over faces [2, nx+3) x [2, ny+3).
// With a fold, the extra row of x faces (j = ny+2) and column of y faces
// (i = nx+2), which update_halo overwrites, take their halo values instead.
template <typename T>
__global__ void k_flux_calc(Fields<T> F, Mesh<T> m, T dt, int fold) {
  const int i = 2 + blockIdx.x * blockDim.x + threadIdx.x;
  const int j = 2 + blockIdx.y * blockDim.y + threadIdx.y;
  if (i >= m.nx + 3 || j >= m.ny + 3) return;
  const T *u0 = F.f[XVEL0], *v0 = F.f[YVEL0], *u1 = F.f[XVEL1], *v1 = F.f[YVEL1];
  const long long id = m.at(i, j);
  T fx = T(0.25) * dt * m.celldy_t[j] * (u0[id] + u0[m.at(i, j + 1)] + u1[id] + u1[m.at(i, j + 1)]);
  T fy = T(0.25) * dt * m.celldx_t[i] * (v0[id] + v0[m.at(i + 1, j)] + v1[id] + v1[m.at(i + 1, j)]);
  if (!fold) {
    F.f[VOL_FLUX_X][id] = fx;
    F.f[VOL_FLUX_Y][id] = fy;
    return;
  }
  if (j < m.ny + 2) {
    F.f[VOL_FLUX_X][id] = fx;
    fold_halo(F.f[VOL_FLUX_X], m, halo_rule(VOL_FLUX_X), fold, i, j, fx);
  }
  if (i < m.nx + 2) {
    F.f[VOL_FLUX_Y][id] = fy;
    fold_halo(F.f[VOL_FLUX_Y], m, halo_rule(VOL_FLUX_Y), fold, i, j, fy);
  }
}

// ---------------------------------------------------------------------------
// advec_cell: src/serial/advec_cell.cpp:28-220, the three loops of one sweep
// fused into one pass.  Reads density1/energy1 from (sd, se), writes the
// update to (dd, de) -- the host swaps the buffers afterwards -- and writes
// the mass flux of the sweep direction.  pre_vol/ener_flux stay on chip:
// a block first computes the fluxes of its faces (one more face than cells
// per line) into shared memory, then updates its cells.
template <typename T>
__device__ __forceinline__ T cell_limiter(T sigma, T sigma3, T sigma4, T diffuw, T diffdw) {
  const T one_by_six = T(1.0 / 6.0);
  T wind = T(1.0);
  if (diffdw <= T(0.0)) wind = T(-1.0);
  if (diffuw * diffdw > T(0.0)) {
    return (T(1.0) - sigma) * wind * fmin(fmin(fabs(diffuw), fabs(diffdw)), one_by_six * (sigma3 * fabs(diffuw) + sigma4 * fabs(diffdw)));
  }
  return T(0.0);
}

// pre_vol of cell (i, j) for the given sweep/direction (advec_cell.cpp:42-61 and :134-153).
template <typename T>
__device__ __forceinline__ T cell_pre_vol(const T *vfx, const T *vfy, const Mesh<T> &m, int sweep, int dir, int i, int j) {
  const T vol = m.celldx_t[i] * m.celldy_t[j];
  if (dir == 1) {
    if (sweep == 1) return vol + (vfx[m.at(i + 1, j)] - vfx[m.at(i, j)] + vfy[m.at(i, j + 1)] - vfy[m.at(i, j)]);
    return vol + vfx[m.at(i + 1, j)] - vfx[m.at(i, j)];
  }
  if (sweep == 1) return vol + (vfy[m.at(i, j + 1)] - vfy[m.at(i, j)] + vfx[m.at(i + 1, j)] - vfx[m.at(i, j)]);
  return vol + vfy[m.at(i, j + 1)] - vfy[m.at(i, j)];
}

// Block shapes of the cell sweeps.  threadIdx.x always runs along x so every
// warp reads consecutive addresses; in the x sweep the TA = 32 x-threads cover
// NA = 64 cells and the 8 y-threads 8 rows, in the y sweep the 8 y-threads
// cover NA = 32 cells along y and the 32 x-threads 32 columns.
template <int DIR> struct CellSweep;
template <> struct CellSweep<1> { static constexpr int TX = 32, TY = 8, TA = 32, NA = 64, NL = 8; };
template <> struct CellSweep<2> { static constexpr int TX = 32, TY = 8, TA = 8, NA = 32, NL = 32; };

// Mass and energy flux through face f of line `line` (an x face, the left
// face of cell f, when DIR == 1; a y face when DIR == 2): the flux loop body
// of advec_cell.cpp:68-113 / :160-205.  Returns the mass flux; the energy
// flux is formed in FP64 (the FP32 form keeps that accumulation in FP64).
template <typename T, int DIR>
__device__ __forceinline__ double cell_face_flux(const T *d1, const T *e1, const T *vfx, const T *vfy, const Mesh<T> &m, int sweep,
                                                 int f, int line, double *ef) {
  const int nmax = DIR == 1 ? m.nx : m.ny;
  const T *vf = DIR == 1 ? vfx : vfy;
  const double *vdx = DIR == 1 ? m.vertexdx : m.vertexdy;
  auto at = [&](int a) { return DIR == 1 ? m.at(a, line) : m.at(line, a); };
  auto pv = [&](int a) {
    return DIR == 1 ? cell_pre_vol(vfx, vfy, m, sweep, DIR, a, line) : cell_pre_vol(vfx, vfy, m, sweep, DIR, line, a);
  };
  const T flux = vf[at(f)];
  int upwind, donor, downwind, dif;
  if (flux > T(0.0)) {
    upwind = f - 2; donor = f - 1; downwind = f; dif = donor;
  } else {
    upwind = (f + 1 < nmax + 2) ? f + 1 : nmax + 2;
    donor = f; downwind = f - 1; dif = upwind;
  }
  const T pre_vol_d = pv(donor);
  T sigmat = fabs(flux) / pre_vol_d;
  T sigma3 = (T(1.0) + sigmat) * (T)(vdx[f] / vdx[dif]);
  T sigma4 = T(2.0) - sigmat;
  T sigmav = sigmat;
  const T dd = d1[at(donor)], du = d1[at(upwind)], dw = d1[at(downwind)];
  T limiter = cell_limiter(sigmav, sigma3, sigma4, dd - du, dw - dd);
  T mass_flux = flux * (dd + limiter);
  T sigmam = fabs(mass_flux) / (dd * pre_vol_d);
  const T ed = e1[at(donor)], eu = e1[at(upwind)], ew = e1[at(downwind)];
  limiter = cell_limiter(sigmam, sigma3, sigma4, ed - eu, ew - ed);
  *ef = (double)mass_flux * (double)(ed + limiter);
  return (double)mass_flux;
}

template <typename T, int DIR>
__global__ void __launch_bounds__(256) k_advec_cell(Fields<T> F, Mesh<T> m, int sweep, const T *sd, const T *se, T *dd, T *de,
                                                    int fold) {
  using K = CellSweep<DIR>;
  constexpr int NA = K::NA, NL = K::NL, TA = K::TA;
  __shared__ double s_mf[(NA + 1) * NL];
  __shared__ double s_ef[(NA + 1) * NL];
  // shared layout keeps the warp's fastest thread index contiguous
  auto sidx = [](int p, int l) { return DIR == 1 ? l * (NA + 1) + p : p * NL + l; };
  const int ta = DIR == 1 ? threadIdx.x : threadIdx.y;
  const int tl = DIR == 1 ? threadIdx.y : threadIdx.x;
  const int na = DIR == 1 ? m.nx : m.ny, nl = DIR == 1 ? m.ny : m.nx;
  const int a0 = 2 + (DIR == 1 ? blockIdx.x : blockIdx.y) * NA;
  const int line = 2 + (DIR == 1 ? blockIdx.y : blockIdx.x) * NL + tl;
  const bool line_ok = line < nl + 2;
  T *mf = F.f[DIR == 1 ? MASS_FLUX_X : MASS_FLUX_Y];
  const T *vfx = F.f[VOL_FLUX_X], *vfy = F.f[VOL_FLUX_Y];
  auto at = [&](int aa, int ll) { return DIR == 1 ? m.at(aa, ll) : m.at(ll, aa); };
  // faces a0 .. a0 + NA (faces run to na + 3)
  for (int p = ta; p <= NA; p += TA) {
    const int f = a0 + p;
    if (!line_ok || f > na + 3) continue;
    double ef;
    const double mfv = cell_face_flux<T, DIR>(sd, se, vfx, vfy, m, sweep, f, line, &ef);
    s_mf[sidx(p, tl)] = mfv;
    s_ef[sidx(p, tl)] = ef;
    if (!(fold && f == na + 3)) mf[at(f, line)] = (T)mfv; // with a fold, face na+3 takes its halo value
    if (fold && f < na + 3) {
      if (DIR == 1) fold_halo(mf, m, halo_rule(MASS_FLUX_X), fold, f, line, (T)mfv);
      else fold_halo(mf, m, halo_rule(MASS_FLUX_Y), fold, line, f, (T)mfv);
    }
  }
  __syncthreads();
  const T *vf = DIR == 1 ? vfx : vfy;
  for (int p = ta; p < NA; p += TA) {
    const int a = a0 + p;
    if (!line_ok || a >= na + 2) continue;
    const long long id = at(a, line);
    const int i = DIR == 1 ? a : line, j = DIR == 1 ? line : a;
    const T pre_vol = cell_pre_vol(vfx, vfy, m, sweep, DIR, i, j);
    // advec_cell.cpp:122-128: the mass/energy accumulation, in FP64 in both forms
    double pre_mass_s = (double)sd[id] * (double)pre_vol;
    double post_mass_s = pre_mass_s + s_mf[sidx(p, tl)] - s_mf[sidx(p + 1, tl)];
    double post_ener_s = ((double)se[id] * pre_mass_s + s_ef[sidx(p, tl)] - s_ef[sidx(p + 1, tl)]) / post_mass_s;
    double advec_vol_s = (double)pre_vol + (double)vf[id] - (double)vf[at(a + 1, line)];
    T dnew = (T)(post_mass_s / advec_vol_s);
    T enew = (T)post_ener_s;
    dd[id] = dnew;
    de[id] = enew;
    if (fold) {
      fold_halo(dd, m, halo_rule(DENSITY1), fold, i, j, dnew);
      fold_halo(de, m, halo_rule(ENERGY1), fold, i, j, enew);
    }
  }
}

// ---------------------------------------------------------------------------
// advec_mom: src/serial/advec_mom.cpp:30-225, both velocity components in
// one pass when vel_mask == 3 (the which_vel == 1 call computes node flux
// and node masses that the which_vel == 2 call reuses, :81-103).  Reads
// velocities from (su, sv), writes to (du, dv); the host swaps buffers.
// node_flux, node masses and mom_flux stay in shared memory.
template <typename T>
__device__ __forceinline__ T mom_limited(T vdiffuw, T vdiffdw, T sigma, T width, T dx_dif) {
  T limiter = T(0.0);
  if (vdiffuw * vdiffdw > T(0.0)) {
    T auw = fabs(vdiffuw);
    T adw = fabs(vdiffdw);
    T wind = T(1.0);
    if (vdiffdw <= T(0.0)) wind = T(-1.0);
    limiter = wind * fmin(fmin(width * ((T(2.0) - sigma) * adw / width + (T(1.0) + sigma) * auw / dx_dif) / T(6.0), auw), adw);
  }
  return limiter;
}

// post_vol of cell (i, j) (advec_mom.cpp:42-77): mom_sweep 1 (x, sweep 1)
// vol + vfy diff; 2 (y, sweep 1) vol + vfx diff; 3, 4 (sweep 2) vol.
template <typename T>
__device__ __forceinline__ T mom_post_vol(const T *vfx, const T *vfy, const Mesh<T> &m, int mom_sweep, int i, int j) {
  const T vol = m.celldx_t[i] * m.celldy_t[j];
  if (mom_sweep == 1) return vol + vfy[m.at(i, j + 1)] - vfy[m.at(i, j)];
  if (mom_sweep == 2) return vol + vfx[m.at(i + 1, j)] - vfx[m.at(i, j)];
  return vol;
}

// Block shapes of the momentum sweeps: NA nodes along the sweep axis per
// block (plus two on each side that only feed the fluxes of the inner ones),
// NL lines across; threadIdx.x runs along x in both directions.
template <int DIR> struct MomSweep;
template <> struct MomSweep<1> { static constexpr int TX = 32, TY = 8, TA = 32, NA = 64, NL = 8; };
template <> struct MomSweep<2> { static constexpr int TX = 32, TY = 8, TA = 8, NA = 32, NL = 32; };

template <typename T, int DIR>
__global__ void __launch_bounds__(256) k_advec_mom(Fields<T> F, Mesh<T> m, int vel_mask, int sweep, const T *su, const T *sv, T *du,
                                                   T *dv, int fold) {
  using K = MomSweep<DIR>;
  constexpr int NA = K::NA, NL = K::NL, TA = K::TA, NP = NA + 4;
  __shared__ T s_nf[NP * NL];     // node_flux
  __shared__ T s_nmpre[NP * NL];  // node_mass_pre
  __shared__ T s_nmpost[NP * NL]; // node_mass_post
  __shared__ T s_mfu[NP * NL];    // mom_flux of the x velocity
  __shared__ T s_mfv[NP * NL];    // mom_flux of the y velocity
  auto sidx = [](int p, int l) { return DIR == 1 ? l * NP + p : p * NL + l; };
  const int mom_sweep = DIR + 2 * (sweep - 1);
  const int ta = DIR == 1 ? threadIdx.x : threadIdx.y;
  const int tl = DIR == 1 ? threadIdx.y : threadIdx.x;
  const int na = DIR == 1 ? m.nx : m.ny, nl = DIR == 1 ? m.ny : m.nx;
  const int a0 = 2 + (DIR == 1 ? blockIdx.x : blockIdx.y) * NA; // first updated node; position p <-> node a0 - 2 + p
  const int line = 2 + (DIR == 1 ? blockIdx.y : blockIdx.x) * NL + tl;
  const bool line_ok = line < nl + 3;
  auto at = [&](int aa, int ll) { return DIR == 1 ? m.at(aa, ll) : m.at(ll, aa); };
  const T *vfx = F.f[VOL_FLUX_X], *vfy = F.f[VOL_FLUX_Y];
  const T *d1 = F.f[DENSITY1];
  const T *mflux = F.f[DIR == 1 ? MASS_FLUX_X : MASS_FLUX_Y];
  // node_flux over nodes [0, na+3] (advec_mom.cpp:84-88 / :156-160)
  for (int p = ta; p < NP; p += TA) {
    const int a = a0 - 2 + p;
    T nf = T(0.0);
    if (line_ok && a >= 0 && a <= na + 3) {
      if (DIR == 1)
        nf = T(0.25) * (mflux[m.at(a, line - 1)] + mflux[m.at(a, line)] + mflux[m.at(a + 1, line - 1)] + mflux[m.at(a + 1, line)]);
      else
        nf = T(0.25) * (mflux[m.at(line - 1, a)] + mflux[m.at(line, a)] + mflux[m.at(line - 1, a + 1)] + mflux[m.at(line, a + 1)]);
    }
    s_nf[sidx(p, tl)] = nf;
  }
  __syncthreads();
  // node_mass_post / node_mass_pre over nodes [1, na+3] (:93-102 / :165-174)
  for (int p = ta; p < NP; p += TA) {
    const int a = a0 - 2 + p;
    T nmpost = T(1.0), nmpre = T(1.0);
    if (line_ok && p >= 1 && a >= 1 && a <= na + 3) {
      const int i = DIR == 1 ? a : line, j = DIR == 1 ? line : a;
      nmpost = T(0.25) * (d1[m.at(i, j - 1)] * mom_post_vol(vfx, vfy, m, mom_sweep, i, j - 1) +
                          d1[m.at(i, j)] * mom_post_vol(vfx, vfy, m, mom_sweep, i, j) +
                          d1[m.at(i - 1, j - 1)] * mom_post_vol(vfx, vfy, m, mom_sweep, i - 1, j - 1) +
                          d1[m.at(i - 1, j)] * mom_post_vol(vfx, vfy, m, mom_sweep, i - 1, j));
      nmpre = nmpost - s_nf[sidx(p - 1, tl)] + s_nf[sidx(p, tl)];
    }
    s_nmpost[sidx(p, tl)] = nmpost;
    s_nmpre[sidx(p, tl)] = nmpre;
  }
  __syncthreads();
  // mom_flux over nodes [1, na+2] (:108-133 / :180-205): positions [1, NA+1]
  const T *celld = DIR == 1 ? m.celldx_t : m.celldy_t;
  for (int p = 1 + ta; p <= NA + 1; p += TA) {
    const int a = a0 - 2 + p;
    if (!line_ok || a < 1 || a > na + 2) continue;
    const T nf = s_nf[sidx(p, tl)];
    int upwind, donor, downwind, dif;
    if (nf < T(0.0)) {
      upwind = a + 2; donor = a + 1; downwind = a; dif = donor;
    } else {
      upwind = a - 1; donor = a; downwind = a + 1; dif = upwind;
    }
    const T sigma = fabs(nf) / s_nmpre[sidx(p + (donor - a), tl)];
    const T width = celld[a];
    if (vel_mask & 1) {
      const T vd = su[at(donor, line)];
      T lim = mom_limited(vd - su[at(upwind, line)], su[at(downwind, line)] - vd, sigma, width, celld[dif]);
      s_mfu[sidx(p, tl)] = (vd + (T(1.0) - sigma) * lim) * nf;
    }
    if (vel_mask & 2) {
      const T vd = sv[at(donor, line)];
      T lim = mom_limited(vd - sv[at(upwind, line)], sv[at(downwind, line)] - vd, sigma, width, celld[dif]);
      s_mfv[sidx(p, tl)] = (vd + (T(1.0) - sigma) * lim) * nf;
    }
  }
  __syncthreads();
  // velocity update over nodes [2, na+2] (:139-144 / :211-216): positions [2, NA+2)
  for (int p = 2 + ta; p < NA + 2; p += TA) {
    const int a = a0 - 2 + p;
    if (!line_ok || a > na + 2) continue;
    const long long id = at(a, line);
    const int i = DIR == 1 ? a : line, j = DIR == 1 ? line : a;
    const T nmpre = s_nmpre[sidx(p, tl)], nmpost = s_nmpost[sidx(p, tl)];
    if (vel_mask & 1) {
      T v = (su[id] * nmpre + s_mfu[sidx(p - 1, tl)] - s_mfu[sidx(p, tl)]) / nmpost;
      du[id] = v;
      if (fold) fold_halo(du, m, halo_rule(XVEL1), fold, i, j, v);
    }
    if (vel_mask & 2) {
      T v = (sv[id] * nmpre + s_mfv[sidx(p - 1, tl)] - s_mfv[sidx(p, tl)]) / nmpost;
      dv[id] = v;
      if (fold) fold_halo(dv, m, halo_rule(YVEL1), fold, i, j, v);
    }
  }
}

// ---------------------------------------------------------------------------
// reset_field: src/serial/reset_field.cpp:28-51.
// With a fold, level 0 also gets the halo update_halo(depth) would give it.
template <typename T>
__global__ void k_reset_field(Fields<T> F, Mesh<T> m, int fold) {
  const int i = 2 + blockIdx.x * blockDim.x + threadIdx.x;
  const int j = 2 + blockIdx.y * blockDim.y + threadIdx.y;
  if (i >= m.nx + 3 || j >= m.ny + 3) return;
  const long long id = m.at(i, j);
  if (i < m.nx + 2 && j < m.ny + 2) {
    const T d = F.f[DENSITY1][id], e = F.f[ENERGY1][id];
    F.f[DENSITY0][id] = d;
    F.f[ENERGY0][id] = e;
    if (fold) {
      fold_halo(F.f[DENSITY0], m, halo_rule(DENSITY0), fold, i, j, d);
      fold_halo(F.f[ENERGY0], m, halo_rule(ENERGY0), fold, i, j, e);
    }
  }
  const T u = F.f[XVEL1][id], v = F.f[YVEL1][id];
  F.f[XVEL0][id] = u;
  F.f[YVEL0][id] = v;
  if (fold) {
    fold_halo(F.f[XVEL0], m, halo_rule(XVEL0), fold, i, j, u);
    fold_halo(F.f[YVEL0], m, halo_rule(YVEL0), fold, i, j, v);
  }
}

// Copies the elements of `src` outside the rectangle [ilo, ihi] x [jlo, jhi]
// (the ring of width 2 or 3 around it) into `dst`, so a double-buffered
// update leaves dst's halo exactly as the in-place reference leaves it.
template <typename T>
__global__ void k_copy_ring(const T *src, T *dst, Mesh<T> m, int ilo, int ihi, int jlo, int jhi, int ext_x, int ext_y) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int w = ext_x, h = ext_y;
  if (t >= w * h) return;
  const int i = t % w, j = t / w;
  if (i >= ilo && i <= ihi && j >= jlo && j <= jhi) return;
  dst[m.at(i, j)] = src[m.at(i, j)];
}

// ---------------------------------------------------------------------------
// update_halo: src/serial/update_halo.cpp:33-684 in two launches: pass 0 does
// bottom then top for every column, pass 1 left then right for every row, so
// corner and tiny-mesh semantics are the reference's exactly.
template <typename T>
__global__ void k_update_halo(Fields<T> F, Mesh<T> m, HaloJob job, int depth, int pass) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int fi = blockIdx.y;
  if (fi >= job.nfields) return;
  const int f = job.field[fi];
  const HaloRule r = halo_rule(f);
  T *a = F.f[f];
  const int d = depth;
  if (pass == 0) {
    const int jcol = 2 - d + t;
    if (jcol >= m.nx + r.xe + d + 2) return;
    for (int k = 0; k < d; ++k) {
      int src = r.soundspeed_bottom_quirk ? k : r.bot_src + k;
      a[m.at(jcol, 1 - k)] = (T)(r.sign_bt * (double)a[m.at(jcol, src)]);
    }
    for (int k = 0; k < d; ++k) a[m.at(jcol, m.ny + r.top_dst + k)] = (T)(r.sign_bt * (double)a[m.at(jcol, m.ny + r.top_src - k)]);
  } else {
    const int krow = 2 - d + t;
    if (krow >= m.ny + r.ye + d + 2) return;
    for (int k = 0; k < d; ++k) a[m.at(1 - k, krow)] = (T)(r.sign_lr * (double)a[m.at(r.left_src + k, krow)]);
    for (int k = 0; k < d; ++k) a[m.at(m.nx + r.right_dst + k, krow)] = (T)(r.sign_lr * (double)a[m.at(m.nx + r.right_src - k, krow)]);
  }
}

// ---------------------------------------------------------------------------
// field_summary: src/serial/field_summary.cpp:44-104 -- ideal_gas on level 0
// (writing pressure and soundspeed as the reference does), then the five
// sums.  Per-cell terms are formed exactly as the reference forms them; the
// sums are FP64 block partials, reduced by the last block in block order, so
// the result does not depend on scheduling.
template <typename T>
__global__ void k_field_summary(Fields<T> F, Mesh<T> m, T gm1, double *partials, unsigned int *counter, double *out,
                                int tiles_x, int ntiles) {
  double s[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const int i = 2 + (t % tiles_x) * blockDim.x + threadIdx.x;
    const int j = 2 + (t / tiles_x) * blockDim.y + threadIdx.y;
    if (i >= m.nx + 2 || j >= m.ny + 2) continue;
    const long long id = m.at(i, j);
    const T d0 = F.f[DENSITY0][id], e0 = F.f[ENERGY0][id];
    T p, c;
    eos(d0, e0, gm1, p, c);
    F.f[PRESSURE][id] = p;
    F.f[SOUNDSPEED][id] = c;
    const T *u = F.f[XVEL0], *v = F.f[YVEL0];
    double vsqrd = 0.0;
    for (int kv = j; kv <= j + 1; ++kv)
      for (int jv = i; jv <= i + 1; ++jv) {
        const double uu = u[m.at(jv, kv)], vv = v[m.at(jv, kv)];
        vsqrd += 0.25 * (uu * uu + vv * vv);
      }
    const double cell_vol = m.celldx[i] * m.celldy[j];
    const double cell_mass = cell_vol * (double)d0;
    s[0] += cell_vol;
    s[1] += cell_mass;
    s[2] += cell_mass * (double)e0;
    s[3] += cell_mass * 0.5 * vsqrd;
    s[4] += cell_vol * (double)p;
  }
  // block reduction (fixed tree order)
  __shared__ double red[5][256];
  const int tid = threadIdx.y * blockDim.x + threadIdx.x;
  const int nt = blockDim.x * blockDim.y;
  for (int q = 0; q < 5; ++q) red[q][tid] = s[q];
  __syncthreads();
  for (int w = nt / 2; w > 0; w >>= 1) {
    if (tid < w)
      for (int q = 0; q < 5; ++q) red[q][tid] += red[q][tid + w];
    __syncthreads();
  }
  const unsigned int nb = gridDim.x;
  const unsigned int b = blockIdx.x;
  __shared__ bool last;
  if (tid == 0) {
    for (int q = 0; q < 5; ++q) partials[(size_t)q * nb + b] = red[q][0];
    __threadfence();
    last = atomicAdd(counter, 1u) == nb - 1;
  }
  __syncthreads();
  if (!last) return;
  __threadfence();
  // the last block sums the partials: each thread a strided slice, then a tree
  for (int q = 0; q < 5; ++q) {
    double acc = 0.0;
    for (unsigned int p = tid; p < nb; p += nt) acc += ((volatile double *)partials)[(size_t)q * nb + p];
    red[q][tid] = acc;
  }
  __syncthreads();
  for (int w = nt / 2; w > 0; w >>= 1) {
    if (tid < w)
      for (int q = 0; q < 5; ++q) red[q][tid] += red[q][tid + w];
    __syncthreads();
  }
  if (tid == 0) {
    for (int q = 0; q < 5; ++q) out[q] = red[q][0];
    *counter = 0u;
  }
}

} // namespace cb
