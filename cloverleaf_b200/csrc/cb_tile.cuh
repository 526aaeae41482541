// cb_tile.cuh -- the stencil phases as TMA-tiled kernels.
//
// Every kernel here stages the halo-padded tiles of its input fields into
// shared memory with bulk tensor copies (cb_tma.cuh), computes its outputs
// from shared memory, keeps the phase's intermediate work arrays (pre_vol,
// fluxes, node masses, momentum fluxes) in shared memory, and writes its
// outputs with coalesced stores -- folding in the reflective halo the next
// update_halo would write, on blocks that touch the mesh edge.
//
// Block: 64 x 4 threads.  Tile: 64 columns (x) x TY rows (y); thread (tx, ty)
// owns column x0 + tx and rows y0 + ty + 4r.  Staged element (i, j) sits at
// box[(j - y0 + HALO) * BOX_X + (i - x0 + HALO)].
//
// All arithmetic keeps the reference's expression order (the cited
// src/serial/NAME.cpp lines); FP64 builds without contraction are
// bit-identical to the reference serial model.
#pragma once

#include "cb_mesh.cuh"
#include "cb_ops.h"
#include "cb_tma.cuh"

namespace cb {

template <int TY> struct Tile {
  static constexpr int BH = TY + 2 * HALO;
  static constexpr int BOX = BOX_X * BH; // elements per staged field
  static constexpr int RPT = TY / 4;     // rows per thread
};

// Global element offset of (i, j) from a field's logical origin.
__device__ __forceinline__ int gidx(int pitch, int i, int j) { return j * pitch + i; }

// True when the block's tile lies within 10 cells of a mesh edge, where
// the halo fold may have something to write.
__device__ __forceinline__ bool edge_tile(int nx, int ny, int x0, int y0, int ty) {
  return x0 < 12 || x0 + TILE_X > nx - 8 || y0 < 12 || y0 + ty > ny - 8;
}

// Re-armable staging for blocks that loop over several tiles: the barrier
// is initialised once (init) and completes one phase per tile.
template <typename T>
__device__ __forceinline__ bool stage_loop(T *sm, const Maps &maps, int nf, int box_elems, int off, int x0, int y0, uint64_t *bar,
                                           unsigned phase, bool init, int *err) {
  const bool leader = threadIdx.x == 0 && threadIdx.y == 0;
  if (init && leader) mbar_init(bar, 1);
  __syncthreads(); // the previous tile's readers are done with the boxes
  if (leader) {
    mbar_expect_tx(bar, (unsigned)(nf * box_elems * sizeof(T)));
    for (int f = 0; f < nf; ++f) tma_load_2d(sm + f * box_elems, &maps.m[f], off + x0 - HALO, y0 - HALO, bar);
  }
  bool ok = mbar_wait(bar, phase, err);
  if (!ok) mbar_wait(bar, phase, nullptr);
  return __syncthreads_and(ok) != 0;
}

// ---------------------------------------------------------------------------
// viscosity: src/serial/viscosity.cpp:30-68 (diry quirk at :57 kept).
template <typename T>
__device__ __forceinline__ T viscosity_value(T u00, T u10, T u01, T u11, T v00, T v10, T v01, T v11, T p_l, T p_r, T p_b, T p_t,
                                             T density0, T cdx, T cdx1, T cdy, T cdy2) {
  T ugrad = (u10 + u11) - (u00 + u01);
  T vgrad = (v01 + v11) - (v00 + v10);
  T div = (cdx * (ugrad) + cdy * (vgrad));
  T strain2 = (T(0.5) * (u01 + u11 - u00 - u10)) / (cdy) + (T(0.5) * (v10 + v11 - v00 - v01)) / (cdx);
  T pgradx = (p_r - p_l) / (cdx + cdx1);
  T pgrady = (p_t - p_b) / (cdy + cdy2);
  T pgradx2 = pgradx * pgradx;
  T pgrady2 = pgrady * pgrady;
  T limiter = (((T(0.5) * (ugrad)) / (cdx)) * pgradx2 + ((T(0.5) * (vgrad)) / (cdy)) * pgrady2 + strain2 * pgradx * pgrady) / (fmax(pgradx2 + pgrady2, T(g_small)));
  if ((limiter > T(0.0)) || (div >= T(0.0))) return T(0.0);
  T dirx = T(1.0);
  if (pgradx < T(0.0)) dirx = T(-1.0);
  pgradx = dirx * fmax(T(g_small), fabs(pgradx));
  T diry = T(1.0);
  if (pgradx < T(0.0)) diry = T(-1.0);
  pgrady = diry * fmax(T(g_small), fabs(pgrady));
  T pgrad = sqrt(pgradx * pgradx + pgrady * pgrady);
  T xgrad = fabs((cdx * pgrad) / (pgradx));
  T ygrad = fabs((cdy * pgrad) / (pgrady));
  T grad = fmin(xgrad, ygrad);
  T grad2 = grad * grad;
  return T(2.0) * density0 * grad2 * limiter * limiter;
}

// fields: 0 pressure, 1 density0, 2 xvel0, 3 yvel0
template <typename T>
__global__ void __launch_bounds__(256) kt_viscosity(const __grid_constant__ Maps maps, T *q_out, Mesh<T> m, int off, int fold, int *err) {
  constexpr int TY = 16;
  using C = Tile<TY>;
  extern __shared__ __align__(128) unsigned char smraw[];
  __shared__ uint64_t bar;
  T *sm = reinterpret_cast<T *>(smraw);
  const int x0 = 2 + blockIdx.x * TILE_X, y0 = 2 + blockIdx.y * TY;
  if (!stage_tiles(sm, maps, 4, C::BOX, off, x0, y0, &bar, err)) return;
  const T *P = sm, *R = sm + C::BOX, *U = sm + 2 * C::BOX, *V = sm + 3 * C::BOX;
  const int i = x0 + threadIdx.x, lx = HALO + threadIdx.x;
  if (i >= m.nx + 2) return;
  const bool do_fold = fold && edge_tile(m.nx, m.ny, x0, y0, TY);
  const HaloRule rule = halo_rule(VISCOSITY);
  const T cdx = m.celldx_t[i], cdx1 = m.celldx_t[i + 1];
  const int pitch = (int)m.pitch;
#pragma unroll
  for (int r = 0; r < C::RPT; ++r) {
    const int j = y0 + threadIdx.y + 4 * r, ly = HALO + threadIdx.y + 4 * r;
    if (j >= m.ny + 2) break;
    const int b = ly * BOX_X + lx;
    T q = viscosity_value(U[b], U[b + 1], U[b + BOX_X], U[b + BOX_X + 1], V[b], V[b + 1], V[b + BOX_X], V[b + BOX_X + 1], P[b - 1],
                          P[b + 1], P[b - BOX_X], P[b + BOX_X], R[b], cdx, cdx1, m.celldy_t[j], m.celldy_t[j + 2]);
    q_out[gidx(pitch, i, j)] = q;
    if (do_fold) fold_halo(q_out, m, rule, fold, i, j, q);
  }
}

// ---------------------------------------------------------------------------
// calc_dt: src/serial/calc_dt.cpp:30-79.  Blocks loop over tiles; each
// keeps the minimum of its cells and folds it into the result once.
// fields: 0 soundspeed, 1 viscosity, 2 density0, 3 xvel0, 4 yvel0
template <typename T>
__device__ __forceinline__ T dt_value(T ss, T q, T d0, T u00, T u10, T u01, T u11, T v00, T v10, T v01, T v11, T dsx, T dsy,
                                      const DtConsts &k) {
  const T vol = dsx * dsy;        // volume(i, j) = dx * dy
  const T xa0 = dsy, xa1 = dsy;   // xarea(i, j), xarea(i+1, j) = celldy[j]
  const T ya0 = dsx, ya1 = dsx;   // yarea(i, j), yarea(i, j+1) = celldx[i]
  T cc = ss * ss;
  cc = cc + (T(2.0) * q) / (d0);
  cc = fmax(sqrt(cc), T(g_small));
  T dtct = (T(k.dtc_safe) * fmin(dsx, dsy)) / (cc);
  T div = T(0.0);
  T dv1 = (u00 + u01) * xa0;
  T dv2 = (u10 + u11) * xa1;
  div = div + dv2 - dv1;
  T dtut = (T(k.dtu_safe) * T(2.0) * vol) / (fmax(fmax(fabs(dv1), fabs(dv2)), T(g_small) * vol));
  dv1 = (v00 + v10) * ya0;
  dv2 = (v01 + v11) * ya1;
  div = div + dv2 - dv1;
  T dtvt = (T(k.dtv_safe) * T(2.0) * vol) / (fmax(fmax(fabs(dv1), fabs(dv2)), T(g_small) * vol));
  div = (div) / (T(2.0) * vol);
  T dtdivt;
  if (div < T(-g_small)) {
    dtdivt = T(k.dtdiv_safe) * ((T(-1.0)) / (div));
  } else {
    dtdivt = T(g_big);
  }
  return fmin(dtct, fmin(dtut, fmin(dtvt, fmin(dtdivt, T(g_big)))));
}

template <typename T>
__global__ void __launch_bounds__(256) kt_calc_dt(const __grid_constant__ Maps maps, Mesh<T> m, int off, DtConsts k, int tiles_x,
                                                  int ntiles, unsigned long long *dt_bits, int *err) {
  constexpr int TY = 16;
  using C = Tile<TY>;
  extern __shared__ __align__(128) unsigned char smraw[];
  __shared__ uint64_t bar;
  T *sm = reinterpret_cast<T *>(smraw);
  const T *S = sm, *Q = sm + C::BOX, *R = sm + 2 * C::BOX, *U = sm + 3 * C::BOX, *V = sm + 4 * C::BOX;
  double vmin = g_big;
  unsigned phase = 0;
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x, phase ^= 1u) {
    const int x0 = 2 + (t % tiles_x) * TILE_X, y0 = 2 + (t / tiles_x) * TY;
    if (!stage_loop(sm, maps, 5, C::BOX, off, x0, y0, &bar, phase, t == (int)blockIdx.x, err)) return;
    const int i = x0 + threadIdx.x, lx = HALO + threadIdx.x;
    if (i < m.nx + 2) {
      const T dsx = m.celldx_t[i];
#pragma unroll
      for (int r = 0; r < C::RPT; ++r) {
        const int j = y0 + threadIdx.y + 4 * r, ly = HALO + threadIdx.y + 4 * r;
        if (j >= m.ny + 2) break;
        const int b = ly * BOX_X + lx;
        const double c = (double)dt_value(S[b], Q[b], R[b], U[b], U[b + 1], U[b + BOX_X], U[b + BOX_X + 1], V[b], V[b + 1],
                                          V[b + BOX_X], V[b + BOX_X + 1], dsx, m.celldy_t[j], k);
        vmin = fmin(c, vmin); // fmin drops a NaN candidate, as the reference's fmin does
      }
    }
  }
  block_min_to(vmin, dt_bits);
}

// ---------------------------------------------------------------------------
// PdV: src/serial/PdV.cpp:36-87; mode 1 also does the predictor's
// ideal_gas, pressure halo and revert (:92-133) in the same pass.
// fields: 0 density0, 1 energy0, 2 pressure, 3 viscosity, 4 xvel0, 5 yvel0, [6 xvel1, 7 yvel1]
template <typename T>
__device__ __forceinline__ void pdv_value(bool predict, T dt, T xa, T ya, T vol, T u00, T u01, T u10, T u11, T v00, T v10, T v01, T v11,
                                          T w00, T w01, T w10, T w11, T z00, T z10, T z01, T z11, T d0, T e0, T p, T q, T &density1,
                                          T &energy1) {
  const T xa_l = xa, xa_r = xa, ya_b = ya, ya_t = ya;
  T left_flux, right_flux, bottom_flux, top_flux;
  if (predict) {
    left_flux = (xa_l * (u00 + u01 + u00 + u01)) * T(0.25) * dt * T(0.5);
    right_flux = (xa_r * (u10 + u11 + u10 + u11)) * T(0.25) * dt * T(0.5);
    bottom_flux = (ya_b * (v00 + v10 + v00 + v10)) * T(0.25) * dt * T(0.5);
    top_flux = (ya_t * (v01 + v11 + v01 + v11)) * T(0.25) * dt * T(0.5);
  } else {
    left_flux = (xa_l * (u00 + u01 + w00 + w01)) * T(0.25) * dt;
    right_flux = (xa_r * (u10 + u11 + w10 + w11)) * T(0.25) * dt;
    bottom_flux = (ya_b * (v00 + v10 + z00 + z10)) * T(0.25) * dt;
    top_flux = (ya_t * (v01 + v11 + z01 + z11)) * T(0.25) * dt;
  }
  T total_flux = right_flux - left_flux + top_flux - bottom_flux;
  T volume_change_s = (vol) / (vol + total_flux);
  T recip_volume = (T(1.0)) / (vol);
  T energy_change = ((p) / (d0) + (q) / (d0)) * total_flux * recip_volume;
  energy1 = e0 - energy_change;
  density1 = d0 * volume_change_s;
}

template <typename T>
__device__ __forceinline__ void eos_value(T density, T energy, T gm1, T &pressure, T &soundspeed) {
  T v = (T(1.0)) / (density);
  pressure = gm1 * density * energy;
  T pressurebyenergy = gm1 * density;
  T pressurebyvolume = -density * pressure;
  T sound_speed_squared = v * v * (pressure * pressurebyenergy - pressurebyvolume);
  soundspeed = sqrt(sound_speed_squared);
}

struct PdvOut {
  void *density1, *energy1, *pressure, *soundspeed;
};

template <typename T>
__global__ void __launch_bounds__(256) kt_pdv(const __grid_constant__ Maps maps, PdvOut out, Mesh<T> m, int off, int predict, T dt,
                                              int mode, T gm1, int fold, int *err) {
  constexpr int TY = 8;
  using C = Tile<TY>;
  extern __shared__ __align__(128) unsigned char smraw[];
  __shared__ uint64_t bar;
  T *sm = reinterpret_cast<T *>(smraw);
  const int x0 = 2 + blockIdx.x * TILE_X, y0 = 2 + blockIdx.y * TY;
  const int nf = predict ? 6 : 8;
  if (!stage_tiles(sm, maps, nf, C::BOX, off, x0, y0, &bar, err)) return;
  const T *D0 = sm, *E0 = sm + C::BOX, *P = sm + 2 * C::BOX, *Q = sm + 3 * C::BOX, *U0 = sm + 4 * C::BOX, *V0 = sm + 5 * C::BOX;
  const T *U1 = sm + 6 * C::BOX, *V1 = sm + 7 * C::BOX;
  const int i = x0 + threadIdx.x, lx = HALO + threadIdx.x;
  if (i >= m.nx + 2) return;
  const bool do_fold = fold && edge_tile(m.nx, m.ny, x0, y0, TY);
  const int pitch = (int)m.pitch;
  const T cdx = m.celldx_t[i];
#pragma unroll
  for (int r = 0; r < C::RPT; ++r) {
    const int j = y0 + threadIdx.y + 4 * r, ly = HALO + threadIdx.y + 4 * r;
    if (j >= m.ny + 2) break;
    const int b = ly * BOX_X + lx;
    const T cdy = m.celldy_t[j];
    const T vol = cdx * cdy;
    T w00 = T(0), w01 = T(0), w10 = T(0), w11 = T(0), z00 = T(0), z10 = T(0), z01 = T(0), z11 = T(0);
    if (!predict) {
      w00 = U1[b], w01 = U1[b + BOX_X], w10 = U1[b + 1], w11 = U1[b + BOX_X + 1];
      z00 = V1[b], z10 = V1[b + 1], z01 = V1[b + BOX_X], z11 = V1[b + BOX_X + 1];
    }
    T d1, e1;
    pdv_value(predict != 0, dt, cdy, cdx, vol, U0[b], U0[b + BOX_X], U0[b + 1], U0[b + BOX_X + 1], V0[b], V0[b + 1], V0[b + BOX_X],
              V0[b + BOX_X + 1], w00, w01, w10, w11, z00, z10, z01, z11, D0[b], E0[b], P[b], Q[b], d1, e1);
    const int g = gidx(pitch, i, j);
    if (mode == 0) {
      ((T *)out.density1)[g] = d1;
      ((T *)out.energy1)[g] = e1;
      if (do_fold) {
        fold_halo((T *)out.density1, m, halo_rule(DENSITY1), fold, i, j, d1);
        fold_halo((T *)out.energy1, m, halo_rule(ENERGY1), fold, i, j, e1);
      }
    } else {
      T p, c;
      eos_value(d1, e1, gm1, p, c);
      ((T *)out.pressure)[g] = p;
      ((T *)out.soundspeed)[g] = c;
      if (do_fold) fold_halo((T *)out.pressure, m, halo_rule(PRESSURE), fold, i, j, p);
      ((T *)out.density1)[g] = D0[b];
      ((T *)out.energy1)[g] = E0[b];
    }
  }
}

// ---------------------------------------------------------------------------
// accelerate: src/serial/accelerate.cpp:28-56, nodes [2, nx+2] x [2, ny+2].
// fields: 0 density0, 1 pressure, 2 viscosity, 3 xvel0, 4 yvel0
template <typename T>
__global__ void __launch_bounds__(256) kt_accelerate(const __grid_constant__ Maps maps, T *u_out, T *v_out, Mesh<T> m, int off, T dt,
                                                     int fold, int *err) {
  constexpr int TY = 16;
  using C = Tile<TY>;
  extern __shared__ __align__(128) unsigned char smraw[];
  __shared__ uint64_t bar;
  T *sm = reinterpret_cast<T *>(smraw);
  const int x0 = 2 + blockIdx.x * TILE_X, y0 = 2 + blockIdx.y * TY;
  if (!stage_tiles(sm, maps, 5, C::BOX, off, x0, y0, &bar, err)) return;
  const T *D0 = sm, *P = sm + C::BOX, *Q = sm + 2 * C::BOX, *U0 = sm + 3 * C::BOX, *V0 = sm + 4 * C::BOX;
  const int i = x0 + threadIdx.x, lx = HALO + threadIdx.x;
  if (i >= m.nx + 3) return;
  const bool do_fold = fold && edge_tile(m.nx, m.ny, x0, y0, TY);
  const int pitch = (int)m.pitch;
  const T halfdt = T(0.5) * dt;
  const T cdx = m.celldx_t[i], cdxm = m.celldx_t[i - 1];
#pragma unroll
  for (int r = 0; r < C::RPT; ++r) {
    const int j = y0 + threadIdx.y + 4 * r, ly = HALO + threadIdx.y + 4 * r;
    if (j >= m.ny + 3) break;
    const int b = ly * BOX_X + lx;
    const T cdy = m.celldy_t[j], cdym = m.celldy_t[j - 1];
    const T vol_mm = cdxm * cdym, vol_m0 = cdxm * cdy, vol_00 = cdx * cdy, vol_0m = cdx * cdym;
    const int c00 = b, cm0 = b - 1, c0m = b - BOX_X, cmm = b - BOX_X - 1;
    T stepbymass_s = (halfdt) / (((D0[cmm] * vol_mm + D0[cm0] * vol_m0 + D0[c00] * vol_00 + D0[c0m] * vol_0m) * T(0.25)));
    const T xa = cdy, xa_m = cdym; // xarea(i, j), xarea(i, j-1)
    const T ya = cdx, ya_m = cdxm; // yarea(i, j), yarea(i-1, j)
    T u = U0[c00] - stepbymass_s * (xa * (P[c00] - P[cm0]) + xa_m * (P[c0m] - P[cmm]));
    T v = V0[c00] - stepbymass_s * (ya * (P[c00] - P[c0m]) + ya_m * (P[cm0] - P[cmm]));
    u = u - stepbymass_s * (xa * (Q[c00] - Q[cm0]) + xa_m * (Q[c0m] - Q[cmm]));
    v = v - stepbymass_s * (ya * (Q[c00] - Q[c0m]) + ya_m * (Q[cm0] - Q[cmm]));
    const int g = gidx(pitch, i, j);
    u_out[g] = u;
    v_out[g] = v;
    if (do_fold) {
      fold_halo(u_out, m, halo_rule(XVEL1), fold, i, j, u);
      fold_halo(v_out, m, halo_rule(YVEL1), fold, i, j, v);
    }
  }
}

// ---------------------------------------------------------------------------
// flux_calc: src/serial/flux_calc.cpp:27-43, faces [2, nx+2] x [2, ny+2].
// With a fold, the extra row of x faces and column of y faces (overwritten
// by update_halo) take their halo values.
// fields: 0 xvel0, 1 yvel0, 2 xvel1, 3 yvel1
template <typename T>
__global__ void __launch_bounds__(256) kt_flux_calc(const __grid_constant__ Maps maps, T *fx_out, T *fy_out, Mesh<T> m, int off, T dt,
                                                    int fold, int *err) {
  constexpr int TY = 16;
  using C = Tile<TY>;
  extern __shared__ __align__(128) unsigned char smraw[];
  __shared__ uint64_t bar;
  T *sm = reinterpret_cast<T *>(smraw);
  const int x0 = 2 + blockIdx.x * TILE_X, y0 = 2 + blockIdx.y * TY;
  if (!stage_tiles(sm, maps, 4, C::BOX, off, x0, y0, &bar, err)) return;
  const T *U0 = sm, *V0 = sm + C::BOX, *U1 = sm + 2 * C::BOX, *V1 = sm + 3 * C::BOX;
  const int i = x0 + threadIdx.x, lx = HALO + threadIdx.x;
  if (i >= m.nx + 3) return;
  const bool do_fold = fold && edge_tile(m.nx, m.ny, x0, y0, TY);
  const int pitch = (int)m.pitch;
  const T cdx = m.celldx_t[i];
#pragma unroll
  for (int r = 0; r < C::RPT; ++r) {
    const int j = y0 + threadIdx.y + 4 * r, ly = HALO + threadIdx.y + 4 * r;
    if (j >= m.ny + 3) break;
    const int b = ly * BOX_X + lx;
    T fx = T(0.25) * dt * m.celldy_t[j] * (U0[b] + U0[b + BOX_X] + U1[b] + U1[b + BOX_X]);
    T fy = T(0.25) * dt * cdx * (V0[b] + V0[b + 1] + V1[b] + V1[b + 1]);
    const int g = gidx(pitch, i, j);
    if (!fold) {
      fx_out[g] = fx;
      fy_out[g] = fy;
      continue;
    }
    if (j < m.ny + 2) {
      fx_out[g] = fx;
      if (do_fold) fold_halo(fx_out, m, halo_rule(VOL_FLUX_X), fold, i, j, fx);
    }
    if (i < m.nx + 2) {
      fy_out[g] = fy;
      if (do_fold) fold_halo(fy_out, m, halo_rule(VOL_FLUX_Y), fold, i, j, fy);
    }
  }
}

// ---------------------------------------------------------------------------
// advec_cell: src/serial/advec_cell.cpp:28-220, one sweep in one pass.
// pre_vol of the cells the faces need, then the face fluxes, then the
// update, all through shared memory.  TY = 8.
// fields: 0 density1, 1 energy1, 2 vol_flux_x, 3 vol_flux_y
template <typename T>
__device__ __forceinline__ T cell_limiter_value(T sigma, T sigma3, T sigma4, T diffuw, T diffdw) {
  const T one_by_six = T(1.0 / 6.0);
  T wind = T(1.0);
  if (diffdw <= T(0.0)) wind = T(-1.0);
  if (diffuw * diffdw > T(0.0)) {
    return (T(1.0) - sigma) * wind * fmin(fmin(fabs(diffuw), fabs(diffdw)), one_by_six * (sigma3 * fabs(diffuw) + sigma4 * fabs(diffdw)));
  }
  return T(0.0);
}

struct CellOut {
  void *density1, *energy1, *mass_flux;
};

// Shared layout of the cell sweep beyond the staged boxes.
template <int DIR> struct CellShared {
  static constexpr int TY = 8;
  // pre_vol: DIR 1: rows TY x cells [x0-2, x0+66); DIR 2: rows [y0-2, y0+TY+2) x 64 columns
  static constexpr int PV_W = DIR == 1 ? TILE_X + 4 : TILE_X, PV_H = DIR == 1 ? TY : TY + 4;
  // fluxes: DIR 1: TY rows x 65 faces; DIR 2: TY+1 face rows x 64 columns
  static constexpr int F_W = DIR == 1 ? TILE_X + 1 : TILE_X, F_H = DIR == 1 ? TY : TY + 1;
};

template <typename T, int DIR>
__global__ void __launch_bounds__(256) kt_advec_cell(const __grid_constant__ Maps maps, CellOut out, Mesh<T> m, int off, int sweep,
                                                     int fold, int *err) {
  using L = CellShared<DIR>;
  constexpr int TY = L::TY;
  using C = Tile<TY>;
  extern __shared__ __align__(128) unsigned char smraw[];
  __shared__ uint64_t bar;
  T *sm = reinterpret_cast<T *>(smraw);
  double *s_mf = reinterpret_cast<double *>(smraw + 4 * C::BOX * sizeof(T));
  double *s_ef = s_mf + L::F_W * L::F_H;
  T *s_pv = reinterpret_cast<T *>(s_ef + L::F_W * L::F_H);
  const int x0 = 2 + blockIdx.x * TILE_X, y0 = 2 + blockIdx.y * TY;
  const int nf = (sweep == 1) ? 4 : (DIR == 1 ? 3 : 4); // sweep 2 of x needs no y fluxes
  if (!stage_tiles(sm, maps, nf, C::BOX, off, x0, y0, &bar, err)) return;
  const T *D1 = sm, *E1 = sm + C::BOX, *VFX = sm + 2 * C::BOX, *VFY = sm + 3 * C::BOX;
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int na = DIR == 1 ? m.nx : m.ny;
  const int pitch = (int)m.pitch;
  // (1) pre_vol (advec_cell.cpp:42-61 / :134-153) of the cells the sweep touches
  for (int py = ty; py < L::PV_H; py += 4)
    for (int px = tx; px < L::PV_W; px += 64) {
      const int i = DIR == 1 ? x0 - 2 + px : x0 + px;
      const int j = DIR == 1 ? y0 + py : y0 - 2 + py;
      if (i > m.nx + 3 || j > m.ny + 3) continue;
      const int b = (j - y0 + HALO) * BOX_X + (i - x0 + HALO);
      const T vol = m.celldx_t[i] * m.celldy_t[j];
      T pv;
      if (DIR == 1) {
        pv = sweep == 1 ? vol + (VFX[b + 1] - VFX[b] + VFY[b + BOX_X] - VFY[b]) : vol + VFX[b + 1] - VFX[b];
      } else {
        pv = sweep == 1 ? vol + (VFY[b + BOX_X] - VFY[b] + VFX[b + 1] - VFX[b]) : vol + VFY[b + BOX_X] - VFY[b];
      }
      s_pv[py * L::PV_W + px] = pv;
    }
  __syncthreads();
  // (2) face fluxes (:63-113 / :155-205), faces [x0, x0+64] or [y0, y0+TY]
  const double *vdx = DIR == 1 ? m.vertexdx : m.vertexdy;
  for (int fy = ty; fy < L::F_H; fy += 4)
    for (int fx = tx; fx < L::F_W; fx += 64) {
      const int i = x0 + fx, j = y0 + fy;         // face (i, j)
      const int f = DIR == 1 ? i : j;             // position along the sweep
      if (i > (DIR == 1 ? m.nx + 3 : m.nx + 1) || j > (DIR == 1 ? m.ny + 1 : m.ny + 3)) continue;
      const int b = (j - y0 + HALO) * BOX_X + (i - x0 + HALO);
      const int step = DIR == 1 ? 1 : BOX_X;      // box stride along the sweep
      const T flux = DIR == 1 ? VFX[b] : VFY[b];
      int upwind, donor, downwind, dif;
      if (flux > T(0.0)) {
        upwind = f - 2; donor = f - 1; downwind = f; dif = donor;
      } else {
        upwind = (f + 1 < na + 2) ? f + 1 : na + 2;
        donor = f; downwind = f - 1; dif = upwind;
      }
      const int bd = b + (donor - f) * step, bu = b + (upwind - f) * step, bw = b + (downwind - f) * step;
      const T pre_vol_d = DIR == 1 ? s_pv[fy * L::PV_W + (donor - (x0 - 2))] : s_pv[(donor - (y0 - 2)) * L::PV_W + fx];
      T sigmat = (fabs(flux)) / (pre_vol_d);
      T sigma3 = (T(1.0) + sigmat) * (T)((vdx[f]) / (vdx[dif]));
      T sigma4 = T(2.0) - sigmat;
      T sigmav = sigmat;
      const T dd = D1[bd], du = D1[bu], dw = D1[bw];
      T limiter = cell_limiter_value(sigmav, sigma3, sigma4, dd - du, dw - dd);
      T mass_flux = flux * (dd + limiter);
      T sigmam = (fabs(mass_flux)) / ((dd * pre_vol_d));
      const T ed = E1[bd], eu = E1[bu], ew = E1[bw];
      limiter = cell_limiter_value(sigmam, sigma3, sigma4, ed - eu, ew - ed);
      s_mf[fy * L::F_W + fx] = (double)mass_flux;
      s_ef[fy * L::F_W + fx] = (double)mass_flux * (double)(ed + limiter);
      T *mf = (T *)out.mass_flux;
      const bool halo_face = fold && f == na + 3; // with a fold, face na+3 takes its halo value
      if (!halo_face) mf[gidx(pitch, i, j)] = mass_flux;
      if (fold && f < na + 3 && edge_tile(m.nx, m.ny, x0, y0, TY))
        fold_halo(mf, m, halo_rule(DIR == 1 ? MASS_FLUX_X : MASS_FLUX_Y), fold, i, j, mass_flux);
    }
  __syncthreads();
  // (3) the update (:117-129 / :209-221), mass/energy accumulation in FP64
  const int i = x0 + tx;
  if (i >= m.nx + 2) return;
  const bool do_fold = fold && edge_tile(m.nx, m.ny, x0, y0, TY);
#pragma unroll
  for (int r = 0; r < C::RPT; ++r) {
    const int j = y0 + ty + 4 * r, ly = HALO + ty + 4 * r;
    if (j >= m.ny + 2) break;
    const int b = ly * BOX_X + HALO + tx;
    const int fy = ty + 4 * r;
    const T pre_vol = DIR == 1 ? s_pv[fy * L::PV_W + tx + 2] : s_pv[(fy + 2) * L::PV_W + tx];
    const double mf_lo = DIR == 1 ? s_mf[fy * L::F_W + tx] : s_mf[fy * L::F_W + tx];
    const double mf_hi = DIR == 1 ? s_mf[fy * L::F_W + tx + 1] : s_mf[(fy + 1) * L::F_W + tx];
    const double ef_lo = DIR == 1 ? s_ef[fy * L::F_W + tx] : s_ef[fy * L::F_W + tx];
    const double ef_hi = DIR == 1 ? s_ef[fy * L::F_W + tx + 1] : s_ef[(fy + 1) * L::F_W + tx];
    const T vf_lo = DIR == 1 ? VFX[b] : VFY[b];
    const T vf_hi = DIR == 1 ? VFX[b + 1] : VFY[b + BOX_X];
    double pre_mass_s = (double)D1[b] * (double)pre_vol;
    double post_mass_s = pre_mass_s + mf_lo - mf_hi;
    double post_ener_s = ((double)E1[b] * pre_mass_s + ef_lo - ef_hi) / (post_mass_s);
    double advec_vol_s = (double)pre_vol + (double)vf_lo - (double)vf_hi;
    const T dnew = (T)((post_mass_s) / (advec_vol_s));
    const T enew = (T)post_ener_s;
    const int g = gidx(pitch, i, j);
    ((T *)out.density1)[g] = dnew;
    ((T *)out.energy1)[g] = enew;
    if (do_fold) {
      fold_halo((T *)out.density1, m, halo_rule(DENSITY1), fold, i, j, dnew);
      fold_halo((T *)out.energy1, m, halo_rule(ENERGY1), fold, i, j, enew);
    }
  }
}

template <typename T, int DIR> constexpr size_t cell_smem_bytes() {
  using L = CellShared<DIR>;
  return 4 * Tile<L::TY>::BOX * sizeof(T) + 2 * L::F_W * L::F_H * sizeof(double) + L::PV_W * L::PV_H * sizeof(T);
}

// ---------------------------------------------------------------------------
// advec_mom: src/serial/advec_mom.cpp:30-225, both velocities in one pass.
// Positions p along the sweep map to nodes a = a0 - 2 + p (two extra nodes
// on each side feed the fluxes of the updated ones).  TY = 8.
// fields: 0 density1, 1 mass flux of the sweep, 2 xvel1, 3 yvel1, [4 the
// other-direction volume flux, for post_vol of sweep 1]
template <typename T>
__device__ __forceinline__ T mom_limiter_value(T vdiffuw, T vdiffdw, T sigma, T width, T dx_dif) {
  T limiter = T(0.0);
  if (vdiffuw * vdiffdw > T(0.0)) {
    T auw = fabs(vdiffuw);
    T adw = fabs(vdiffdw);
    T wind = T(1.0);
    if (vdiffdw <= T(0.0)) wind = T(-1.0);
    limiter = wind * fmin(fmin((width * (((T(2.0) - sigma) * adw) / (width) + ((T(1.0) + sigma) * auw) / (dx_dif))) / (T(6.0)), auw), adw);
  }
  return limiter;
}

struct MomOut {
  void *xvel1, *yvel1;
};

template <int DIR> struct MomShared {
  static constexpr int TY = 8;
  // positions along the sweep x lines across
  static constexpr int NP = DIR == 1 ? TILE_X + 4 : TY + 4; // node positions along the sweep
  static constexpr int NL = DIR == 1 ? TY : TILE_X;         // lines
  static constexpr int N = NP * NL;
};

template <typename T, int DIR>
__global__ void __launch_bounds__(256) kt_advec_mom(const __grid_constant__ Maps maps, MomOut out, Mesh<T> m, int off, int vel_mask,
                                                    int sweep, int fold, int *err) {
  using L = MomShared<DIR>;
  constexpr int TY = L::TY, NP = L::NP, NL = L::NL;
  using C = Tile<TY>;
  extern __shared__ __align__(128) unsigned char smraw[];
  __shared__ uint64_t bar;
  T *sm = reinterpret_cast<T *>(smraw);
  T *s_nf = sm + 5 * C::BOX, *s_nmpre = s_nf + L::N, *s_nmpost = s_nmpre + L::N, *s_mfu = s_nmpost + L::N, *s_mfv = s_mfu + L::N;
  // shared index of (position p, line l): the fastest thread index walks the contiguous dimension
  auto sidx = [](int p, int l) { return DIR == 1 ? l * NP + p : p * NL + l; };
  const int mom_sweep = DIR + 2 * (sweep - 1);
  const int x0 = 2 + blockIdx.x * TILE_X, y0 = 2 + blockIdx.y * TY;
  const int nf = mom_sweep <= 2 ? 5 : 4;
  if (!stage_tiles(sm, maps, nf, C::BOX, off, x0, y0, &bar, err)) return;
  const T *D1 = sm, *MF = sm + C::BOX, *U1 = sm + 2 * C::BOX, *V1 = sm + 3 * C::BOX, *VFO = sm + 4 * C::BOX;
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int na = DIR == 1 ? m.nx : m.ny, nlmax = DIR == 1 ? m.ny : m.nx;
  const int a0 = DIR == 1 ? x0 : y0;
  const int pitch = (int)m.pitch;
  const int ST = DIR == 1 ? 1 : BOX_X; // box stride along the sweep
  const int SL = DIR == 1 ? BOX_X : 1; // box stride across
  // the thread's (position, line) walk: DIR 1 -> p along x (tx), l = rows (ty); DIR 2 -> p along y (ty), l = columns (tx)
  const int p_start = DIR == 1 ? tx : ty, p_step = DIR == 1 ? 64 : 4;
  const int l_start = DIR == 1 ? ty : tx, l_step = DIR == 1 ? 4 : 64;
  auto box_of = [&](int a, int line) { // box index of node (a along the sweep, line across)
    return DIR == 1 ? (line - y0 + HALO) * BOX_X + (a - x0 + HALO) : (a - y0 + HALO) * BOX_X + (line - x0 + HALO);
  };
  // post_vol of cell c = box index b (:42-77): mom_sweep 1 vol + vfy diff, 2 vol + vfx diff, 3/4 vol
  auto post_vol = [&](int b, int ci, int cj) -> T {
    const T vol = m.celldx_t[ci] * m.celldy_t[cj];
    if (mom_sweep == 1) return vol + VFO[b + BOX_X] - VFO[b];
    if (mom_sweep == 2) return vol + VFO[b + 1] - VFO[b];
    return vol;
  };
  // (1) node_flux over nodes [0, na+3] (:84-88 / :156-160)
  for (int l = l_start; l < NL; l += l_step) {
    const int line = (DIR == 1 ? y0 : x0) + l;
    for (int p = p_start; p < NP; p += p_step) {
      const int a = a0 - 2 + p;
      T nf = T(0.0);
      if (line < nlmax + 3 && a >= 0 && a <= na + 3) {
        const int b = box_of(a, line);
        // dir 1: mf(a, j-1) + mf(a, j) + mf(a+1, j-1) + mf(a+1, j); dir 2: mf(i-1, a) + mf(i, a) + mf(i-1, a+1) + mf(i, a+1)
        nf = T(0.25) * (MF[b - SL] + MF[b] + MF[b + ST - SL] + MF[b + ST]);
      }
      s_nf[sidx(p, l)] = nf;
    }
  }
  __syncthreads();
  // (2) node_mass_post / node_mass_pre over nodes [1, na+3] (:93-102 / :165-174)
  for (int l = l_start; l < NL; l += l_step) {
    const int line = (DIR == 1 ? y0 : x0) + l;
    for (int p = p_start; p < NP; p += p_step) {
      const int a = a0 - 2 + p;
      T nmpost = T(1.0), nmpre = T(1.0);
      if (line < nlmax + 3 && p >= 1 && a >= 1 && a <= na + 3) {
        const int i = DIR == 1 ? a : line, j = DIR == 1 ? line : a;
        const int b = box_of(a, line); // node (i, j) = cell (i, j) in the box
        nmpost = T(0.25) * (D1[b - BOX_X] * post_vol(b - BOX_X, i, j - 1) + D1[b] * post_vol(b, i, j) +
                            D1[b - BOX_X - 1] * post_vol(b - BOX_X - 1, i - 1, j - 1) + D1[b - 1] * post_vol(b - 1, i - 1, j));
        nmpre = nmpost - s_nf[sidx(p - 1, l)] + s_nf[sidx(p, l)];
      }
      s_nmpost[sidx(p, l)] = nmpost;
      s_nmpre[sidx(p, l)] = nmpre;
    }
  }
  __syncthreads();
  // (3) mom_flux over nodes [1, na+2] (:108-133 / :180-205): positions [1, NP-2]
  const T *celld = DIR == 1 ? m.celldx_t : m.celldy_t;
  for (int l = l_start; l < NL; l += l_step) {
    const int line = (DIR == 1 ? y0 : x0) + l;
    for (int p = p_start; p < NP; p += p_step) {
      const int a = a0 - 2 + p;
      if (p < 1 || p > NP - 2 || line >= nlmax + 3 || a < 1 || a > na + 2) continue;
      const T nf = s_nf[sidx(p, l)];
      int upwind, donor, downwind, dif;
      if (nf < T(0.0)) {
        upwind = a + 2; donor = a + 1; downwind = a; dif = donor;
      } else {
        upwind = a - 1; donor = a; downwind = a + 1; dif = upwind;
      }
      const T sigma = (fabs(nf)) / (s_nmpre[sidx(p + (donor - a), l)]);
      const T width = celld[a];
      const int b = box_of(a, line);
      const int bd = b + (donor - a) * ST, bu = b + (upwind - a) * ST, bw = b + (downwind - a) * ST;
      if (vel_mask & 1) {
        const T vd = U1[bd];
        T lim = mom_limiter_value(vd - U1[bu], U1[bw] - vd, sigma, width, celld[dif]);
        s_mfu[sidx(p, l)] = (vd + (T(1.0) - sigma) * lim) * nf;
      }
      if (vel_mask & 2) {
        const T vd = V1[bd];
        T lim = mom_limiter_value(vd - V1[bu], V1[bw] - vd, sigma, width, celld[dif]);
        s_mfv[sidx(p, l)] = (vd + (T(1.0) - sigma) * lim) * nf;
      }
    }
  }
  __syncthreads();
  // (4) velocity update over nodes [2, na+2] (:139-144 / :211-216): positions [2, NP-2)
  const bool do_fold = fold && edge_tile(m.nx, m.ny, x0, y0, TY);
  for (int l = l_start; l < NL; l += l_step) {
    const int line = (DIR == 1 ? y0 : x0) + l;
    for (int p = p_start; p < NP; p += p_step) {
      const int a = a0 - 2 + p;
      if (p < 2 || p >= NP - 2 || line >= nlmax + 3 || a > na + 2) continue;
      const int i = DIR == 1 ? a : line, j = DIR == 1 ? line : a;
      const int b = box_of(a, line);
      const T nmpre = s_nmpre[sidx(p, l)], nmpost = s_nmpost[sidx(p, l)];
      const int g = gidx(pitch, i, j);
      if (vel_mask & 1) {
        T v = (U1[b] * nmpre + s_mfu[sidx(p - 1, l)] - s_mfu[sidx(p, l)]) / (nmpost);
        ((T *)out.xvel1)[g] = v;
        if (do_fold) fold_halo((T *)out.xvel1, m, halo_rule(XVEL1), fold, i, j, v);
      }
      if (vel_mask & 2) {
        T v = (V1[b] * nmpre + s_mfv[sidx(p - 1, l)] - s_mfv[sidx(p, l)]) / (nmpost);
        ((T *)out.yvel1)[g] = v;
        if (do_fold) fold_halo((T *)out.yvel1, m, halo_rule(YVEL1), fold, i, j, v);
      }
    }
  }
}

template <typename T, int DIR> constexpr size_t mom_smem_bytes() {
  using L = MomShared<DIR>;
  return (5 * Tile<L::TY>::BOX + 5 * L::N) * sizeof(T);
}

} // namespace cb
