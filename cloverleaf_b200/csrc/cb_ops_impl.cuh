// cb_ops_impl.cuh -- definitions of the phase-kernel launchers (declared in
// cb_ops.h).  Included only by cb_fp64.cu and cb_fp32.cu, which instantiate
// Ops<double> and Ops<float>.
#pragma once

#include <algorithm>
#include <initializer_list>

#include "cb_ops.h"
#include "cb_phase.cuh"
#include "cb_sweep.cuh"
#include "cb_tile.cuh"

namespace cb {

namespace detail {

template <typename T> Fields<T> fields(const Chunk &c) {
  Fields<T> F;
  for (int f = 0; f < NUM_FIELDS; ++f) F.f[f] = f < 15 ? (T *)c.base(f) : nullptr; // work arrays and geometry are not stored
  return F;
}

template <typename T> Mesh<T> mesh(const Chunk &c) {
  Mesh<T> m;
  m.nx = c.nx;
  m.ny = c.ny;
  m.pitch = c.pitch;
  m.celldx = c.geom_d[CELLDX];
  m.celldy = c.geom_d[CELLDY];
  m.vertexdx = c.geom_d[VERTEXDX];
  m.vertexdy = c.geom_d[VERTEXDY];
  m.celldx_t = (const T *)c.geom_t[CELLDX];
  m.celldy_t = (const T *)c.geom_t[CELLDY];
  m.rcelldx = c.rgeom_d;
  m.rcelldy = c.rgeom_d + c.geom_len;
  m.rvertexdx = c.rgeom_d + 2 * c.geom_len;
  m.rvertexdy = c.rgeom_d + 3 * c.geom_len;
  return m;
}

inline dim3 grid2(int w, int h, dim3 b) { return dim3((w + b.x - 1) / b.x, (h + b.y - 1) / b.y); }

// Counts one kernel launch and returns its launch status.
inline cudaError_t launched(Chunk &c) {
  ++c.launches;
  return cudaGetLastError();
}

template <typename T> T gm1(const Chunk &c) { return (T)(c.gamma - 1.0); }

inline int reduce_grid(const Chunk &c, int ntiles) { return std::min(ntiles, c.summary_grid); }

// Copies the ring around the updated rectangle [ilo, ihi] x [jlo, jhi] from
// src to dst for each of the n (1 or 2) pairs (double-buffered phases whose
// halo is not folded).
template <typename T>
cudaError_t copy_ring(Chunk &c, const RingPair &rp, int n, int ilo, int ihi, int jlo, int jhi, int ex, int ey) {
  if (n == 0) return cudaSuccess;
  const long long ring = (long long)ex * ey - (long long)(ihi - ilo + 1) * (jhi - jlo + 1);
  dim3 g((unsigned)((ring + 255) / 256), n);
  k_copy_ring<T><<<g, 256, 0, c.stream>>>(rp, mesh<T>(c), ilo, ihi, jlo, jhi, ex, ey);
  return launched(c);
}

// Tensor maps of the listed fields for staged boxes of H rows.
template <int H> Maps maps_of(const Chunk &c, std::initializer_list<int> fields) {
  Maps mp;
  int k = 0;
  for (int f : fields) mp.m[k++] = *c.map<H>(f);
  return mp;
}

// Raises a kernel's dynamic shared-memory limit (a cheap host-side call).
template <typename K> cudaError_t allow_smem(K kernel, size_t bytes) {
  return cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
}

} // namespace detail

using namespace detail;

template <typename T> cudaError_t Ops<T>::generate_chunk(Chunk &c, const DevState *d_states, int nstates) {
  dim3 b(32, 8);
  k_generate_chunk<T><<<grid2(c.nx + 5, c.ny + 5, b), b, 0, c.stream>>>(fields<T>(c), mesh<T>(c), d_states, nstates, c.geom_d[CELLX],
                                                                        c.geom_d[CELLY], c.geom_d[VERTEXX], c.geom_d[VERTEXY]);
  return launched(c);
}

template <typename T> cudaError_t Ops<T>::ideal_gas(Chunk &c, int predict, int fold) {
  dim3 b(32, 8);
  k_ideal_gas<T><<<grid2((c.nx + Vec16<T>::N - 1) / Vec16<T>::N, c.ny, b), b, 0, c.stream>>>(fields<T>(c), mesh<T>(c), predict, gm1<T>(c), fold);
  return launched(c);
}

template <typename T> cudaError_t Ops<T>::viscosity(Chunk &c, int fold) {
  constexpr int TY = 16;
  using B = Box1<T, TY>;
  const size_t smem = 3 * B::BOXS * sizeof(T);
  cudaError_t e = allow_smem(kt_viscosity<T>, smem);
  if (e != cudaSuccess) return e;
  dim3 g((c.nx + TILE_X - 1) / TILE_X, (c.ny + TY - 1) / TY);
  kt_viscosity<T><<<g, dim3(64, 4), smem, c.stream>>>(maps_of<B::BH>(c, {PRESSURE, XVEL0, YVEL0}), (const T *)c.base(DENSITY0),
                                                      (T *)c.base(VISCOSITY), mesh<T>(c), (int)c.off, fold, c.d_err);
  return launched(c);
}

template <typename T> cudaError_t Ops<T>::calc_dt(Chunk &c, const DtConsts &k) {
  constexpr int TY = 16;
  using B = Box1<T, TY>;
  const size_t smem = (2 * B::BOXS + (sizeof(T) == sizeof(double) ? REST_MEMO_ELEMS : 0)) * sizeof(T);
  cudaError_t e = allow_smem(kt_calc_dt<T>, smem);
  if (e != cudaSuccess) return e;
  const int tx = (c.nx + TILE_X - 1) / TILE_X, ty = (c.ny + TY - 1) / TY, nt = tx * ty;
  int per_sm = 0;
  if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kt_calc_dt<T>, 256, smem)) != cudaSuccess) return e;
  const int grid = std::min(nt, c.sms * std::max(per_sm, 1));
  DtIn in{c.base(SOUNDSPEED), c.base(VISCOSITY), c.base(DENSITY0)};
  kt_calc_dt<T><<<grid, dim3(64, 4), smem, c.stream>>>(maps_of<B::BH>(c, {XVEL0, YVEL0}), in, mesh<T>(c), (int)c.off, k, tx, nt,
                                                       c.d_dt_bits, c.d_err);
  return launched(c);
}

template <typename T> cudaError_t Ops<T>::pdv(Chunk &c, int predict, double dt, int mode, int fold) {
  constexpr int TY = 8;
  using B = Box1<T, TY>;
  const size_t smem = (predict ? 2 : 4) * B::BOXS * sizeof(T);
  // FP64: the four-blocks-per-SM form; FP32: the compiler's register choice
  auto kern = sizeof(T) == sizeof(double) ? kt_pdv4<T> : kt_pdv<T>;
  cudaError_t e = allow_smem(kern, 4 * B::BOXS * sizeof(T));
  if (e != cudaSuccess) return e;
  dim3 g((c.nx + TILE_X - 1) / TILE_X, (c.ny + TY - 1) / TY);
  PdvIn in{c.base(DENSITY0), c.base(ENERGY0), c.base(PRESSURE), c.base(VISCOSITY)};
  PdvOut out{c.base(DENSITY1), c.base(ENERGY1), c.base(PRESSURE), c.base(SOUNDSPEED)};
  Maps mp = maps_of<B::BH>(c, {XVEL0, YVEL0, XVEL1, YVEL1});
  kern<<<g, dim3(64, 4), smem, c.stream>>>(mp, in, out, mesh<T>(c), (int)c.off, predict, (T)dt, c.dt_dev, mode, gm1<T>(c), fold, c.d_err);
  return launched(c);
}

template <typename T> cudaError_t Ops<T>::revert(Chunk &c) {
  dim3 b(32, 8);
  k_revert<T><<<grid2(c.nx, c.ny, b), b, 0, c.stream>>>(fields<T>(c), mesh<T>(c));
  return launched(c);
}

template <typename T> cudaError_t Ops<T>::accelerate(Chunk &c, double dt, int fold) {
  constexpr int TY = 16;
  const size_t smem = acc_smem<T, TY>();
  cudaError_t e = allow_smem(kt_accelerate<T>, smem);
  if (e != cudaSuccess) return e;
  dim3 g((c.nx + 1 + TILE_X - 1) / TILE_X, (c.ny + 1 + TY - 1) / TY);
  kt_accelerate<T><<<g, dim3(64, 4), smem, c.stream>>>(maps_of<Box1<T, TY>::BH>(c, {DENSITY0, PRESSURE, VISCOSITY, XVEL0, YVEL0}),
                                                       (T *)c.base(XVEL1), (T *)c.base(YVEL1), mesh<T>(c), (int)c.off, (T)dt, c.dt_dev,
                                                       fold, c.d_err);
  return launched(c);
}

template <typename T> cudaError_t Ops<T>::flux_calc(Chunk &c, double dt, int fold) {
  constexpr int TY = 16;
  const size_t smem = flux_smem<T, TY>();
  cudaError_t e = allow_smem(kt_flux_calc<T>, smem);
  if (e != cudaSuccess) return e;
  dim3 g((c.nx + 1 + TILE_X - 1) / TILE_X, (c.ny + 1 + TY - 1) / TY);
  kt_flux_calc<T><<<g, dim3(64, 4), smem, c.stream>>>(maps_of<Box1<T, TY>::BH>(c, {XVEL0, YVEL0, XVEL1, YVEL1}), (T *)c.base(VOL_FLUX_X),
                                                      (T *)c.base(VOL_FLUX_Y), mesh<T>(c), (int)c.off, (T)dt, c.dt_dev, fold, c.d_err);
  return launched(c);
}


template <typename T, int DIR, int TY> cudaError_t launch_advec_cell(Chunk &c, int sweep, int fold, void *dd, void *de, int reset_fold) {
  using L = CellLayout<T, DIR, TY>;
  CellOut out{dd, de, c.base(DIR == 1 ? MASS_FLUX_X : MASS_FLUX_Y)};
  if (reset_fold >= 0) {
    out.density0 = c.base(DENSITY0);
    out.energy0 = c.base(ENERGY0);
    out.rfold = reset_fold;
  }
  Maps mp = maps_of<L::BH>(c, {DENSITY1, ENERGY1, VOL_FLUX_X, VOL_FLUX_Y});
  cudaError_t e = allow_smem(kt_advec_cell<T, DIR, TY>, L::SMEM);
  if (e != cudaSuccess) return e;
  dim3 g((c.nx + TILE_X - 1) / TILE_X, (c.ny + TY - 1) / TY);
  kt_advec_cell<T, DIR, TY><<<g, dim3(64, 4), L::SMEM, c.stream>>>(mp, out, mesh<T>(c), (int)c.off, sweep, fold, c.d_err);
  return launched(c);
}

// dir 1 = x, 2 = y.  The updated density/energy go to (dd, de); the caller swaps buffers.
template <typename T> cudaError_t Ops<T>::advec_cell(Chunk &c, int sweep, int dir, int fold, void *dd, void *de, int reset_fold) {
  const T *sd = (const T *)c.base(DENSITY1), *se = (const T *)c.base(ENERGY1);
  cudaError_t e;
  if (!dd) return cudaErrorInvalidValue;
  if (!de) {
    if (reset_fold < 0 || fold != 2) return cudaErrorInvalidValue; // energy to level 0 only, reset_field's copy done
  } else if (fold != 2) { // keep the halo ring exactly as the in-place reference leaves it
    RingPair rp{{sd, se}, {dd, de}};
    if ((e = copy_ring<T>(c, rp, 2, 2, c.nx + 1, 2, c.ny + 1, c.nx + 4, c.ny + 4)) != cudaSuccess) return e;
  }
  return dir == 1 ? launch_advec_cell<T, 1, AdvecTiles<T>::CELL_X>(c, sweep, fold, dd, de, reset_fold)
                  : launch_advec_cell<T, 2, AdvecTiles<T>::CELL_Y>(c, sweep, fold, dd, de, reset_fold);
}


template <typename T, int DIR, int TY>
cudaError_t launch_advec_mom(Chunk &c, int vel_mask, int sweep, int fold, void *du, void *dv, int reset_fold) {
  using L = MomLayout<T, DIR, TY>;
  const int mom_sweep = DIR + 2 * (sweep - 1);
  const int mf = DIR == 1 ? MASS_FLUX_X : MASS_FLUX_Y;
  Maps mp = mom_sweep == 1   ? maps_of<L::BH>(c, {XVEL1, YVEL1, DENSITY1, mf, VOL_FLUX_Y})
            : mom_sweep == 2 ? maps_of<L::BH>(c, {XVEL1, YVEL1, DENSITY1, mf, VOL_FLUX_X})
                             : maps_of<L::BH>(c, {XVEL1, YVEL1, DENSITY1, mf});
  cudaError_t e = allow_smem(kt_advec_mom<T, DIR, TY>, L::SMEM);
  if (e != cudaSuccess) return e;
  // nodes [2, n+2] along both axes: n+1 of them
  dim3 g((c.nx + 1 + TILE_X - 1) / TILE_X, (c.ny + 1 + TY - 1) / TY);
  MomOut out{du, dv};
  if (reset_fold >= 0) {
    out.xvel0 = (vel_mask & 1) ? c.base(XVEL0) : nullptr;
    out.yvel0 = (vel_mask & 2) ? c.base(YVEL0) : nullptr;
    out.rfold = reset_fold;
  }
  kt_advec_mom<T, DIR, TY><<<g, dim3(64, 4), L::SMEM, c.stream>>>(mp, out, mesh<T>(c), (int)c.off, vel_mask, sweep, fold, c.d_err);
  return launched(c);
}

template <typename T>
cudaError_t Ops<T>::advec_mom(Chunk &c, int vel_mask, int sweep, int dir, int fold, void *du, void *dv, int reset_fold) {
  const T *su = (const T *)c.base(XVEL1), *sv = (const T *)c.base(YVEL1);
  cudaError_t e;
  if (!du || !dv) {
    if (reset_fold < 0 || du || dv) return cudaErrorInvalidValue; // level 0 only: both outputs skipped, reset_field's copy done
  } else if (fold != 2) {
    RingPair rp{};
    int n = 0;
    if (vel_mask & 1) rp.src[n] = su, rp.dst[n++] = du;
    if (vel_mask & 2) rp.src[n] = sv, rp.dst[n++] = dv;
    if ((e = copy_ring<T>(c, rp, n, 2, c.nx + 2, 2, c.ny + 2, c.nx + 5, c.ny + 5)) != cudaSuccess) return e;
  }
  return dir == 1 ? launch_advec_mom<T, 1, AdvecTiles<T>::MOM_X>(c, vel_mask, sweep, fold, du, dv, reset_fold)
                  : launch_advec_mom<T, 2, AdvecTiles<T>::MOM_Y>(c, vel_mask, sweep, fold, du, dv, reset_fold);
}

// The interior tiles (edge_tile false) of the advection tile grid with TY
// rows: x0 = 2 + 64 bx >= 12 and x0 + 64 <= nx - 8, likewise in y.
template <int TY> EdgeSet sweep_tiles(const Chunk &c, bool nodes) {
  EdgeSet e;
  e.tx = (c.nx + (nodes ? 1 : 0) + TILE_X - 1) / TILE_X;
  e.ty = (c.ny + (nodes ? 1 : 0) + TY - 1) / TY;
  e.bx_lo = 1;
  e.bx_hi = c.nx >= 74 ? (c.nx - 74) / TILE_X : -1;
  e.by_lo = (10 + TY - 1) / TY;
  e.by_hi = c.ny >= 10 + TY ? (c.ny - 10 - TY) / TY : -1;
  return e;
}

// FP64 only: the FP32 form's advection kernels are issue-bound, and the
// pass's recomputed ring costs more than the reread it saves (measured at
// 7680^2: FP32 step 2.88 -> 3.19 ms with it, FP64 5.26 -> 5.22 ms).
template <typename T> bool Ops<T>::sweep_x_fusable(const Chunk &c) {
  if (sizeof(T) != sizeof(double)) return false;
  constexpr int TY = AdvecTiles<T>::CELL_X;
  const EdgeSet e = sweep_tiles<TY>(c, false);
  return c.can_fold() && e.bx_hi >= e.bx_lo && e.by_hi >= e.by_lo;
}

template <typename T>
cudaError_t Ops<T>::advec_sweep_x(Chunk &c, int sweep, int cell_fold, int mom_fold, int reset_fold, bool level0_only,
                                  const int *store_mf) {
  constexpr int TY = AdvecTiles<T>::CELL_X;
  static_assert(AdvecTiles<T>::MOM_X == TY, "the x sweep's cell and momentum tiles of the same height");
  if (!sweep_x_fusable(c) || cell_fold != 2 || (level0_only && reset_fold < 0)) return cudaErrorNotSupported;
  const EdgeSet ec = sweep_tiles<TY>(c, false), en = sweep_tiles<TY>(c, true);
  void *dd = c.spare_base(0), *de = c.spare_base(1), *du = c.spare_base(2), *dv = c.spare_base(3);
  const int mf = MASS_FLUX_X;
  cudaError_t e;
  if (mom_fold != 2 && !level0_only) { // the velocities' halo ring as the in-place reference leaves it
    RingPair rp{{c.base(XVEL1), c.base(YVEL1)}, {du, dv}};
    if ((e = copy_ring<T>(c, rp, 2, 2, c.nx + 2, 2, c.ny + 2, c.nx + 5, c.ny + 5)) != cudaSuccess) return e;
  }
  SweepOut so;
  so.store_mf = store_mf;
  so.cell = CellOut{dd, level0_only ? nullptr : de, c.base(mf)};
  so.mom = MomOut{level0_only ? nullptr : du, level0_only ? nullptr : dv};
  if (reset_fold >= 0) {
    so.cell.density0 = c.base(DENSITY0);
    so.cell.energy0 = c.base(ENERGY0);
    so.cell.rfold = reset_fold;
    so.mom.xvel0 = c.base(XVEL0);
    so.mom.yvel0 = c.base(YVEL0);
    so.mom.rfold = reset_fold;
  }
  // (1) the interior tiles, one pass
  using SL = SweepXLayout<T, TY>;
  if ((e = allow_smem(kt_advec_sweep_x<T, TY>, SL::SMEM)) != cudaSuccess) return e;
  dim3 gi(ec.bx_hi - ec.bx_lo + 1, ec.by_hi - ec.by_lo + 1);
  kt_advec_sweep_x<T, TY><<<gi, dim3(64, 4), SL::SMEM, c.stream>>>(
      maps_of<SL::BH>(c, {DENSITY1, ENERGY1, VOL_FLUX_X, VOL_FLUX_Y, XVEL1, YVEL1}), so, mesh<T>(c), (int)c.off, sweep, ec.bx_lo, ec.by_lo,
      c.d_err);
  if ((e = launched(c)) != cudaSuccess) return e;
  // (2) the edge strip's cells
  using CL = CellLayout<T, 1, TY>;
  if ((e = allow_smem(kt_advec_cell_edges<T, 1, TY>, CL::SMEM)) != cudaSuccess) return e;
  kt_advec_cell_edges<T, 1, TY><<<ec.count(), dim3(64, 4), CL::SMEM, c.stream>>>(
      maps_of<CL::BH>(c, {DENSITY1, ENERGY1, VOL_FLUX_X, VOL_FLUX_Y}), so.cell, mesh<T>(c), (int)c.off, sweep, cell_fold, ec, c.d_err);
  if ((e = launched(c)) != cudaSuccess) return e;
  // (3) the edge strip's nodes, reading the new density (spare 0) as the
  // swapped buffer map will hold it
  using ML = MomLayout<T, 1, TY>;
  Maps mp = maps_of<ML::BH>(c, {XVEL1, YVEL1, DENSITY1, mf, VOL_FLUX_Y});
  mp.m[2] = c.tmap[c.sbuf[0]][box_slot<ML::BH>()];
  if ((e = allow_smem(kt_advec_mom_edges<T, 1, TY>, ML::SMEM)) != cudaSuccess) return e;
  kt_advec_mom_edges<T, 1, TY><<<en.count(), dim3(64, 4), ML::SMEM, c.stream>>>(mp, so.mom, mesh<T>(c), (int)c.off, 3, sweep, mom_fold, en,
                                                                               c.d_err);
  return launched(c);
}

template <typename T> cudaError_t Ops<T>::restore_level1(Chunk &c, const void *u_ring, const void *v_ring) {
  dim3 b(32, 8);
  k_level1_from_level0<T><<<dim3((c.nx + 1 + 31) / 32, (c.ny + 1 + 7) / 8), b, 0, c.stream>>>(fields<T>(c), mesh<T>(c));
  cudaError_t e = launched(c);
  if (e != cudaSuccess) return e;
  HaloJob job{};
  job.nfields = 1;
  job.field[0] = ENERGY1;
  if ((e = update_halo(c, job, 2)) != cudaSuccess) return e;
  RingPair rp{{u_ring, v_ring}, {c.base(XVEL1), c.base(YVEL1)}};
  return copy_ring<T>(c, rp, 2, 2, c.nx + 2, 2, c.ny + 2, c.nx + 5, c.ny + 5);
}

template <typename T> cudaError_t Ops<T>::reset_field(Chunk &c, int fold) {
  dim3 b(32, 8);
  k_reset_field<T><<<grid2((c.nx + 1 + Vec16<T>::N - 1) / Vec16<T>::N, c.ny + 1, b), b, 0, c.stream>>>(fields<T>(c), mesh<T>(c), fold);
  return launched(c);
}

template <typename T> cudaError_t Ops<T>::update_halo(Chunk &c, const HaloJob &job, int depth) {
  if (job.nfields == 0) return cudaSuccess;
  const int len = std::max(c.nx, c.ny) + 5 + 2 * depth;
  dim3 g((len + 127) / 128, job.nfields);
  for (int pass = 0; pass < 2; ++pass) {
    k_update_halo<T><<<g, 128, 0, c.stream>>>(fields<T>(c), mesh<T>(c), job, depth, pass, c.external_faces);
    cudaError_t e = launched(c);
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

template <typename T> cudaError_t Ops<T>::tile_halo(Chunk &dst, const Chunk &src, int side, const HaloJob &job, int depth) {
  if (job.nfields == 0) return cudaSuccess;
  const int n = std::max(dst.nx, dst.ny) + 2 * depth + 1;
  dim3 g((n * depth + 127) / 128, job.nfields);
  k_tile_halo<T><<<g, 128, 0, dst.stream>>>(fields<T>(dst), mesh<T>(dst), fields<T>(src), mesh<T>(src), job, side, depth);
  return launched(dst);
}

template <typename T> cudaError_t Ops<T>::ig_visc_dt(Chunk &c, const DtConsts &k, int ig_fold, int fold, bool write_ss, bool write_p) {
  constexpr int TY = VISC_TY;
  using B = Box1<T, TY>;
  const size_t smem = (4 * B::BOXS + (sizeof(T) == sizeof(double) ? REST_MEMO_ELEMS : 0)) * sizeof(T);
  cudaError_t e = allow_smem(kt_ig_visc_dt<T>, smem);
  if (e != cudaSuccess) return e;
  const int tx = (c.nx + TILE_X - 1) / TILE_X, ty = (c.ny + TY - 1) / TY, nt = tx * ty;
  int per_sm = 0;
  if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kt_ig_visc_dt<T>, 256, smem)) != cudaSuccess) return e;
  const int grid = std::min(nt, c.sms * std::max(per_sm, 1));
  kt_ig_visc_dt<T><<<grid, dim3(64, 4), smem, c.stream>>>(maps_of<B::BH>(c, {DENSITY0, ENERGY0, XVEL0, YVEL0}),
                                                          write_p ? (T *)c.base(PRESSURE) : nullptr,
                                                          write_ss ? (T *)c.base(SOUNDSPEED) : nullptr, (T *)c.base(VISCOSITY), mesh<T>(c), (int)c.off, k,
                                                          gm1<T>(c), ig_fold, fold, tx, nt, c.d_dt_bits, c.d_err);
  return launched(c);
}

template <typename T>
cudaError_t Ops<T>::lagrange(Chunk &c, void *p_out, double dt, int p_fold, int acc_fold, int pdv_fold, int flux_fold, bool keep_ring,
                             const int *store_ps, bool p_from_de) {
  if (p_fold <= 0 || acc_fold <= 0 || pdv_fold <= 0 || flux_fold <= 0) return cudaErrorInvalidValue;
  if (keep_ring) {
    RingPair rp{{c.base(PRESSURE), nullptr}, {p_out, nullptr}};
    cudaError_t e = copy_ring<T>(c, rp, 1, 1, c.nx + 2, 1, c.ny + 2, c.nx + 4, c.ny + 4);
    if (e != cudaSuccess) return e;
  }
  // Tile rows: the pressure formed from density0 and energy0 (five staged
  // boxes) leaves room for 12 rows at three blocks per SM in FP64 (4.90 ->
  // 4.89 ms a fused step at 7680^2; 16 rows at two blocks: 5.07); with the
  // pressure staged, 8 rows (four blocks per SM).  FP32: 12 rows both ways.
  constexpr int TY = sizeof(T) == sizeof(double) ? 8 : 12, TYP = 12;
  // the nodes and faces reach one column and one row past the cells
  dim3 g((c.nx + 1 + TILE_X - 1) / TILE_X, (c.ny + 1 + TY - 1) / TY);
  const LagOut<T> out{(T *)p_out, (T *)c.base(SOUNDSPEED), (T *)c.base(XVEL1), (T *)c.base(YVEL1), (T *)c.base(DENSITY1),
                      (T *)c.base(ENERGY1), (T *)c.base(VOL_FLUX_X), (T *)c.base(VOL_FLUX_Y), store_ps};
  const LagFolds fd{p_fold, acc_fold, pdv_fold, flux_fold};
  cudaError_t e;
  if (p_from_de) { // the pressure formed from density0 and energy0 (they must agree: the caller's step has run ideal_gas on them)
    using L = LagLayout<T, TYP, true>;
    const dim3 gp((c.nx + 1 + TILE_X - 1) / TILE_X, (c.ny + 1 + TYP - 1) / TYP);
    if ((e = allow_smem(kt_lagrange<T, TYP, true>, L::SMEM)) != cudaSuccess) return e;
    kt_lagrange<T, TYP, true><<<gp, dim3(64, 4), L::SMEM, c.stream>>>(maps_of<L::BH>(c, {XVEL0, YVEL0, DENSITY0, ENERGY0, VISCOSITY}),
                                                                      out, mesh<T>(c), (int)c.off, (T)dt, c.dt_dev, gm1<T>(c), fd, c.d_err);
  } else {
    using L = LagLayout<T, TY>;
    if ((e = allow_smem(kt_lagrange<T, TY>, L::SMEM)) != cudaSuccess) return e;
    kt_lagrange<T, TY><<<g, dim3(64, 4), L::SMEM, c.stream>>>(maps_of<L::BH>(c, {XVEL0, YVEL0, DENSITY0, ENERGY0, PRESSURE, VISCOSITY}),
                                                              out, mesh<T>(c), (int)c.off, (T)dt, c.dt_dev, gm1<T>(c), fd, c.d_err);
  }
  return launched(c);
}

template <typename T> cudaError_t Ops<T>::face_strip(Chunk &c, int side, const StripJob &job, int depth, void *buf, bool pack) {
  if (job.nfields == 0) return cudaSuccess;
  const int n = std::max(c.nx, c.ny) + 2 * depth + 1;
  dim3 g((n * depth + 127) / 128, job.nfields);
  k_face_strip<T><<<g, 128, 0, c.stream>>>(fields<T>(c), mesh<T>(c), job, side, depth, (T *)buf, pack ? 1 : 0);
  return launched(c);
}

template <typename T> cudaError_t Ops<T>::field_summary(Chunk &c, const int *store_ps) {
  dim3 b(32, 8);
  const int tx = (c.nx + 31) / 32, ty = (c.ny + 7) / 8;
  const int nt = tx * ty;
  k_field_summary<T><<<reduce_grid(c, nt), b, 0, c.stream>>>(fields<T>(c), mesh<T>(c), gm1<T>(c), c.d_partials, c.d_counter, c.d_sums,
                                                             tx, nt, store_ps);
  return launched(c);
}

} // namespace cb
