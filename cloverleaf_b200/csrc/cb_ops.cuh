// cb_ops.cuh -- host-side launchers for the phase kernels, templated on the
// storage type.  cb_fp64.cu instantiates Ops<double> (built with
// -fmad=false: bit parity with the reference serial model), cb_fp32.cu
// instantiates Ops<float>.
#pragma once

#include <algorithm>
#include <cstring>
#include <utility>

#include "cb_chunk.h"
#include "cb_phase.cuh"

namespace cb {

template <typename T> struct Ops {
  static Fields<T> fields(const Chunk &c) {
    Fields<T> F;
    for (int f = 0; f < NUM_FIELDS; ++f) F.f[f] = (T *)c.base(f);
    return F;
  }
  static Mesh<T> mesh(const Chunk &c) {
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
    return m;
  }
  static dim3 grid2(int w, int h, dim3 b) { return dim3((w + b.x - 1) / b.x, (h + b.y - 1) / b.y); }
  // Counts one kernel launch and returns its launch status.
  static cudaError_t launched(Chunk &c) {
    ++c.launches;
    return cudaGetLastError();
  }
  static T gm1(const Chunk &c) { return (T)(c.gamma - 1.0); }

  static cudaError_t generate_chunk(Chunk &c, const DevState *d_states, int nstates) {
    dim3 b(32, 8);
    k_generate_chunk<T><<<grid2(c.nx + 5, c.ny + 5, b), b, 0, c.stream>>>(fields(c), mesh(c), d_states, nstates, c.geom_d[CELLX],
                                                                          c.geom_d[CELLY], c.geom_d[VERTEXX], c.geom_d[VERTEXY]);
    return launched(c);
  }

  static cudaError_t ideal_gas(Chunk &c, int predict, int fold) {
    dim3 b(32, 8);
    k_ideal_gas<T><<<grid2(c.nx, c.ny, b), b, 0, c.stream>>>(fields(c), mesh(c), predict, gm1(c), fold);
    return launched(c);
  }

  static cudaError_t viscosity(Chunk &c, int fold) {
    dim3 b(32, 8);
    k_viscosity<T><<<grid2(c.nx, c.ny, b), b, 0, c.stream>>>(fields(c), mesh(c), fold);
    return launched(c);
  }

  static int reduce_grid(const Chunk &c, int ntiles) { return std::min(ntiles, c.summary_grid); }

  static cudaError_t calc_dt(Chunk &c, const DtConsts &k) {
    dim3 b(32, 8);
    const int tx = (c.nx + 31) / 32, ty = (c.ny + 7) / 8;
    const int nt = tx * ty;
    k_calc_dt<T><<<reduce_grid(c, nt), b, 0, c.stream>>>(fields(c), mesh(c), k, c.d_dt_bits, tx, nt);
    return launched(c);
  }

  static cudaError_t pdv(Chunk &c, int predict, double dt, int mode, int fold) {
    dim3 b(32, 8);
    k_pdv<T><<<grid2(c.nx, c.ny, b), b, 0, c.stream>>>(fields(c), mesh(c), predict, (T)dt, mode, gm1(c), fold);
    return launched(c);
  }

  static cudaError_t revert(Chunk &c) {
    dim3 b(32, 8);
    k_revert<T><<<grid2(c.nx, c.ny, b), b, 0, c.stream>>>(fields(c), mesh(c));
    return launched(c);
  }

  static cudaError_t accelerate(Chunk &c, double dt, int fold) {
    dim3 b(32, 8);
    k_accelerate<T><<<grid2(c.nx + 1, c.ny + 1, b), b, 0, c.stream>>>(fields(c), mesh(c), (T)dt, fold);
    return launched(c);
  }

  static cudaError_t flux_calc(Chunk &c, double dt, int fold) {
    dim3 b(32, 8);
    k_flux_calc<T><<<grid2(c.nx + 1, c.ny + 1, b), b, 0, c.stream>>>(fields(c), mesh(c), (T)dt, fold);
    return launched(c);
  }

  // Copies the ring around the updated rectangle from src to dst (for the
  // double-buffered phases when the halo is not folded).
  static cudaError_t copy_ring(Chunk &c, const void *src, void *dst, int ilo, int ihi, int jlo, int jhi, int ex, int ey) {
    const int n = ex * ey;
    k_copy_ring<T><<<(n + 255) / 256, 256, 0, c.stream>>>((const T *)src, (T *)dst, mesh(c), ilo, ihi, jlo, jhi, ex, ey);
    return launched(c);
  }

  // dir 1 = x, 2 = y.  dst buffers are spares 0 and 1; the caller swaps.
  static cudaError_t advec_cell(Chunk &c, int sweep, int dir, int fold, void *dd, void *de) {
    constexpr int BX = 64, BY = 4;
    const int na = dir == 1 ? c.nx : c.ny, nl = dir == 1 ? c.ny : c.nx;
    dim3 g((na + BX - 1) / BX, (nl + BY - 1) / BY);
    const T *sd = (const T *)c.base(DENSITY1), *se = (const T *)c.base(ENERGY1);
    cudaError_t e;
    if (fold != 2) { // keep the halo ring exactly as the in-place reference leaves it
      if ((e = copy_ring(c, sd, dd, 2, c.nx + 1, 2, c.ny + 1, c.nx + 4, c.ny + 4)) != cudaSuccess) return e;
      if ((e = copy_ring(c, se, de, 2, c.nx + 1, 2, c.ny + 1, c.nx + 4, c.ny + 4)) != cudaSuccess) return e;
    }
    k_advec_cell<T, BX, BY><<<g, dim3(BX, BY), 0, c.stream>>>(fields(c), mesh(c), sweep, dir, sd, se, (T *)dd, (T *)de, fold);
    return launched(c);
  }

  static cudaError_t advec_mom(Chunk &c, int vel_mask, int sweep, int dir, int fold, void *du, void *dv) {
    constexpr int BX = 128, BY = 2;
    const int na = dir == 1 ? c.nx : c.ny, nl = dir == 1 ? c.ny : c.nx;
    dim3 g((na + 1 + (BX - 4) - 1) / (BX - 4), (nl + 1 + BY - 1) / BY);
    const T *su = (const T *)c.base(XVEL1), *sv = (const T *)c.base(YVEL1);
    cudaError_t e;
    if (fold != 2) {
      if ((vel_mask & 1) && (e = copy_ring(c, su, du, 2, c.nx + 2, 2, c.ny + 2, c.nx + 5, c.ny + 5)) != cudaSuccess) return e;
      if ((vel_mask & 2) && (e = copy_ring(c, sv, dv, 2, c.nx + 2, 2, c.ny + 2, c.nx + 5, c.ny + 5)) != cudaSuccess) return e;
    }
    k_advec_mom<T, BX, BY><<<g, dim3(BX, BY), 0, c.stream>>>(fields(c), mesh(c), vel_mask, sweep, dir, su, sv, (T *)du, (T *)dv, fold);
    return launched(c);
  }

  static cudaError_t reset_field(Chunk &c, int fold) {
    dim3 b(32, 8);
    k_reset_field<T><<<grid2(c.nx + 1, c.ny + 1, b), b, 0, c.stream>>>(fields(c), mesh(c), fold);
    return launched(c);
  }

  static cudaError_t update_halo(Chunk &c, const HaloJob &job, int depth) {
    if (job.nfields == 0) return cudaSuccess;
    const int len = std::max(c.nx, c.ny) + 5 + 2 * depth;
    dim3 g((len + 127) / 128, job.nfields);
    for (int pass = 0; pass < 2; ++pass) {
      k_update_halo<T><<<g, 128, 0, c.stream>>>(fields(c), mesh(c), job, depth, pass);
      cudaError_t e = launched(c);
      if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
  }

  static cudaError_t field_summary(Chunk &c) {
    dim3 b(32, 8);
    const int tx = (c.nx + 31) / 32, ty = (c.ny + 7) / 8;
    const int nt = tx * ty;
    k_field_summary<T><<<reduce_grid(c, nt), b, 0, c.stream>>>(fields(c), mesh(c), gm1(c), c.d_partials, c.d_counter, c.d_sums, tx, nt);
    return launched(c);
  }
};

} // namespace cb
