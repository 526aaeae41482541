// cb_sweep.cuh -- one x sweep of the advection in one pass: advec_cell then
// advec_mom of both velocities (src/serial/advec_cell.cpp:28-220 and
// src/serial/advec_mom.cpp:30-225, direction 1), for the tiles away from the
// mesh edge (edge_tile false); the existing one-phase kernels run the tiles
// of the edge strip (kt_advec_cell_edges / kt_advec_mom_edges below).
//
// A tile of 64 x TY nodes updates its cells' density and energy and its
// nodes' velocities.  The momentum update of a node needs the new density
// (as cell mass) of the cells x0-2 .. x0+64 and the mass fluxes of the faces
// x0-2 .. x0+65, on the rows y0-1 .. y0+TY-1; those faces need the staged
// density and energy of the cells x0-4 .. x0+66.  The tile evaluates that
// ring itself from the staged level-1 state -- the same value functions as
// the one-phase kernels, so the values are those the separate passes would
// store and reread -- and writes only its own cells, faces and nodes.  As a
// first sweep the one-phase kernels move 14 arrays (7 each); this pass reads
// density1, energy1, vol_flux_x, vol_flux_y, xvel1, yvel1 and writes
// density1, energy1, mass_flux_x, xvel1, yvel1: 11.  As a second sweep
// writing level 0 (the resident loop) it moves 11 where they move 13.
//
// Outputs are double-buffered like the one-phase kernels' (the caller swaps):
// other tiles still read the old level-1 state of their rings.  With the
// level-0 outputs set the pass also does reset_field's copy of what it
// writes (interior tiles fold nothing).
#pragma once

#include "cb_tile.cuh"

namespace cb {

template <typename T, int TY> struct SweepXLayout {
  static constexpr int BH = TY + 2; // staged rows y0 - 1 .. y0 + TY
  static constexpr int BOXS = (BOX_X * BH * (int)sizeof(T) + 127) / 128 * 128 / (int)sizeof(T);
  static constexpr int NFACE = TILE_X + 4; // faces x0 - 2 .. x0 + 65
  static constexpr int NCELL = TILE_X + 3; // cells x0 - 2 .. x0 + 64; nodes x0 - 2 .. x0 + 64
  static constexpr int NLC = TY + 1;       // cell and face lines y0 - 1 .. y0 + TY - 1
  static constexpr int NLN = TY;           // node lines y0 .. y0 + TY - 1
  // work arrays after the six boxes: the faces' mass and energy fluxes in
  // FP64 (the momentum fluxes, storage type, reuse their space), then the
  // cell masses and node fluxes (storage type)
  static constexpr int FACES = 2 * NLC * NFACE;     // doubles
  static constexpr int CM = NLC * NCELL, NF = NLN * NCELL; // storage type
  static_assert(2 * NLN * NCELL * (int)sizeof(T) <= FACES * (int)sizeof(double), "the momentum fluxes fit the face fluxes' space");
  static constexpr size_t FACE_OFF = (size_t)6 * BOXS * sizeof(T);
  static constexpr size_t CM_OFF = FACE_OFF + (size_t)FACES * sizeof(double);
  static constexpr size_t GEO_OFF = (CM_OFF + (size_t)(CM + NF) * sizeof(T) + 15) / 16 * 16;
  // then the widths: the x vertex widths and their reciprocals (FP64), celldx, celldy (storage type)
  static constexpr size_t SMEM = GEO_OFF + (size_t)2 * BOX_X * sizeof(double) + (size_t)(BOX_X + BH) * sizeof(T);
};

struct SweepOut {
  CellOut cell; // density1 / energy1 (spares), mass_flux_x, level 0 when set
  MomOut mom;   // xvel1 / yvel1 (spares, or null for level 0 only), level 0 when set
  // when set: the mass flux is stored by the tiles on the border of the
  // interior rectangle (the edge strip's momentum tiles read it), and by the
  // others only if *store_mf is nonzero (the resident loop's last step: the
  // pass's own momentum update takes it from shared memory, and the next
  // sweep in x rewrites it unread)
  const int *store_mf = nullptr;
};

// The interior tile (bx, by) of the x sweep; staged: ms 0 density1,
// 1 energy1, 2 vol_flux_x, 3 vol_flux_y (sweep 1), 4 xvel1, 5 yvel1.
template <typename T, int TY>
__device__ __forceinline__ void sweep_x_tile(TileCtx &cx, T *sm, const Maps &maps, const SweepOut &out, const Mesh<T> &m, int off,
                                             int sweep, int bx, int by) {
  using L = SweepXLayout<T, TY>;
  constexpr int NFACE = L::NFACE, NCELL = L::NCELL, NLC = L::NLC, NLN = L::NLN;
  const int x0 = 2 + bx * TILE_X, y0 = 2 + by * TY;
  const T *D1 = sm, *E1 = sm + L::BOXS, *VFX = sm + 2 * L::BOXS, *VFY = sm + 3 * L::BOXS, *U1 = sm + 4 * L::BOXS,
          *V1 = sm + 5 * L::BOXS;
  char *raw = reinterpret_cast<char *>(sm);
  double *s_mf = reinterpret_cast<double *>(raw + L::FACE_OFF), *s_ef = s_mf + NLC * NFACE;
  T *s_mfu = reinterpret_cast<T *>(s_mf), *s_mfv = s_mfu + NLN * NCELL; // once the face fluxes are dead
  T *s_cm = reinterpret_cast<T *>(raw + L::CM_OFF), *s_nf = s_cm + L::CM;
  double *g_vd = reinterpret_cast<double *>(raw + L::GEO_OFF), *g_rvd = g_vd + BOX_X;
  T *g_x = reinterpret_cast<T *>(g_rvd + BOX_X), *g_y = g_x + BOX_X;
  // staging: density1, energy1, vol_flux_x, [vol_flux_y], then the velocities
  {
    const MapSet ms = map_set(maps, 6);
    const bool leader = threadIdx.x == 0 && threadIdx.y == 0;
    if (cx.fresh && leader) mbar_init(cx.bar, 1);
    __syncthreads();
    if (leader) {
      const int nb = sweep == 1 ? 6 : 5;
      mbar_expect_tx(cx.bar, (unsigned)(nb * BOX_X * L::BH * sizeof(T)));
      const int xs = off + x0 - HALO, ys = y0 - 1;
      for (int f = 0; f < 6; ++f)
        if (f != 3 || sweep == 1) tma_load_2d(sm + f * L::BOXS, ms.m[f], xs, ys, cx.bar);
    }
    fill_widths(m, x0, y0, 1, L::BH, 1, g_x, g_y, g_vd, g_rvd);
    if (!stage_wait(cx)) return;
  }
  const int pitch = (int)m.pitch;
  auto bidx = [&](int i, int j) { return (j - y0 + 1) * BOX_X + (i - x0 + HALO); };
  auto pre_vol_of = [&](int i, int j) -> T {
    const int b = bidx(i, j);
    const T vol = g_x[i - x0 + HALO] * g_y[j - y0 + 1];
    return sweep == 1 ? cell_pre_vol1(vol, VFX[b], VFX[b + 1], VFY[b], VFY[b + BOX_X]) : cell_pre_vol2(vol, VFX[b], VFX[b + 1]);
  };
  const bool border = blockIdx.x == 0 || blockIdx.x == gridDim.x - 1 || blockIdx.y == 0 || blockIdx.y == gridDim.y - 1;
  const bool store_mf = border || !out.store_mf || *out.store_mf != 0;
  // (A) face fluxes (advec_cell.cpp:63-113), faces x0-2+p on lines y0-1+l
  Items<1, NFACE, NLC>::each([&](int, int p, int l) {
    const int f = x0 - 2 + p, j = y0 - 1 + l;
    const int b = bidx(f, j);
    const T flux = VFX[b];
    int upwind, donor, downwind, dif;
    if (flux > T(0.0)) {
      upwind = f - 2; donor = f - 1; downwind = f; dif = donor;
    } else {
      upwind = f + 1; donor = f; downwind = f - 1; dif = upwind;
    }
    const int bd = b + (donor - f), bu = b + (upwind - f), bw = b + (downwind - f);
    T ratio;
    if constexpr (sizeof(T) == sizeof(double))
      ratio = width_ratio(g_vd[f - x0 + HALO], g_vd[dif - x0 + HALO], g_rvd[dif - x0 + HALO]);
    else
      ratio = lim_div((T)g_vd[f - x0 + HALO], (T)g_vd[dif - x0 + HALO]);
    T mass_flux, e_adv;
    cell_face_value(flux, pre_vol_of(donor, j), ratio, D1[bd], D1[bu], D1[bw], E1[bd], E1[bu], E1[bw], mass_flux, e_adv);
    s_mf[l * NFACE + p] = (double)mass_flux;
    s_ef[l * NFACE + p] = (double)mass_flux * (double)e_adv; // FP32: the exact product
    if (store_mf && p >= 2 && p < TILE_X + 2 && l >= 1) ((T *)out.cell.mass_flux)[gidx(pitch, f, j)] = mass_flux;
  });
  __syncthreads();
  // (B) the cell update (advec_cell.cpp:117-129) on cells x0-2+p, lines y0-1+l,
  // with each cell's mass density1 * post_vol (advec_mom.cpp:42-77, :93-96)
  Items<1, NCELL, NLC>::each([&](int, int p, int l) {
    const int i = x0 - 2 + p, j = y0 - 1 + l;
    const int b = bidx(i, j);
    const T pre_vol = pre_vol_of(i, j);
    const double mf_lo = s_mf[l * NFACE + p], mf_hi = s_mf[l * NFACE + p + 1];
    const double ef_lo = s_ef[l * NFACE + p], ef_hi = s_ef[l * NFACE + p + 1];
    const T vf_lo = VFX[b], vf_hi = VFX[b + 1];
    T dnew, enew;
    if constexpr (sizeof(T) == sizeof(double)) {
      double dn, en;
      cell_update_value<double>(D1[b], E1[b], pre_vol, mf_lo, mf_hi, ef_lo, ef_hi, vf_lo, vf_hi, dn, en);
      dnew = (T)dn;
      enew = (T)en;
    } else {
      double pre_mass_s = (double)D1[b] * (double)pre_vol;
      double post_mass_s = pre_mass_s + mf_lo - mf_hi;
      double ener_s = (double)E1[b] * pre_mass_s + ef_lo - ef_hi;
      double advec_vol_s = (double)pre_vol + (double)vf_lo - (double)vf_hi;
      dnew = (T)post_mass_s / (T)advec_vol_s;
      enew = (T)ener_s / (T)post_mass_s;
    }
    if (p >= 2 && p < TILE_X + 2 && l >= 1) {
      const int g = gidx(pitch, i, j);
      ((T *)out.cell.density1)[g] = dnew;
      if (out.cell.energy1) ((T *)out.cell.energy1)[g] = enew;
      if (out.cell.density0) {
        ((T *)out.cell.density0)[g] = dnew;
        ((T *)out.cell.energy0)[g] = enew;
      }
    }
    const T vol = g_x[i - x0 + HALO] * g_y[j - y0 + 1];
    const T pv = sweep == 1 ? mom_post_vol(1, vol, VFY[b], VFY[b + BOX_X]) : vol; // mom_sweep 1 or 3
    s_cm[l * NCELL + p] = dnew * pv;
  });
  // (C) node fluxes (advec_mom.cpp:84-88) on nodes x0-2+p, lines y0+l
  Items<1, NCELL, NLN>::each([&](int, int p, int l) {
    s_nf[l * NCELL + p] = quarter_sum((T)s_mf[l * NFACE + p], (T)s_mf[(l + 1) * NFACE + p], (T)s_mf[l * NFACE + p + 1],
                                      (T)s_mf[(l + 1) * NFACE + p + 1]);
  });
  __syncthreads();
  auto cm = [&](int p, int lc) -> T { return s_cm[lc * NCELL + p]; };
  auto nf = [&](int p, int l) -> T { return s_nf[l * NCELL + p]; };
  // node_mass_post (:93-96) of node (p, l): cells (i, j-1), (i, j), (i-1, j-1), (i-1, j)
  auto node_mass_post = [&](int p, int l) -> T { return quarter_sum(cm(p, l), cm(p, l + 1), cm(p - 1, l), cm(p - 1, l + 1)); };
  // (D) momentum fluxes (:108-133) on nodes x0-2+p, p = 1 .. 65
  const T *celld = g_x + HALO - x0; // celldx of column i at celld[i]
  Items<1, TILE_X + 1, NLN>::each([&](int, int q, int l) {
    const int p = q + 1;
    const int a = x0 - 2 + p, j = y0 + l;
    const T nfv = nf(p, l);
    int upwind, donor, downwind, dif;
    if (nfv < T(0.0)) {
      upwind = a + 2; donor = a + 1; downwind = a; dif = donor;
    } else {
      upwind = a - 1; donor = a; downwind = a + 1; dif = upwind;
    }
    const int pd = p + (donor - a);
    const T sigma = mom_sigma(nfv, mom_node_mass_pre(node_mass_post(pd, l), nf(pd - 1, l), nf(pd, l)));
    const T width = celld[a], dxd = celld[dif];
    const int b = bidx(a, j);
    const int bd = b + (donor - a), bu = b + (upwind - a), bw = b + (downwind - a);
    s_mfu[l * NCELL + p] = mom_flux_value(sigma, nfv, width, dxd, U1[bd], U1[bu], U1[bw]);
    s_mfv[l * NCELL + p] = mom_flux_value(sigma, nfv, width, dxd, V1[bd], V1[bu], V1[bw]);
  });
  __syncthreads();
  // (E) velocity update (:139-144) on the tile's nodes x0 .. x0+63
  Items<1, TILE_X, NLN>::each([&](int, int q, int l) {
    const int p = q + 2;
    const int i = x0 + q, j = y0 + l;
    const int b = bidx(i, j);
    const T nmpost = node_mass_post(p, l), nmpre = mom_node_mass_pre(nmpost, nf(p - 1, l), nf(p, l));
    const T u = mom_update_value(U1[b], nmpre, nmpost, s_mfu[l * NCELL + p - 1], s_mfu[l * NCELL + p]);
    const T v = mom_update_value(V1[b], nmpre, nmpost, s_mfv[l * NCELL + p - 1], s_mfv[l * NCELL + p]);
    const int g = gidx(pitch, i, j);
    if (out.mom.xvel1) {
      ((T *)out.mom.xvel1)[g] = u;
      ((T *)out.mom.yvel1)[g] = v;
    }
    if (out.mom.xvel0) {
      ((T *)out.mom.xvel0)[g] = u;
      ((T *)out.mom.yvel0)[g] = v;
    }
  });
}

template <typename T, int TY>
__global__ void __launch_bounds__(256) kt_advec_sweep_x(const __grid_constant__ Maps maps, SweepOut out, Mesh<T> m, int off, int sweep,
                                                        int bx0, int by0, int *err) {
  extern __shared__ __align__(128) unsigned char smraw[];
  __shared__ uint64_t bar;
  TileCtx cx = tile_ctx(&bar, err);
  sweep_x_tile<T, TY>(cx, reinterpret_cast<T *>(smraw), maps, out, m, off, sweep, bx0 + blockIdx.x, by0 + blockIdx.y);
}

// The tiles of a tx x ty grid outside the interior rectangle [bx_lo, bx_hi] x
// [by_lo, by_hi]: the rows below, the rows above, then the two side strips
// of the rows in between.
struct EdgeSet {
  int tx, ty, bx_lo, bx_hi, by_lo, by_hi;
  __host__ __device__ int count() const { return tx * ty - (bx_hi - bx_lo + 1) * (by_hi - by_lo + 1); }
  __device__ void tile(int k, int &bx, int &by) const {
    const int nb = by_lo * tx;
    if (k < nb) {
      bx = k % tx, by = k / tx;
      return;
    }
    k -= nb;
    const int nt = (ty - 1 - by_hi) * tx;
    if (k < nt) {
      bx = k % tx, by = by_hi + 1 + k / tx;
      return;
    }
    k -= nt;
    const int left = bx_lo, per = left + (tx - 1 - bx_hi);
    by = by_lo + k / per;
    const int c = k % per;
    bx = c < left ? c : bx_hi + 1 + (c - left);
  }
};

template <typename T, int DIR, int TY>
__global__ void __launch_bounds__(256, cell_min_blocks<T>()) kt_advec_cell_edges(const __grid_constant__ Maps maps, CellOut out, Mesh<T> m,
                                                                                int off, int sweep, int fold, EdgeSet es, int *err) {
  extern __shared__ __align__(128) unsigned char smraw[];
  __shared__ uint64_t bar;
  TileCtx cx = tile_ctx(&bar, err);
  int bx, by;
  es.tile(blockIdx.x, bx, by);
  advec_cell_tile<T, DIR, TY>(cx, reinterpret_cast<T *>(smraw), map_set(maps, 4), out, m, off, sweep, fold, bx, by);
}

template <typename T, int DIR, int TY>
__global__ void __launch_bounds__(256) kt_advec_mom_edges(const __grid_constant__ Maps maps, MomOut out, Mesh<T> m, int off, int vel_mask,
                                                          int sweep, int fold, EdgeSet es, int *err) {
  extern __shared__ __align__(128) unsigned char smraw[];
  __shared__ uint64_t bar;
  TileCtx cx = tile_ctx(&bar, err);
  int bx, by;
  es.tile(blockIdx.x, bx, by);
  advec_mom_tile<T, DIR, TY>(cx, reinterpret_cast<T *>(smraw), map_set(maps, 5), out, m, off, vel_mask, sweep, fold, bx, by);
}

} // namespace cb
