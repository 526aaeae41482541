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

#include <limits>

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

// The (p, l) items of a stage of NP positions along a sweep times NL lines
// across it that the calling thread owns, for 256 threads as 64 x 4: the
// coordinate along x (p for the x sweep, DIR = 1; l for the y sweep) on
// threadIdx.x, the other on threadIdx.y + 4 k, and the items past lane 63
// (a few positions or one line) spread over the block's first threads.  A
// thread's main items share one x coordinate, so their addresses differ by
// constants.  f(k, p, l) gets the item's slot k < K, the same for every
// thread's k-th item.
template <int DIR, int NP, int NL> struct Items {
  static constexpr int NA = DIR == 1 ? NP : NL; // along threadIdx.x
  static constexpr int NB = DIR == 1 ? NL : NP; // along threadIdx.y
  static constexpr int KB = (NB + 3) / 4;
  static constexpr int TAIL = NA > 64 ? (NA - 64) * NB : 0;
  static constexpr int KT = (TAIL + 255) / 256;
  static constexpr int K = KB + KT;
  // UNROLL = false keeps the loops as loops: one copy of f's body (for a
  // caller that holds many phases in one kernel and must stay small)
  template <bool UNROLL = true, typename F> __device__ __forceinline__ static void each(F &&f) {
    constexpr int UB = UNROLL ? KB : 1, UT = UNROLL ? KT : 1;
    const int tx = threadIdx.x, ty = threadIdx.y;
    if (NA >= 64 || tx < NA) {
#pragma unroll UB
      for (int kb = 0; kb < KB; ++kb) {
        const int b = ty + 4 * kb;
        if (NB % 4 == 0 || b < NB) {
          if constexpr (DIR == 1)
            f(kb, tx, b);
          else
            f(kb, b, tx);
        }
      }
    }
    if constexpr (TAIL > 0) {
      const int tid = ty * 64 + tx;
#pragma unroll UT
      for (int kt = 0; kt < KT; ++kt) {
        const int t = tid + 256 * kt;
        if (t < TAIL) {
          const int a = 64 + t % (NA - 64), b = t / (NA - 64);
          if constexpr (DIR == 1)
            f(KB + kt, a, b);
          else
            f(KB + kt, b, a);
        }
      }
    }
  }
};

// Staged boxes whose first row is y0 - 1: BH = rows + 2 (a one-row halo
// above and below the tile), stride rounded to 128 bytes.
template <typename T, int TY> struct Box1 {
  static constexpr int BH = TY + 2;
  static constexpr int BOXS = (BOX_X * BH * (int)sizeof(T) + 127) / 128 * 128 / (int)sizeof(T);
  // box index of element (i, j) of the tile at (x0, y0)
  __device__ static constexpr int at(int i, int j, int x0, int y0) { return (j - y0 + 1) * BOX_X + (i - x0 + HALO); }
};

// Map pointers of the fields a tile stages: the tensor maps live in kernel
// parameter space (one-launch kernels) or in global memory (the batch
// kernel); either address is valid for a bulk tensor copy.
struct MapSet {
  const CUtensorMap *m[8];
};

__device__ __forceinline__ MapSet map_set(const Maps &maps, int nf) {
  MapSet s;
#pragma unroll
  for (int f = 0; f < 8; ++f) s.m[f] = f < nf ? &maps.m[f] : nullptr;
  return s;
}

// Staging state of a block: its shared-memory mbarrier, the parity of the
// next completion, and whether the barrier still needs its init.  A
// one-launch kernel stages once; the batch kernel re-arms the same barrier
// for every tile it processes.
struct TileCtx {
  uint64_t *bar;
  unsigned phase;
  bool fresh;
  int *err;
};

__device__ __forceinline__ TileCtx tile_ctx(uint64_t *bar, int *err) { return TileCtx{bar, 0u, true, err}; }

// Stages fields ms.m[0..nf) as boxes of BOX_X x bh elements whose first
// element is tensor coordinate (xs, ys), `stride` elements apart in shared
// memory (stride * sizeof(T) a multiple of 128 bytes).  Called by every
// thread of the block; returns false in every thread if the copies did not
// arrive within the wait limit.
// stage() in two halves, for tiles that fill other shared memory while the
// copies are in flight: stage_issue (every thread; the previous tile's
// readers are done when it returns) and stage_wait (every thread; the boxes
// and whatever the block wrote in between are visible when it returns).
template <typename T>
__device__ __forceinline__ void stage_issue(TileCtx &cx, T *sm, const MapSet &ms, int nf, int stride, int bh, int xs, int ys) {
  const bool leader = threadIdx.x == 0 && threadIdx.y == 0;
  if (cx.fresh && leader) mbar_init(cx.bar, 1);
  __syncthreads(); // barrier initialised; the previous tile's readers are done with the boxes
  if (leader) {
    // the block's generic-proxy accesses to the boxes (reads, and the work
    // arrays some tiles write over them) come before the copies' writes
    if (!cx.fresh) asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    mbar_expect_tx(cx.bar, (unsigned)(nf * BOX_X * bh * sizeof(T)));
    for (int f = 0; f < nf; ++f) tma_load_2d(sm + f * stride, ms.m[f], xs, ys, cx.bar);
  }
}

__device__ __forceinline__ bool stage_wait(TileCtx &cx) {
  bool ok = mbar_wait(cx.bar, cx.phase, cx.err);
  if (!ok) mbar_wait(cx.bar, cx.phase, nullptr); // a second bounded wait for copies still in flight
  cx.phase ^= 1u;
  cx.fresh = false;
  return __syncthreads_and(ok) != 0;
}

template <typename T>
__device__ __forceinline__ bool stage(TileCtx &cx, T *sm, const MapSet &ms, int nf, int stride, int bh, int xs, int ys) {
  stage_issue(cx, sm, ms, nf, stride, bh, xs, ys);
  return stage_wait(cx);
}

// The 1-D widths a tile reads, copied to shared memory while its boxes are
// in flight: gx[k] = celldx of column x0 - HALO + k (BOX_X of them), gy[r] =
// celldy of row y0 - yh + r (bh of them), and -- when gv is given -- the
// sweep direction's vertex widths and their reciprocals, indexed like gx
// (x sweep) or gy (y sweep).  Indices past the arrays' ends are clamped:
// those entries belong to positions no extent check lets through.
template <typename T>
__device__ __forceinline__ void fill_widths(const Mesh<T> &m, int x0, int y0, int yh, int bh, int dir, T *gx, T *gy, double *gv,
                                            double *grv) {
  const int tid = threadIdx.y * 64 + threadIdx.x;
  if (tid < BOX_X) {
    gx[tid] = m.celldx_t[min(max(x0 - HALO + tid, 0), m.nx + 3)];
  } else if (tid < BOX_X + bh) {
    const int r = tid - BOX_X;
    gy[r] = m.celldy_t[min(max(y0 - yh + r, 0), m.ny + 3)];
  } else if (gv && tid >= 128 && tid < 128 + (dir == 1 ? BOX_X : bh)) {
    const int k = tid - 128;
    const int idx = dir == 1 ? min(max(x0 - HALO + k, 0), m.nx + 4) : min(max(y0 - yh + k, 0), m.ny + 4);
    gv[k] = dir == 1 ? m.vertexdx[idx] : m.vertexdy[idx];
    grv[k] = dir == 1 ? m.rvertexdx[idx] : m.rvertexdy[idx];
  }
}

// ---------------------------------------------------------------------------
// viscosity: src/serial/viscosity.cpp:30-68 (diry quirk at :57 kept).  The
// result is 0 whenever div >= 0 (:50), so the divisions are only evaluated
// where the cell is compressed; the value is the same either way.
template <typename T>
__device__ __forceinline__ T viscosity_value(T u00, T u10, T u01, T u11, T v00, T v10, T v01, T v11, T p_l, T p_r, T p_b, T p_t,
                                             T density0, T cdx, T cdx1, T cdy, T cdy2) {
  T ugrad = (u10 + u11) - (u00 + u01);
  T vgrad = (v01 + v11) - (v00 + v10);
  T div = (cdx * (ugrad) + cdy * (vgrad));
  if (div >= T(0.0)) return T(0.0);
  T strain2 = lim_div(T(0.5) * (u01 + u11 - u00 - u10), cdy) + lim_div(T(0.5) * (v10 + v11 - v00 - v01), cdx);
  T pgradx = lim_div(p_r - p_l, cdx + cdx1);
  T pgrady = lim_div(p_t - p_b, cdy + cdy2);
  T pgradx2 = pgradx * pgradx;
  T pgrady2 = pgrady * pgrady;
  T limiter = lim_div(lim_div(T(0.5) * (ugrad), cdx) * pgradx2 + lim_div(T(0.5) * (vgrad), cdy) * pgrady2 + strain2 * pgradx * pgrady,
                      fmax(pgradx2 + pgrady2, T(g_small)));
  if (limiter > T(0.0)) return T(0.0);
  T dirx = T(1.0);
  if (pgradx < T(0.0)) dirx = T(-1.0);
  pgradx = dirx * fmax(T(g_small), fabs(pgradx));
  T diry = T(1.0);
  if (pgradx < T(0.0)) diry = T(-1.0);
  pgrady = diry * fmax(T(g_small), fabs(pgrady));
  T pgrad = sqrt(pgradx * pgradx + pgrady * pgrady);
  T xgrad = fabs(lim_div(cdx * pgrad, pgradx));
  T ygrad = fabs(lim_div(cdy * pgrad, pgrady));
  T grad = fmin(xgrad, ygrad);
  T grad2 = grad * grad;
  return T(2.0) * density0 * grad2 * limiter * limiter;
}

// One viscosity tile (64 x 16 cells at tile coordinates (bx, by)).
// Staged: ms 0 pressure, 1 xvel0, 2 yvel0; density0 is read directly.
constexpr int VISC_TY = 16;
template <typename T> constexpr size_t visc_smem() { return 3 * Box1<T, VISC_TY>::BOXS * sizeof(T); }

template <typename T>
__device__ __forceinline__ bool viscosity_tile(TileCtx &cx, T *sm, const MapSet &ms, const T *d0, T *q_out, const Mesh<T> &m, int off,
                                               int bx, int by, int fold) {
  constexpr int TY = VISC_TY;
  using B = Box1<T, TY>;
  const int x0 = 2 + bx * TILE_X, y0 = 2 + by * TY;
  if (!stage(cx, sm, ms, 3, B::BOXS, B::BH, off + x0 - HALO, y0 - 1)) return false;
  const T *P = sm, *U = sm + B::BOXS, *V = sm + 2 * B::BOXS;
  const int i = x0 + threadIdx.x;
  if (i >= m.nx + 2) return true;
  const bool do_fold = fold && edge_tile(m.nx, m.ny, x0, y0, TY);
  const HaloRule rule = halo_rule(VISCOSITY);
  const T cdx = m.celldx_t[i], cdx1 = m.celldx_t[i + 1];
  const int pitch = (int)m.pitch;
  constexpr int RPT = TY / 4;
  T rho[RPT];
#pragma unroll
  for (int r = 0; r < RPT; ++r) {
    const int j = y0 + threadIdx.y + 4 * r;
    rho[r] = j < m.ny + 2 ? d0[gidx(pitch, i, j)] : T(0);
  }
#pragma unroll
  for (int r = 0; r < RPT; ++r) {
    const int j = y0 + threadIdx.y + 4 * r;
    if (j >= m.ny + 2) break;
    const int b = B::at(i, j, x0, y0);
    T q = viscosity_value(U[b], U[b + 1], U[b + BOX_X], U[b + BOX_X + 1], V[b], V[b + 1], V[b + BOX_X], V[b + BOX_X + 1], P[b - 1],
                          P[b + 1], P[b - BOX_X], P[b + BOX_X], rho[r], cdx, cdx1, m.celldy_t[j], m.celldy_t[j + 2]);
    q_out[gidx(pitch, i, j)] = q;
    if (do_fold) fold_halo(q_out, m, rule, fold, i, j, q);
  }
  return true;
}

template <typename T>
__global__ void __launch_bounds__(256, 4) kt_viscosity(const __grid_constant__ Maps maps, const T *__restrict__ d0, T *q_out, Mesh<T> m, int off,
                                                    int fold, int *err) {
  extern __shared__ __align__(128) unsigned char smraw[];
  __shared__ uint64_t bar;
  TileCtx cx = tile_ctx(&bar, err);
  viscosity_tile(cx, reinterpret_cast<T *>(smraw), map_set(maps, 3), d0, q_out, m, off, blockIdx.x, blockIdx.y, fold);
}

// ---------------------------------------------------------------------------
// calc_dt: src/serial/calc_dt.cpp:30-79.  Blocks loop over tiles; each
// keeps the minimum of its cells and folds it into the result once.
template <typename T>
__device__ __forceinline__ T dt_value(T ss, T q, T d0, T u00, T u10, T u01, T u11, T v00, T v10, T v01, T v11, T dsx, T dsy,
                                      const DtConsts &k) {
  const T vol = dsx * dsy;        // volume(i, j) = dx * dy
  const T xa0 = dsy, xa1 = dsy;   // xarea(i, j), xarea(i+1, j) = celldy[j]
  const T ya0 = dsx, ya1 = dsx;   // yarea(i, j), yarea(i, j+1) = celldx[i]
  T cc = ss * ss;
  cc = cc + lim_div(T(2.0) * q, d0);
  cc = fmax(sqrt(cc), T(g_small));
  T dtct = lim_div(T(k.dtc_safe) * fmin(dsx, dsy), cc);
  T div = T(0.0);
  T dv1 = (u00 + u01) * xa0;
  T dv2 = (u10 + u11) * xa1;
  div = div + dv2 - dv1;
  T dtut = lim_div(T(k.dtu_safe) * T(2.0) * vol, fmax(fmax(fabs(dv1), fabs(dv2)), T(g_small) * vol));
  dv1 = (v00 + v10) * ya0;
  dv2 = (v01 + v11) * ya1;
  div = div + dv2 - dv1;
  T dtvt = lim_div(T(k.dtv_safe) * T(2.0) * vol, fmax(fmax(fabs(dv1), fabs(dv2)), T(g_small) * vol));
  div = lim_div(div, T(2.0) * vol);
  T dtdivt;
  if (div < T(-g_small)) {
    dtdivt = T(k.dtdiv_safe) * lim_div(T(-1.0), div);
  } else {
    dtdivt = T(g_big);
  }
  return fmin(dtct, fmin(dtut, fmin(dtvt, fmin(dtdivt, T(g_big)))));
}

// An estimate of dt_value<double> for the minimum search: the same
// expressions with the quotients (__fdividef) and the square root taken in
// single precision from the double operands.  Error bound, relative to the
// exact value of each term: operands rounded to float 2^-24 each, the
// quotients within 2 ulp (2^-22), the root correctly rounded; dtct carries
// at most 6e-7, dtut and dtvt 4e-7, dtdivt 8e-7 (its branch is taken for
// quotients within 1e-5 of the threshold, so the estimate of a term can only
// fall below the exact one there), and min() keeps the largest of those.
// Operand magnitudes stay inside float's range for every state the
// reference admits (quotients below g_big = 1e21, denominators above
// g_small * volume).
__device__ __forceinline__ double dt_estimate(double ss, double q, double d0, double u00, double u10, double u01, double u11, double v00,
                                              double v10, double v01, double v11, double dsx, double dsy, const DtConsts &k) {
  const double vol = dsx * dsy;
  const double cc = ss * ss + (double)__fdividef((float)(2.0 * q), (float)d0);
  const float ccs = fmaxf(sqrtf((float)cc), (float)g_small);
  const float dtct = __fdividef((float)(k.dtc_safe * fmin(dsx, dsy)), ccs);
  double dv1 = (u00 + u01) * dsy, dv2 = (u10 + u11) * dsy;
  double div = dv2 - dv1;
  const float dtut = __fdividef((float)(k.dtu_safe * 2.0 * vol), (float)fmax(fmax(fabs(dv1), fabs(dv2)), g_small * vol));
  dv1 = (v00 + v10) * dsx;
  dv2 = (v01 + v11) * dsx;
  div = div + dv2 - dv1;
  const float dtvt = __fdividef((float)(k.dtv_safe * 2.0 * vol), (float)fmax(fmax(fabs(dv1), fabs(dv2)), g_small * vol));
  const float divq = __fdividef((float)div, (float)(2.0 * vol));
  const float dtdivt = divq < -(float)g_small * (1.0f - 1e-5f) ? (float)k.dtdiv_safe * __fdividef(-1.0f, divq) : (float)g_big;
  return (double)fminf(dtct, fminf(dtut, fminf(dtvt, fminf(dtdivt, (float)g_big))));
}

// Cells whose estimate exceeds the minimum found so far by more than this
// factor cannot hold the minimum (the estimate's error is below 1e-6).
constexpr double DT_SKIP = 1.0 + 1e-4;

// The dt of a cell at rest (viscosity and the eight corner velocities zero,
// of either sign) is a function of its sound speed, density and two widths
// alone.  A thread that meets a cell at rest with the same four values as
// the last one it evaluated skips it: that value is already in the thread's
// minimum, or the filter showed it cannot lower it.
template <typename T> struct RestMemo {
  T ss, d0, dx, dy;
  bool valid = false;
  __device__ __forceinline__ bool seen(bool rest, T s, T d, T x, T y) {
    if (!rest) return false;
    if (valid && s == ss && d == d0 && x == dx && y == dy) return true;
    ss = s, d0 = d, dx = x, dy = y, valid = true;
    return false;
  }
};

// RestMemo with its four values in shared memory (value k of thread t at
// k * 256 + t): the same test, without the registers (for kernels whose
// registers are spent elsewhere).  The values start as NaN, which no value
// equals.
template <typename T> struct RestMemoShared {
  T *v;
  __device__ __forceinline__ explicit RestMemoShared(T *base) : v(base + threadIdx.y * 64 + threadIdx.x) {
    v[0] = v[256] = v[512] = v[768] = std::numeric_limits<T>::quiet_NaN();
  }
  __device__ __forceinline__ bool seen(bool rest, T s, T d, T x, T y) {
    if (!rest) return false;
    if (s == v[0] && d == v[256] && x == v[512] && y == v[768]) return true;
    v[0] = s, v[256] = d, v[512] = x, v[768] = y;
    return false;
  }
};
constexpr int REST_MEMO_ELEMS = 4 * 256;
template <typename M, typename T> __device__ __forceinline__ M make_memo(T *base) {
  if constexpr (std::is_same<M, RestMemoShared<T>>::value)
    return M(base);
  else
    return M();
}

template <typename T>
__device__ __forceinline__ bool at_rest(T q, T u00, T u10, T u01, T u11, T v00, T v10, T v01, T v11) {
  return q == T(0) && u00 == T(0) && u10 == T(0) && u01 == T(0) && u11 == T(0) && v00 == T(0) && v10 == T(0) && v01 == T(0) &&
         v11 == T(0);
}

struct DtIn {
  const void *soundspeed, *viscosity, *density0;
};

// One calc_dt tile (64 x 16 cells); folds the tile's candidates into vmin.
// Staged: ms 0 xvel0, 1 yvel0; soundspeed, viscosity, density0 are read directly.
constexpr int DT_TY = 16;
template <typename T> constexpr size_t dt_smem() { return 2 * Box1<T, DT_TY>::BOXS * sizeof(T); }

template <typename T, typename Memo>
__device__ __forceinline__ bool calc_dt_tile(TileCtx &cx, T *sm, const MapSet &ms, const DtIn &in, const Mesh<T> &m, int off,
                                             const DtConsts &k, int bx, int by, double &vmin, Memo &memo) {
  constexpr int TY = DT_TY;
  using B = Box1<T, TY>;
  const T *U = sm, *V = sm + B::BOXS;
  const T *S = (const T *)in.soundspeed, *Q = (const T *)in.viscosity, *R = (const T *)in.density0;
  const int pitch = (int)m.pitch;
  constexpr int RPT = TY / 4;
  const int x0 = 2 + bx * TILE_X, y0 = 2 + by * TY;
  const int i = x0 + threadIdx.x;
  // the directly read fields are loaded before the staging wait
  T ss[RPT], qq[RPT], dd[RPT];
#pragma unroll
  for (int r = 0; r < RPT; ++r) {
    const int j = y0 + threadIdx.y + 4 * r;
    const bool in_mesh = i < m.nx + 2 && j < m.ny + 2;
    const int g = gidx(pitch, i, j);
    ss[r] = in_mesh ? S[g] : T(0);
    qq[r] = in_mesh ? Q[g] : T(0);
    dd[r] = in_mesh ? R[g] : T(1);
  }
  if (!stage(cx, sm, ms, 2, B::BOXS, B::BH, off + x0 - HALO, y0 - 1)) return false;
  // FP64: the exact value only where the estimate can beat the warp's minimum so far
  const double thr = sizeof(T) == sizeof(double) ? warp_min(vmin) * DT_SKIP : 0.0;
  if (i < m.nx + 2) {
    const T dsx = m.celldx_t[i];
#pragma unroll
    for (int r = 0; r < RPT; ++r) {
      const int j = y0 + threadIdx.y + 4 * r;
      if (j >= m.ny + 2) break;
      const int b = B::at(i, j, x0, y0);
      // (FP64: only with the memo in shared memory; its registers are spent on the estimate filter)
      if ((sizeof(T) == sizeof(float) || !std::is_same<Memo, RestMemo<T>>::value) &&
          memo.seen(at_rest(qq[r], U[b], U[b + 1], U[b + BOX_X], U[b + BOX_X + 1], V[b], V[b + 1], V[b + BOX_X], V[b + BOX_X + 1]), ss[r],
                    dd[r], dsx, m.celldy_t[j]))
        continue;
      if constexpr (sizeof(T) == sizeof(double)) {
        const double est = dt_estimate(ss[r], qq[r], dd[r], U[b], U[b + 1], U[b + BOX_X], U[b + BOX_X + 1], V[b], V[b + 1], V[b + BOX_X],
                                       V[b + BOX_X + 1], dsx, m.celldy_t[j], k);
        if (est > thr) continue; // NaN estimates fall through to the exact value
      }
      const double c = (double)dt_value(ss[r], qq[r], dd[r], U[b], U[b + 1], U[b + BOX_X], U[b + BOX_X + 1], V[b], V[b + 1],
                                        V[b + BOX_X], V[b + BOX_X + 1], dsx, m.celldy_t[j], k);
      vmin = fmin(c, vmin); // fmin drops a NaN candidate, as the reference's fmin does
    }
  }
  return true;
}

// Blocks loop over tiles; each keeps the minimum of its cells and folds it
// into the result once.
template <typename T>
__global__ void __launch_bounds__(256, 4) kt_calc_dt(const __grid_constant__ Maps maps, DtIn in, Mesh<T> m, int off, DtConsts k, int tiles_x,
                                                  int ntiles, unsigned long long *dt_bits, int *err) {
  extern __shared__ __align__(128) unsigned char smraw[];
  __shared__ uint64_t bar;
  T *sm = reinterpret_cast<T *>(smraw);
  TileCtx cx = tile_ctx(&bar, err);
  const MapSet ms = map_set(maps, 2);
  double vmin = g_big;
  using Memo = std::conditional_t<sizeof(T) == sizeof(double), RestMemoShared<T>, RestMemo<T>>;
  Memo memo = make_memo<Memo>(sm + 2 * Box1<T, DT_TY>::BOXS);
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x)
    if (!calc_dt_tile(cx, sm, ms, in, m, off, k, t % tiles_x, t / tiles_x, vmin, memo)) return;
  block_min_to(vmin, dt_bits);
}

// The ideal-gas law of one cell (src/serial/ideal_gas.cpp:28-48).
template <typename T>
__device__ __forceinline__ void eos_value(T density, T energy, T gm1, T &pressure, T &soundspeed) {
  T v = lim_div(T(1.0), density); // feeds the sound speed only
  pressure = gm1 * density * energy;
  T pressurebyenergy = gm1 * density;
  T pressurebyvolume = -density * pressure;
  T sound_speed_squared = v * v * (pressure * pressurebyenergy - pressurebyvolume);
  soundspeed = sqrt(sound_speed_squared);
}

// ---------------------------------------------------------------------------
// ideal_gas, viscosity and calc_dt in one pass (the resident loop).  A tile
// stages density0, energy0 and the velocities; forms each cell's pressure and
// sound speed as k_ideal_gas does (written, the pressure with its halo of
// depth ig_fold) and the neighbours' pressures viscosity reads from the staged
// density0 / energy0 (their halos hold the mirrored values, so the mirrored
// pressures come out as ideal_gas's fold writes them); computes and stores q
// as viscosity_tile does; and uses it for the cell's dt as calc_dt_tile uses
// the stored q -- the same values and the same minimum as the three phases
// one after the other.  Staged: ms 0 density0, 1 energy0, 2 xvel0, 3 yvel0.
static_assert(VISC_TY == DT_TY, "viscosity and calc_dt tiles of the same height");

template <typename T, typename Memo, int TY = VISC_TY, bool ROLL = false>
__device__ __forceinline__ bool ig_visc_dt_tile(TileCtx &cx, T *sm, const MapSet &ms, T *p_out, T *c_out, T *q_out, const Mesh<T> &m,
                                                int off, const DtConsts &k, T gm1, int ig_fold, int fold, int bx, int by, double &vmin,
                                                Memo &memo) {
  using B = Box1<T, TY>;
  const int pitch = (int)m.pitch;
  constexpr int RPT = TY / 4;
  const int x0 = 2 + bx * TILE_X, y0 = 2 + by * TY;
  const int i = x0 + threadIdx.x;
  if (!stage(cx, sm, ms, 4, B::BOXS, B::BH, off + x0 - HALO, y0 - 1)) return false;
  const T *D = sm, *E = sm + B::BOXS, *U = sm + 2 * B::BOXS, *V = sm + 3 * B::BOXS;
  const double thr = sizeof(T) == sizeof(double) ? warp_min(vmin) * DT_SKIP : 0.0;
  if (i < m.nx + 2) {
    const bool near = edge_tile(m.nx, m.ny, x0, y0, TY);
    const bool do_fold = fold && near;
    const T cdx = m.celldx_t[i], cdx1 = m.celldx_t[i + 1];
#pragma unroll(ROLL ? 1 : RPT)
    for (int r = 0; r < RPT; ++r) {
      const int j = y0 + threadIdx.y + 4 * r;
      if (j >= m.ny + 2) break;
      const int b = B::at(i, j, x0, y0);
      const int g = gidx(pitch, i, j);
      const T cdy = m.celldy_t[j];
      // src/serial/ideal_gas.cpp:28-48 for the cell; pressure alone for its neighbours
      T p, ss;
      eos_value(D[b], E[b], gm1, p, ss);
      // null in the resident loop: the step's Lagrangian pass rewrites the sound
      // speed unread and forms the pressure from density0 and energy0 itself
      if (p_out) {
        p_out[g] = p;
        if (ig_fold && near) fold_halo(p_out, m, halo_rule(PRESSURE), ig_fold, i, j, p);
      }
      if (c_out) c_out[g] = ss;
      const T dd = D[b];
      const T pl = gm1 * D[b - 1] * E[b - 1];
      const T pr = gm1 * D[b + 1] * E[b + 1];
      const T pb = gm1 * D[b - BOX_X] * E[b - BOX_X];
      const T pt = gm1 * D[b + BOX_X] * E[b + BOX_X];
      const T q = viscosity_value(U[b], U[b + 1], U[b + BOX_X], U[b + BOX_X + 1], V[b], V[b + 1], V[b + BOX_X], V[b + BOX_X + 1], pl, pr, pb,
                                  pt, dd, cdx, cdx1, cdy, m.celldy_t[j + 2]);
      q_out[g] = q;
      if (do_fold) fold_halo(q_out, m, halo_rule(VISCOSITY), fold, i, j, q);
      if (memo.seen(at_rest(q, U[b], U[b + 1], U[b + BOX_X], U[b + BOX_X + 1], V[b], V[b + 1], V[b + BOX_X], V[b + BOX_X + 1]), ss, dd, cdx,
                    cdy))
        continue;
      if constexpr (sizeof(T) == sizeof(double)) {
        const double est = dt_estimate(ss, q, dd, U[b], U[b + 1], U[b + BOX_X], U[b + BOX_X + 1], V[b], V[b + 1], V[b + BOX_X],
                                       V[b + BOX_X + 1], cdx, cdy, k);
        if (est > thr) continue; // NaN estimates fall through to the exact value
      }
      const double c = (double)dt_value(ss, q, dd, U[b], U[b + 1], U[b + BOX_X], U[b + BOX_X + 1], V[b], V[b + 1], V[b + BOX_X],
                                        V[b + BOX_X + 1], cdx, cdy, k);
      vmin = fmin(c, vmin);
    }
  }
  return true;
}

// ideal_gas, viscosity and calc_dt in one pass (the resident loop).
template <typename T>
__global__ void __launch_bounds__(256, 4) kt_ig_visc_dt(const __grid_constant__ Maps maps, T *p_out, T *c_out, T *q_out, Mesh<T> m, int off,
                                                     DtConsts k, T gm1, int ig_fold, int fold, int tiles_x, int ntiles,
                                                     unsigned long long *dt_bits, int *err) {
  extern __shared__ __align__(128) unsigned char smraw[];
  __shared__ uint64_t bar;
  T *sm = reinterpret_cast<T *>(smraw);
  TileCtx cx = tile_ctx(&bar, err);
  const MapSet ms = map_set(maps, 4);
  double vmin = g_big;
  // FP64: the memo in shared memory after the four staged boxes (its registers
  // spilled); FP32: in registers (measured faster there)
  using Memo = std::conditional_t<sizeof(T) == sizeof(double), RestMemoShared<T>, RestMemo<T>>;
  Memo memo = make_memo<Memo>(sm + 4 * Box1<T, VISC_TY>::BOXS);
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x)
    if (!ig_visc_dt_tile(cx, sm, ms, p_out, c_out, q_out, m, off, k, gm1, ig_fold, fold, t % tiles_x, t / tiles_x, vmin, memo)) return;
  block_min_to(vmin, dt_bits);
}

// Volume flux through a face (src/serial/flux_calc.cpp:33-40): width is
// xarea (celldy) for x faces, yarea (celldx) for y faces; a0, a1 the level-0
// velocities of the face's two nodes, b0, b1 the level-1 ones.
template <typename T> __device__ __forceinline__ T flux_value(T dt, T width, T a0, T a1, T b0, T b1) {
  return T(0.25) * dt * width * (a0 + a1 + b0 + b1);
}

// ---------------------------------------------------------------------------
// PdV: src/serial/PdV.cpp:36-87; mode 1 also does the predictor's
// ideal_gas, pressure halo and revert (:92-133) in the same pass.
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
  if constexpr (std::is_floating_point<T>::value) {
    // A cell no flux crosses: volume_change = vol / vol = 1 exactly and
    // energy_change is a signed zero, so density1 = d0 and energy1 = e0 to
    // the bit -- given a finite positive vol, quotients p / d0 and q / d0
    // that cannot overflow (bounds below) and a normal e0.  When that holds
    // on every active lane of the warp, the four divisions are skipped.
    const T lo = T(0x1p-60), hi = T(0x1p60);
    const bool still = total_flux == T(0.0) && vol >= lo && vol <= hi && d0 >= lo && d0 <= hi && fabs(p) <= hi && fabs(q) <= hi &&
                       fabs(e0) >= lo && fabs(e0) <= hi;
    if (__all_sync(__activemask(), still)) {
      density1 = d0;
      energy1 = e0;
      return;
    }
  }
  T volume_change_s = (vol) / (vol + total_flux);
  T recip_volume = (T(1.0)) / (vol);
  T energy_change = ((p) / (d0) + (q) / (d0)) * total_flux * recip_volume;
  energy1 = e0 - energy_change;
  density1 = d0 * volume_change_s;
}


struct PdvIn {
  const void *density0, *energy0, *pressure, *viscosity;
};
struct PdvOut {
  void *density1, *energy1, *pressure, *soundspeed;
};

// One PdV tile (64 x 8 cells).
// Staged: ms 0 xvel0, 1 yvel0, [2 xvel1, 3 yvel1]; the cell fields are read directly.
constexpr int PDV_TY = 8;
template <typename T> constexpr size_t pdv_smem() { return 4 * Box1<T, PDV_TY>::BOXS * sizeof(T); }

template <typename T>
__device__ __forceinline__ bool pdv_tile(TileCtx &cx, T *sm, const MapSet &ms, const PdvIn &in, const PdvOut &out, const Mesh<T> &m, int off,
                                         int predict, T dt, int mode, T gm1, int fold, int bx, int by) {
  constexpr int TY = PDV_TY;
  using B = Box1<T, TY>;
  const int x0 = 2 + bx * TILE_X, y0 = 2 + by * TY;
  const int i = x0 + threadIdx.x;
  const int pitch = (int)m.pitch;
  constexpr int RPT = TY / 4;
  // the cell fields are loaded before the staging wait
  T rd[RPT], re[RPT], rp[RPT], rq[RPT];
#pragma unroll
  for (int r = 0; r < RPT; ++r) {
    const int j = y0 + threadIdx.y + 4 * r;
    const bool in_mesh = i < m.nx + 2 && j < m.ny + 2;
    const int g = gidx(pitch, i, j);
    rd[r] = in_mesh ? ((const T *)in.density0)[g] : T(1);
    re[r] = in_mesh ? ((const T *)in.energy0)[g] : T(0);
    rp[r] = in_mesh ? ((const T *)in.pressure)[g] : T(0);
    rq[r] = in_mesh ? ((const T *)in.viscosity)[g] : T(0);
  }
  const int nf = predict ? 2 : 4;
  if (!stage(cx, sm, ms, nf, B::BOXS, B::BH, off + x0 - HALO, y0 - 1)) return false;
  const T *U0 = sm, *V0 = sm + B::BOXS, *U1 = sm + 2 * B::BOXS, *V1 = sm + 3 * B::BOXS;
  if (i >= m.nx + 2) return true;
  const bool do_fold = fold && edge_tile(m.nx, m.ny, x0, y0, TY);
  const T cdx = m.celldx_t[i];
#pragma unroll
  for (int r = 0; r < RPT; ++r) {
    const int j = y0 + threadIdx.y + 4 * r;
    if (j >= m.ny + 2) break;
    const int b = B::at(i, j, x0, y0);
    const int g = gidx(pitch, i, j);
    const T cdy = m.celldy_t[j];
    const T vol = cdx * cdy;
    T w00 = T(0), w01 = T(0), w10 = T(0), w11 = T(0), z00 = T(0), z10 = T(0), z01 = T(0), z11 = T(0);
    if (!predict) {
      w00 = U1[b], w01 = U1[b + BOX_X], w10 = U1[b + 1], w11 = U1[b + BOX_X + 1];
      z00 = V1[b], z10 = V1[b + 1], z01 = V1[b + BOX_X], z11 = V1[b + BOX_X + 1];
    }
    T d1, e1;
    pdv_value(predict != 0, dt, cdy, cdx, vol, U0[b], U0[b + BOX_X], U0[b + 1], U0[b + BOX_X + 1], V0[b], V0[b + 1], V0[b + BOX_X],
              V0[b + BOX_X + 1], w00, w01, w10, w11, z00, z10, z01, z11, rd[r], re[r], rp[r], rq[r], d1, e1);
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
      ((T *)out.density1)[g] = rd[r];
      ((T *)out.energy1)[g] = re[r];
    }
  }
  return true;
}

template <typename T>
__device__ __forceinline__ void pdv_kernel(const Maps &maps, const PdvIn &in, const PdvOut &out, const Mesh<T> &m, int off, int predict, T dt,
                                           const double *dtp, int mode, T gm1, int fold, int *err) {
  extern __shared__ __align__(128) unsigned char smraw[];
  __shared__ uint64_t bar;
  TileCtx cx = tile_ctx(&bar, err);
  pdv_tile(cx, reinterpret_cast<T *>(smraw), map_set(maps, predict ? 2 : 4), in, out, m, off, predict, dtp ? (T)*dtp : dt, mode, gm1, fold,
           blockIdx.x, blockIdx.y);
}

template <typename T>
__global__ void __launch_bounds__(256) kt_pdv(const __grid_constant__ Maps maps, PdvIn in, PdvOut out, Mesh<T> m, int off, int predict, T dt,
                                              const double *dtp, int mode, T gm1, int fold, int *err) {
  pdv_kernel<T>(maps, in, out, m, off, predict, dt, dtp, mode, gm1, fold, err);
}

// The FP64 launch: four blocks per SM (the registers of the quiescent-cell
// test would otherwise leave three).
template <typename T>
__global__ void __launch_bounds__(256, 4) kt_pdv4(const __grid_constant__ Maps maps, PdvIn in, PdvOut out, Mesh<T> m, int off, int predict,
                                                  T dt, const double *dtp, int mode, T gm1, int fold, int *err) {
  pdv_kernel<T>(maps, in, out, m, off, predict, dt, dtp, mode, gm1, fold, err);
}

// ---------------------------------------------------------------------------
// accelerate: src/serial/accelerate.cpp:28-56, nodes [2, nx+2] x [2, ny+2].
// fields: 0 density0, 1 pressure, 2 viscosity, 3 xvel0, 4 yvel0
// Velocity of node (i, j) (src/serial/accelerate.cpp:38-52): cells mm =
// (i-1, j-1), m0 = (i-1, j), 00 = (i, j), 0m = (i, j-1); xa = xarea(i, j),
// xa_m = xarea(i, j-1), ya = yarea(i, j), ya_m = yarea(i-1, j).
template <typename T>
__device__ __forceinline__ void accel_value(T halfdt, T vol_mm, T vol_m0, T vol_00, T vol_0m, T xa, T xa_m, T ya, T ya_m, T d_mm, T d_m0,
                                            T d_00, T d_0m, T p_00, T p_m0, T p_0m, T p_mm, T q_00, T q_m0, T q_0m, T q_mm, T u0, T v0, T &u,
                                            T &v) {
  const T nodal_mass = (d_mm * vol_mm + d_m0 * vol_m0 + d_00 * vol_00 + d_0m * vol_0m) * T(0.25);
  const T fu_p = xa * (p_00 - p_m0) + xa_m * (p_0m - p_mm), fv_p = ya * (p_00 - p_0m) + ya_m * (p_m0 - p_mm);
  const T fu_q = xa * (q_00 - q_m0) + xa_m * (q_0m - q_mm), fv_q = ya * (q_00 - q_0m) + ya_m * (q_m0 - q_mm);
  T stepbymass_s;
  if constexpr (std::is_same<T, double>::value) {
    // A node no force acts on (every pressure and viscosity term a signed
    // zero): stepbymass times each term is that same signed zero for any
    // positive finite stepbymass (the bounds below keep it finite), so 1
    // stands in for it -- the velocities come out to the bit -- and, when
    // that holds on every active lane of the warp, the division is skipped.
    // (FP64 only: the single-precision quotient is cheaper than the test.)
    const T lo = T(0x1p-60), hi = T(0x1p60);
    const bool still = fu_p == T(0.0) && fv_p == T(0.0) && fu_q == T(0.0) && fv_q == T(0.0) && halfdt > T(0.0) && halfdt <= hi &&
                       nodal_mass >= lo;
    if (__all_sync(__activemask(), still))
      stepbymass_s = T(1.0);
    else
      stepbymass_s = (halfdt) / (nodal_mass);
  } else {
    stepbymass_s = (halfdt) / (nodal_mass);
  }
  u = u0 - stepbymass_s * fu_p;
  v = v0 - stepbymass_s * fv_p;
  u = u - stepbymass_s * fu_q;
  v = v - stepbymass_s * fv_q;
}

// One tile of TY node rows; the one-launch kernel uses TY = ACC_TY.
constexpr int ACC_TY = 16;
// Staged boxes start one row above the tile (the nodes' lower cells): Box1.
template <typename T, int TY> constexpr size_t acc_smem() { return 5 * Box1<T, TY>::BOXS * sizeof(T); }

template <typename T, int TY, bool ROLL = false>
__device__ __forceinline__ bool accelerate_tile(TileCtx &cx, T *sm, const MapSet &ms, T *u_out, T *v_out, const Mesh<T> &m, int off, T dt,
                                                int fold, int bx, int by) {
  using B = Box1<T, TY>;
  constexpr int RPT = TY / 4;
  const int x0 = 2 + bx * TILE_X, y0 = 2 + by * TY;
  if (!stage(cx, sm, ms, 5, B::BOXS, B::BH, off + x0 - HALO, y0 - 1)) return false;
  const T *D0 = sm, *P = sm + B::BOXS, *Q = sm + 2 * B::BOXS, *U0 = sm + 3 * B::BOXS, *V0 = sm + 4 * B::BOXS;
  const int i = x0 + threadIdx.x, lx = HALO + threadIdx.x;
  if (i >= m.nx + 3) return true;
  const bool do_fold = fold && edge_tile(m.nx, m.ny, x0, y0, TY);
  const int pitch = (int)m.pitch;
  const T halfdt = T(0.5) * dt;
  const T cdx = m.celldx_t[i], cdxm = m.celldx_t[i - 1];
#pragma unroll(ROLL ? 1 : RPT)
  for (int r = 0; r < RPT; ++r) {
    const int j = y0 + threadIdx.y + 4 * r, ly = 1 + threadIdx.y + 4 * r;
    if (j >= m.ny + 3) break;
    const int b = ly * BOX_X + lx;
    const T cdy = m.celldy_t[j], cdym = m.celldy_t[j - 1];
    const T vol_mm = cdxm * cdym, vol_m0 = cdxm * cdy, vol_00 = cdx * cdy, vol_0m = cdx * cdym;
    const int c00 = b, cm0 = b - 1, c0m = b - BOX_X, cmm = b - BOX_X - 1;
    T u, v;
    accel_value(halfdt, vol_mm, vol_m0, vol_00, vol_0m, cdy, cdym, cdx, cdxm, D0[cmm], D0[cm0], D0[c00], D0[c0m], P[c00], P[cm0], P[c0m],
                P[cmm], Q[c00], Q[cm0], Q[c0m], Q[cmm], U0[c00], V0[c00], u, v);
    const int g = gidx(pitch, i, j);
    u_out[g] = u;
    v_out[g] = v;
    if (do_fold) {
      fold_halo(u_out, m, halo_rule(XVEL1), fold, i, j, u);
      fold_halo(v_out, m, halo_rule(YVEL1), fold, i, j, v);
    }
  }
  return true;
}

template <typename T>
__global__ void __launch_bounds__(256) kt_accelerate(const __grid_constant__ Maps maps, T *u_out, T *v_out, Mesh<T> m, int off, T dt,
                                                     const double *dtp, int fold, int *err) {
  extern __shared__ __align__(128) unsigned char smraw[];
  __shared__ uint64_t bar;
  TileCtx cx = tile_ctx(&bar, err);
  accelerate_tile<T, ACC_TY>(cx, reinterpret_cast<T *>(smraw), map_set(maps, 5), u_out, v_out, m, off, dtp ? (T)*dtp : dt, fold, blockIdx.x,
                             blockIdx.y);
}

// ---------------------------------------------------------------------------
// The Lagrangian step in one pass (the resident loop): the PdV predictor with
// its ideal_gas and pressure halo, accelerate, the PdV corrector and
// flux_calc (src/serial/PdV.cpp:36-133, accelerate.cpp:28-56,
// flux_calc.cpp:27-43).  A tile of 64 x TY cells needs the level-1
// velocities of the nodes around its cells, one node wider than the tile's
// own nodes on their high sides, and those need the predicted pressure of a
// ring one cell wider still on every side: the tile evaluates both rings
// itself (a halo cell through its mirror interior cell, the depth-1
// reflection that the predictor's fold writes), keeps them in shared memory
// and writes the outputs of its own cells, nodes and faces.  The predictor's
// revert is not written: the corrector overwrites density1 and energy1 in
// every interior cell.  Every output is folded (fold depths above zero: the
// halo faces are the fold's).  The predicted pressure goes to
// out.pressure, a buffer other than the pressure's current one, because
// other tiles still read the old pressure of their ring cells; the caller
// swaps the two.
// Staged: 0 xvel0, 1 yvel0, 2 density0, 3 energy0, 4 pressure, 5 viscosity,
// rows y0 - 1 .. y0 + TY + 2.
// PDE: the level-0 pressure formed from density0 and energy0 where it is read
// (eos_value's product, the same bits as the ideal_gas pass stores) instead
// of staged: five boxes.
template <typename T, int TY, bool PDE = false> struct LagLayout {
  static constexpr int NBOX = PDE ? 5 : 6;
  static constexpr int BH = TY + 4;
  static constexpr int BOXS = (BOX_X * BH * (int)sizeof(T) + 127) / 128 * 128 / (int)sizeof(T);
  static constexpr int PCX = TILE_X + 2, PCY = TY + 2; // predicted pressure: cells x0 - 1 + p, y0 - 1 + l
  static constexpr int NNX = TILE_X + 1, NNY = TY + 1; // level-1 velocities: nodes x0 + p, y0 + l
  // + celldx of the box's columns and celldy of its rows (fill_widths)
  static constexpr size_t SMEM = (size_t)(NBOX * BOXS + PCX * PCY + 2 * NNX * NNY + BOX_X + BH) * sizeof(T);
  __device__ static constexpr int at(int i, int j, int x0, int y0) { return (j - y0 + 1) * BOX_X + (i - x0 + HALO); }
};

// The items (p, l), p < NA, l < NB, of a ring stage over the block's eight
// warps: a warp takes 32 consecutive positions of one row (G such groups per
// row), and the R = NA mod 32 positions left at the end of every row are
// packed into shared groups taken last.  Lanes of a full group read
// consecutive elements of one row of shared memory (no bank conflicts), and
// the rounds are as few as the groups allow.  The rounds stay a loop: one
// copy of f's body (the FP32 Lagrangian pass was waiting on instruction
// fetch; 0.80 -> 0.78 ms at 7680^2, FP64 unchanged).
template <int NA, int NB, typename F> __device__ __forceinline__ void each_rows(F &&f) {
  constexpr int G = NA / 32, R = NA % 32;
  constexpr int NG = NB * G, NL = (NB * R + 31) / 32;
  const int w = (threadIdx.y * 64 + threadIdx.x) >> 5, lane = threadIdx.x & 31;
#pragma unroll 1
  for (int k = 0; k < (NG + NL + 7) / 8; ++k) {
    const int u = w + 8 * k; // warp-uniform
    if (u < NG) {
      f(32 * (u % G) + lane, u / G);
    } else if (u < NG + NL) {
      const int t = (u - NG) * 32 + lane;
      if (t < NB * R) f(32 * G + t % R, t / R);
    }
  }
}

// store_ps: when set, the predicted pressure and soundspeed are stored only
// if *store_ps is nonzero (the resident loop's last step: in the others the
// next step's pass rewrites both before anything reads them).
template <typename T> struct LagOut {
  T *pressure, *soundspeed, *xvel1, *yvel1, *density1, *energy1, *vol_flux_x, *vol_flux_y;
  const int *store_ps = nullptr;
};
struct LagFolds {
  int pressure, accelerate, pdv, flux;
};

// EDGE: a tile within reach of the mesh edge (edge_tile); the others are
// compiled without extent checks, clamps and halo folds.
// The tile (bx, by) with the block's staging context and shared memory
// (L::SMEM bytes at sm); staged fields ms 0..5 as above.  Returns false when
// the staging wait gave up.
template <typename T, int TY, bool EDGE, bool PDE = false>
__device__ __forceinline__ bool lagrange_tile(TileCtx &cx, T *sm, const MapSet &ms, const LagOut<T> &out, const Mesh<T> &m, int off, T dt,
                                              T gm1, const LagFolds &fd, int bx, int by) {
  using L = LagLayout<T, TY, PDE>;
  const int x0 = 2 + bx * TILE_X, y0 = 2 + by * TY;
  const T *U0 = sm, *V0 = sm + L::BOXS, *D0 = sm + 2 * L::BOXS, *E0 = sm + 3 * L::BOXS, *P = sm + 4 * L::BOXS;
  const T *Q = sm + (L::NBOX - 1) * L::BOXS;
  T *sp = sm + L::NBOX * L::BOXS, *su = sp + L::PCX * L::PCY, *sv = su + L::NNX * L::NNY, *gx = sv + L::NNX * L::NNY, *gy = gx + BOX_X;
  stage_issue(cx, sm, ms, L::NBOX, L::BOXS, L::BH, off + x0 - HALO, y0 - 1);
  fill_widths(m, x0, y0, 1, L::BH, 1, gx, gy, nullptr, nullptr); // gx[i - x0 + HALO] = celldx[i], gy[j - y0 + 1] = celldy[j]
  if (!stage_wait(cx)) return false;
  const int pitch = (int)m.pitch;
  const bool store_ps = !out.store_ps || *out.store_ps != 0;
  // (1) the predictor over the pressure ring
  each_rows<L::PCX, L::PCY>([&](int p, int l) {
    const int i = x0 - 1 + p, j = y0 - 1 + l;
    if (EDGE && (i > m.nx + 2 || j > m.ny + 2)) return; // no node of the mesh reads it
    const int ic = EDGE ? min(max(i, 2), m.nx + 1) : i, jc = EDGE ? min(max(j, 2), m.ny + 1) : j;
    const int b = L::at(ic, jc, x0, y0);
    const T cdx = gx[ic - x0 + HALO], cdy = gy[jc - y0 + 1];
    const T vol = cdx * cdy;
    const T z = T(0);
    T d1, e1;
    pdv_value(true, dt, cdy, cdx, vol, U0[b], U0[b + BOX_X], U0[b + 1], U0[b + BOX_X + 1], V0[b], V0[b + 1], V0[b + BOX_X], V0[b + BOX_X + 1],
              z, z, z, z, z, z, z, z, D0[b], E0[b], PDE ? gm1 * D0[b] * E0[b] : P[b], Q[b], d1, e1);
    sp[l * L::PCX + p] = gm1 * d1 * e1; // eos_value's pressure
    if (store_ps && p >= 1 && p <= TILE_X && l >= 1 && l <= TY && (!EDGE || (i == ic && j == jc))) { // one of the tile's own interior cells
      T pp, cc;
      eos_value(d1, e1, gm1, pp, cc);
      const int g = gidx(pitch, i, j);
      out.pressure[g] = pp;
      out.soundspeed[g] = cc;
      if (EDGE && fd.pressure) fold_halo(out.pressure, m, halo_rule(PRESSURE), fd.pressure, i, j, pp);
    }
  });
  __syncthreads();
  // (2) accelerate over the nodes [x0, x0 + 64] x [y0, y0 + TY]
  const T halfdt = T(0.5) * dt;
  each_rows<L::NNX, L::NNY>([&](int p, int l) {
    const int i = x0 + p, j = y0 + l;
    if (EDGE && (i > m.nx + 2 || j > m.ny + 2)) return;
    const int b = L::at(i, j, x0, y0);
    const int s00 = (l + 1) * L::PCX + (p + 1);
    const T cdx = gx[p + HALO], cdxm = gx[p + HALO - 1], cdy = gy[l + 1], cdym = gy[l];
    const T vol_mm = cdxm * cdym, vol_m0 = cdxm * cdy, vol_00 = cdx * cdy, vol_0m = cdx * cdym;
    const int c00 = b, cm0 = b - 1, c0m = b - BOX_X, cmm = b - BOX_X - 1;
    T u, v;
    accel_value(halfdt, vol_mm, vol_m0, vol_00, vol_0m, cdy, cdym, cdx, cdxm, D0[cmm], D0[cm0], D0[c00], D0[c0m], sp[s00], sp[s00 - 1],
                sp[s00 - L::PCX], sp[s00 - L::PCX - 1], Q[c00], Q[cm0], Q[c0m], Q[cmm], U0[c00], V0[c00], u, v);
    su[l * L::NNX + p] = u;
    sv[l * L::NNX + p] = v;
    if (p < TILE_X && l < TY) { // one of the tile's own nodes
      const int g = gidx(pitch, i, j);
      out.xvel1[g] = u;
      out.yvel1[g] = v;
      if (EDGE && fd.accelerate) {
        fold_halo(out.xvel1, m, halo_rule(XVEL1), fd.accelerate, i, j, u);
        fold_halo(out.yvel1, m, halo_rule(YVEL1), fd.accelerate, i, j, v);
      }
    }
  });
  __syncthreads();
  // (3) the corrector over the tile's cells and flux_calc over its faces
  const int i = x0 + threadIdx.x;
  if (EDGE && i >= m.nx + 3) return true;
  const T cdx = gx[threadIdx.x + HALO];
#pragma unroll
  for (int r = 0; r < TY / 4; ++r) {
    const int j = y0 + threadIdx.y + 4 * r;
    if (EDGE && j >= m.ny + 3) break;
    const int b = L::at(i, j, x0, y0);
    const int n = (j - y0) * L::NNX + (i - x0);
    const int g = gidx(pitch, i, j);
    const T cdy = gy[j - y0 + 1];
    if (!EDGE || (i < m.nx + 2 && j < m.ny + 2)) {
      const T vol = cdx * cdy;
      T d1, e1;
      pdv_value(false, dt, cdy, cdx, vol, U0[b], U0[b + BOX_X], U0[b + 1], U0[b + BOX_X + 1], V0[b], V0[b + 1], V0[b + BOX_X],
                V0[b + BOX_X + 1], su[n], su[n + L::NNX], su[n + 1], su[n + L::NNX + 1], sv[n], sv[n + 1], sv[n + L::NNX],
                sv[n + L::NNX + 1], D0[b], E0[b], sp[(j - y0 + 1) * L::PCX + (i - x0 + 1)], Q[b], d1, e1);
      out.density1[g] = d1;
      out.energy1[g] = e1;
      if (EDGE && fd.pdv) {
        fold_halo(out.density1, m, halo_rule(DENSITY1), fd.pdv, i, j, d1);
        fold_halo(out.energy1, m, halo_rule(ENERGY1), fd.pdv, i, j, e1);
      }
    }
    // flux_calc_tile's face values and folded writes: x faces below row
    // ny + 2, y faces left of column nx + 2 (the fold writes the rest)
    if (!EDGE || j < m.ny + 2) {
      const T fx = flux_value(dt, cdy, U0[b], U0[b + BOX_X], su[n], su[n + L::NNX]);
      out.vol_flux_x[g] = fx;
      if (EDGE) fold_halo(out.vol_flux_x, m, halo_rule(VOL_FLUX_X), fd.flux, i, j, fx);
    }
    if (!EDGE || i < m.nx + 2) {
      const T fy = flux_value(dt, cdx, V0[b], V0[b + 1], sv[n], sv[n + 1]);
      out.vol_flux_y[g] = fy;
      if (EDGE) fold_halo(out.vol_flux_y, m, halo_rule(VOL_FLUX_Y), fd.flux, i, j, fy);
    }
  }
  return true;
}

// Registers capped for the blocks per SM the shared memory allows: FP64 four
// (8 rows) or three (12 rows), FP32 five.
template <typename T, int TY, bool PDE = false>
__global__ void __launch_bounds__(256, sizeof(T) == sizeof(double) ? (TY == 8 ? 4 : 3) : 5)
    kt_lagrange(const __grid_constant__ Maps maps, LagOut<T> out, Mesh<T> m, int off, T dt, const double *dtp, T gm1, LagFolds fd, int *err) {
  extern __shared__ __align__(128) unsigned char smraw[];
  __shared__ uint64_t bar;
  T *sm = reinterpret_cast<T *>(smraw);
  TileCtx cx = tile_ctx(&bar, err);
  const T d = dtp ? (T)*dtp : dt;
  constexpr int NB = LagLayout<T, TY, PDE>::NBOX;
  if (edge_tile(m.nx, m.ny, 2 + blockIdx.x * TILE_X, 2 + blockIdx.y * TY, TY))
    lagrange_tile<T, TY, true, PDE>(cx, sm, map_set(maps, NB), out, m, off, d, gm1, fd, blockIdx.x, blockIdx.y);
  else
    lagrange_tile<T, TY, false, PDE>(cx, sm, map_set(maps, NB), out, m, off, d, gm1, fd, blockIdx.x, blockIdx.y);
}

// ---------------------------------------------------------------------------
// flux_calc: src/serial/flux_calc.cpp:27-43, faces [2, nx+2] x [2, ny+2].
// With a fold, the extra row of x faces and column of y faces (overwritten
// by update_halo) take their halo values.
// fields: 0 xvel0, 1 yvel0, 2 xvel1, 3 yvel1

constexpr int FLUX_TY = 16;
// Staged boxes start one row above the tile: Box1 (the faces need rows j and j + 1).
template <typename T, int TY> constexpr size_t flux_smem() { return 4 * Box1<T, TY>::BOXS * sizeof(T); }

template <typename T, int TY, bool ROLL = false>
__device__ __forceinline__ bool flux_calc_tile(TileCtx &cx, T *sm, const MapSet &ms, T *fx_out, T *fy_out, const Mesh<T> &m, int off, T dt,
                                               int fold, int bx, int by) {
  using B = Box1<T, TY>;
  constexpr int RPT = TY / 4;
  const int x0 = 2 + bx * TILE_X, y0 = 2 + by * TY;
  if (!stage(cx, sm, ms, 4, B::BOXS, B::BH, off + x0 - HALO, y0 - 1)) return false;
  const T *U0 = sm, *V0 = sm + B::BOXS, *U1 = sm + 2 * B::BOXS, *V1 = sm + 3 * B::BOXS;
  const int i = x0 + threadIdx.x, lx = HALO + threadIdx.x;
  if (i >= m.nx + 3) return true;
  const bool do_fold = fold && edge_tile(m.nx, m.ny, x0, y0, TY);
  const int pitch = (int)m.pitch;
  const T cdx = m.celldx_t[i];
#pragma unroll(ROLL ? 1 : RPT)
  for (int r = 0; r < RPT; ++r) {
    const int j = y0 + threadIdx.y + 4 * r, ly = 1 + threadIdx.y + 4 * r;
    if (j >= m.ny + 3) break;
    const int b = ly * BOX_X + lx;
    T fx = flux_value(dt, m.celldy_t[j], U0[b], U0[b + BOX_X], U1[b], U1[b + BOX_X]);
    T fy = flux_value(dt, cdx, V0[b], V0[b + 1], V1[b], V1[b + 1]);
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
  return true;
}

template <typename T>
__global__ void __launch_bounds__(256) kt_flux_calc(const __grid_constant__ Maps maps, T *fx_out, T *fy_out, Mesh<T> m, int off, T dt,
                                                    const double *dtp, int fold, int *err) {
  extern __shared__ __align__(128) unsigned char smraw[];
  __shared__ uint64_t bar;
  TileCtx cx = tile_ctx(&bar, err);
  flux_calc_tile<T, FLUX_TY>(cx, reinterpret_cast<T *>(smraw), map_set(maps, 4), fx_out, fy_out, m, off, dtp ? (T)*dtp : dt, fold, blockIdx.x,
                             blockIdx.y);
}

// ---------------------------------------------------------------------------
// Rows per tile of the advection kernels, x sweep and y sweep: 8 in FP64
// (issue-bound; smaller boxes keep five blocks per SM), 16 in FP32 (half the
// bytes per element: taller tiles halve the per-tile staging overhead and
// the share of cells recomputed in the tile overlaps).
template <typename T> struct AdvecTiles {
  static constexpr int CELL_X = 8, CELL_Y = 8, MOM_X = 8, MOM_Y = 8;
};
template <> struct AdvecTiles<float> {
  static constexpr int CELL_X = 16, CELL_Y = 16, MOM_X = 16, MOM_Y = 16;
};

// ---------------------------------------------------------------------------
// advec_cell: src/serial/advec_cell.cpp:28-220, one sweep in one pass: the
// face fluxes into shared memory, then the update; each stage's items are
// dealt to the threads as Items<> deals them, and pre_vol is formed from the
// staged volume fluxes where a face or an update reads it.
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

// pre_vol of a cell (src/serial/advec_cell.cpp:42-61 / :134-153): sweep 1
// adds both directions' flux differences (the sweep's first), sweep 2 only
// the sweep direction's.
template <typename T> __device__ __forceinline__ T cell_pre_vol1(T vol, T a_lo, T a_hi, T b_lo, T b_hi) {
  return vol + (a_hi - a_lo + b_hi - b_lo);
}
template <typename T> __device__ __forceinline__ T cell_pre_vol2(T vol, T a_lo, T a_hi) { return vol + a_hi - a_lo; }

// Mass flux through a face and the energy the flux carries per unit mass
// (:63-113 / :155-205): flux the face's volume flux, donor/upwind/downwind
// the cells the flux's sign selects (d* densities, e* energies), pre_vol_d
// the donor's pre_vol, vdx_f / vdx_dif the vertex widths at the face and at
// the cell the limiter's ratio uses; ratio = vdx_f / vdx_dif.  The energy
// flux is mass_flux * e_adv.
template <typename T>
__device__ __forceinline__ void cell_face_value(T flux, T pre_vol_d, T ratio, T dd, T du, T dw, T ed, T eu, T ew, T &mass_flux, T &e_adv) {
  T sigmat = sizeof(T) == sizeof(double) ? div_zero_num(fabs(flux), pre_vol_d) : lim_div(fabs(flux), pre_vol_d);
  T sigma3 = (T(1.0) + sigmat) * ratio;
  T sigma4 = T(2.0) - sigmat;
  T sigmav = sigmat;
  T limiter = cell_limiter_value(sigmav, sigma3, sigma4, dd - du, dw - dd);
  mass_flux = flux * (dd + limiter);
  T sigmam = sizeof(T) == sizeof(double) ? div_zero_num(fabs(mass_flux), dd * pre_vol_d) : lim_div(fabs(mass_flux), dd * pre_vol_d);
  limiter = cell_limiter_value(sigmam, sigma3, sigma4, ed - eu, ew - ed);
  e_adv = ed + limiter;
}

// The cell's update (:117-129 / :209-221) in the precision of its mass and
// energy accumulation: mf/ef the mass and energy fluxes of its low and high
// faces, vf the volume fluxes.
template <typename S>
__device__ __forceinline__ void cell_update_value(S d1, S e1, S pre_vol, S mf_lo, S mf_hi, S ef_lo, S ef_hi, S vf_lo, S vf_hi, S &dnew,
                                                  S &enew) {
  S pre_mass_s = d1 * pre_vol;
  S post_mass_s = pre_mass_s + mf_lo - mf_hi;
  S ener_s = e1 * pre_mass_s + ef_lo - ef_hi;
  S advec_vol_s = pre_vol + vf_lo - vf_hi;
  S post_ener_s = (ener_s) / (post_mass_s);
  dnew = (post_mass_s) / (advec_vol_s);
  enew = post_ener_s;
}

// density0 / energy0 set: the sweep also does reset_field's cell copy
// (src/serial/reset_field.cpp:33-40) of the values it writes, with its fold
// depth rfold -- the resident loop's second sweep, which then leaves energy1
// null: energy1 is not read again before the next step's PdV rewrites it,
// and the loop restores it once at its end.  (density1 stays: the momentum
// sweep after it reads its depth-2 halo, which level 0 does not carry.)
struct CellOut {
  void *density1, *energy1, *mass_flux;
  void *density0 = nullptr, *energy0 = nullptr;
  int rfold = 0;
};

// Tile of the cell sweep: LA cells along the sweep x LL lines across.
// Staged boxes (BOX_X x BH, tensor rows from y0 - YH): density1, energy1,
// vol_flux_x, vol_flux_y.  The faces are 0 .. LA along the sweep (their
// donors reach cells -1 .. LA).
template <typename T, int DIR, int TY> struct CellLayout {
  static constexpr int LA = DIR == 1 ? TILE_X : TY;
  static constexpr int LL = DIR == 1 ? TY : TILE_X;
  static constexpr int YH = DIR == 1 ? 1 : 2;
  static constexpr int BH = DIR == 1 ? TY + 2 : TY + 4;
  static constexpr int BOX = BOX_X * BH;
  static constexpr int BOXS = (BOX * (int)sizeof(T) + 127) / 128 * 128 / (int)sizeof(T);
  static constexpr int NF = LA + 1;
  // face scratch: FP64 keeps each face's mass flux and energy flux; FP32
  // keeps the mass flux and e_adv as they were computed (single precision)
  // and forms the FP64 energy flux, an exact product, where it is used
  using FS = std::conditional_t<sizeof(T) == sizeof(double), double, float>;
  static constexpr size_t SCRATCH_BYTES = ((size_t)2 * NF * LL * sizeof(FS) + 15) / 16 * 16;
  // then the widths (fill_widths): vertex widths and reciprocals along the sweep, celldx, celldy
  static constexpr int LV = DIR == 1 ? BOX_X : BH;
  static constexpr size_t GEO_BYTES = (size_t)2 * LV * sizeof(double) + (size_t)(BOX_X + BH) * sizeof(T);
  static constexpr size_t SMEM = (size_t)4 * BOXS * sizeof(T) + SCRATCH_BYTES + GEO_BYTES;
  __device__ static constexpr int fx(int p, int l) { return DIR == 1 ? l * NF + p : p * LL + l; }  // p = face
};

// EDGE = false: a tile whose every position lies inside the mesh's extents
// (no edge_tile), so the extent checks, the upwind clamp and the halo fold
// drop out.
// The tile's work once its boxes are staged at `sm` (density1, energy1,
// vol_flux_x, vol_flux_y, L::BOXS elements apart); `scratch` holds the face
// fluxes and pre_vol (L::SCRATCH_BYTES).
template <typename T, int DIR, int TY, bool EDGE, bool COMPACT = false>
__device__ __forceinline__ void advec_cell_compute(const T *sm, void *scratch, const CellOut &out, const Mesh<T> &m, int sweep, int fold,
                                                   int bx, int by) {
  using L = CellLayout<T, DIR, TY>;
  constexpr int LA = L::LA, LL = L::LL, YH = L::YH;
  using FS = typename L::FS;
  FS *s_mf = reinterpret_cast<FS *>(scratch);
  FS *s_ef = s_mf + L::NF * LL; // FP64: mass_flux * e_adv; FP32: e_adv
  const double *g_vd = reinterpret_cast<const double *>(reinterpret_cast<char *>(scratch) + L::SCRATCH_BYTES);
  const double *g_rvd = g_vd + L::LV;
  const T *g_x = reinterpret_cast<const T *>(g_rvd + L::LV), *g_y = g_x + BOX_X;
  const int x0 = 2 + bx * TILE_X, y0 = 2 + by * TY;
  const int vo = DIR == 1 ? HALO - x0 : YH - y0; // index of the sweep's vertex width of position a: a + vo
  const T *D1 = sm, *E1 = sm + L::BOXS, *VFX = sm + 2 * L::BOXS, *VFY = sm + 3 * L::BOXS;
  const int na = DIR == 1 ? m.nx : m.ny, nlmax = DIR == 1 ? m.ny : m.nx;
  const int a0 = DIR == 1 ? x0 : y0, l0 = DIR == 1 ? y0 : x0;
  const int pitch = (int)m.pitch;
  constexpr int ST = DIR == 1 ? 1 : BOX_X; // box stride along the sweep
  auto bidx = [&](int i, int j) { return (j - y0 + YH) * BOX_X + (i - x0 + HALO); };
  // pre_vol (advec_cell.cpp:42-61 / :134-153) of cell (i, j), formed where
  // it is read (a face's donor, a cell's update) rather than stored
  auto pre_vol_of = [&](int i, int j) -> T {
    const int b = bidx(i, j);
    const T vol = g_x[i - x0 + HALO] * g_y[j - y0 + YH];
    if (DIR == 1)
      return sweep == 1 ? cell_pre_vol1(vol, VFX[b], VFX[b + 1], VFY[b], VFY[b + BOX_X]) : cell_pre_vol2(vol, VFX[b], VFX[b + 1]);
    return sweep == 1 ? cell_pre_vol1(vol, VFY[b], VFY[b + BOX_X], VFX[b], VFX[b + 1]) : cell_pre_vol2(vol, VFY[b], VFY[b + BOX_X]);
  };
  // (2) face fluxes (:63-113 / :155-205), faces a0 .. a0+LA
  const bool edge = EDGE && fold;
  Items<DIR, L::NF, LL>::template each<!COMPACT>([&](int, int p, int l) {
    const int f = a0 + p, line = l0 + l; // position of the face along the sweep
    const int i = DIR == 1 ? f : line, j = DIR == 1 ? line : f;
    if (EDGE && (i > (DIR == 1 ? m.nx + 3 : m.nx + 1) || j > (DIR == 1 ? m.ny + 1 : m.ny + 3))) return;
    const int b = bidx(i, j);
    const T flux = DIR == 1 ? VFX[b] : VFY[b];
    int upwind, donor, downwind, dif;
    if (flux > T(0.0)) {
      upwind = f - 2; donor = f - 1; downwind = f; dif = donor;
    } else {
      upwind = (!EDGE || f + 1 < na + 2) ? f + 1 : na + 2;
      donor = f; downwind = f - 1; dif = upwind;
    }
    const int bd = b + (donor - f) * ST, bu = b + (upwind - f) * ST, bw = b + (downwind - f) * ST;
    const T pre_vol_d = DIR == 1 ? pre_vol_of(donor, line) : pre_vol_of(line, donor);
    T mass_flux, e_adv;
    T ratio;
    if constexpr (sizeof(T) == sizeof(double)) {
      ratio = width_ratio(g_vd[f + vo], g_vd[dif + vo], g_rvd[dif + vo]); // = vertexdx[f] / vertexdx[dif]
    } else {
      ratio = lim_div((T)g_vd[f + vo], (T)g_vd[dif + vo]);
    }
    cell_face_value(flux, pre_vol_d, ratio, D1[bd], D1[bu], D1[bw], E1[bd], E1[bu], E1[bw], mass_flux, e_adv);
    s_mf[L::fx(p, l)] = mass_flux;
    if constexpr (sizeof(T) == sizeof(double))
      s_ef[L::fx(p, l)] = mass_flux * e_adv;
    else
      s_ef[L::fx(p, l)] = e_adv;
    T *mf = (T *)out.mass_flux;
    const bool halo_face = EDGE && fold && f == na + 3; // with a fold, face na+3 takes its halo value
    if (!halo_face) mf[gidx(pitch, i, j)] = mass_flux;
    if (edge && f < na + 3) fold_halo(mf, m, halo_rule(DIR == 1 ? MASS_FLUX_X : MASS_FLUX_Y), fold, i, j, mass_flux);
  });
  __syncthreads();
  // (3) the update (:117-129 / :209-221), mass/energy accumulation in FP64
  Items<DIR, LA, LL>::template each<!COMPACT>([&](int, int p, int l) {
    const int a = a0 + p, line = l0 + l;
    const int i = DIR == 1 ? a : line, j = DIR == 1 ? line : a;
    if (EDGE && (i >= m.nx + 2 || j >= m.ny + 2)) return;
    const int b = bidx(i, j);
    const T pre_vol = pre_vol_of(i, j);
    const double mf_lo = s_mf[L::fx(p, l)], mf_hi = s_mf[L::fx(p + 1, l)];
    double ef_lo, ef_hi;
    if constexpr (sizeof(T) == sizeof(double)) {
      ef_lo = s_ef[L::fx(p, l)], ef_hi = s_ef[L::fx(p + 1, l)];
    } else {
      ef_lo = mf_lo * (double)s_ef[L::fx(p, l)], ef_hi = mf_hi * (double)s_ef[L::fx(p + 1, l)];
    }
    const T vf_lo = DIR == 1 ? VFX[b] : VFY[b];
    const T vf_hi = DIR == 1 ? VFX[b + 1] : VFY[b + BOX_X];
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
      // FP32 form: the sums above stay FP64; the quotients are stored in
      // FP32, so they are formed in FP32 from the rounded sums
      dnew = (T)post_mass_s / (T)advec_vol_s;
      enew = (T)ener_s / (T)post_mass_s;
    }
    const int g = gidx(pitch, i, j);
    ((T *)out.density1)[g] = dnew;
    if (edge) fold_halo((T *)out.density1, m, halo_rule(DENSITY1), fold, i, j, dnew);
    if (out.energy1) {
      ((T *)out.energy1)[g] = enew;
      if (edge) fold_halo((T *)out.energy1, m, halo_rule(ENERGY1), fold, i, j, enew);
    }
    if (out.density0) {
      ((T *)out.density0)[g] = dnew;
      ((T *)out.energy0)[g] = enew;
      if (EDGE && out.rfold) {
        fold_halo((T *)out.density0, m, halo_rule(DENSITY0), out.rfold, i, j, dnew);
        fold_halo((T *)out.energy0, m, halo_rule(ENERGY0), out.rfold, i, j, enew);
      }
    }
  });
}

// Fields the cell sweep stages: sweep 2 of x needs no y fluxes.
template <int DIR> __device__ __forceinline__ int cell_staged(int sweep) { return (sweep == 1) ? 4 : (DIR == 1 ? 3 : 4); }

// One tile: staging, then the work (an edge tile keeps the extent checks).
// ALL_EDGE compiles the edge form only, used for every tile (the same
// values; less code for a caller that holds many phases in one kernel).
template <typename T, int DIR, int TY, bool ALL_EDGE = false>
__device__ __forceinline__ bool advec_cell_tile(TileCtx &cx, T *sm, const MapSet &ms, const CellOut &out, const Mesh<T> &m, int off,
                                                int sweep, int fold, int bx, int by) {
  using L = CellLayout<T, DIR, TY>;
  const int x0 = 2 + bx * TILE_X, y0 = 2 + by * TY;
  stage_issue(cx, sm, ms, cell_staged<DIR>(sweep), L::BOXS, L::BH, off + x0 - HALO, y0 - L::YH);
  {
    char *geo = reinterpret_cast<char *>(sm + 4 * L::BOXS) + L::SCRATCH_BYTES;
    double *gv = reinterpret_cast<double *>(geo), *grv = gv + L::LV;
    T *gx = reinterpret_cast<T *>(grv + L::LV);
    fill_widths(m, x0, y0, L::YH, L::BH, DIR, gx, gx + BOX_X, gv, grv);
  }
  if (!stage_wait(cx)) return false;
  if (ALL_EDGE || edge_tile(m.nx, m.ny, x0, y0, TY))
    advec_cell_compute<T, DIR, TY, true, ALL_EDGE>(sm, sm + 4 * L::BOXS, out, m, sweep, fold, bx, by);
  else
    advec_cell_compute<T, DIR, TY, false>(sm, sm + 4 * L::BOXS, out, m, sweep, fold, bx, by);
  return true;
}

// Blocks per SM the register budget must allow: five in FP64 (the staged
// boxes of five tiles), six in FP32.
template <typename T> constexpr int cell_min_blocks() { return sizeof(T) == sizeof(double) ? 5 : 6; }

template <typename T, int DIR, int TY>
__global__ void __launch_bounds__(256, cell_min_blocks<T>()) kt_advec_cell(const __grid_constant__ Maps maps, CellOut out, Mesh<T> m, int off, int sweep,
                                                     int fold, int *err) {
  extern __shared__ __align__(128) unsigned char smraw[];
  __shared__ uint64_t bar;
  TileCtx cx = tile_ctx(&bar, err);
  advec_cell_tile<T, DIR, TY>(cx, reinterpret_cast<T *>(smraw), map_set(maps, 4), out, m, off, sweep, fold, blockIdx.x, blockIdx.y);
}

// ---------------------------------------------------------------------------
// advec_mom: src/serial/advec_mom.cpp:30-225, both velocities in one pass.
//
// A block updates the nodes of a tile: LA nodes along the sweep (a) times LL
// lines across it.  Positions p = 0 .. LA+2 along the sweep map to nodes
// a = a0 - 2 + p; the stages cover only the positions the tile's outputs
// need (node flux and cell mass p = 0..LA+2, momentum fluxes 1..LA+1,
// updates 2..LA+1), and every stage deals its (position, line) items to the
// threads as Items<> deals them.
//
// Cell masses density1 * post_vol are formed once per cell (the reference
// forms each four times inside node_mass_post, :93-102 / :165-174, with the
// same products and the same order of the sum, so the bits agree);
// node_mass_post and node_mass_pre are re-formed from them and the node
// fluxes where a momentum flux or an update reads them.
//
// Staged boxes (BOX_X x BH, tensor rows from y0 - YH): xvel1, yvel1, then
// density1, the sweep's mass flux and (sweep 1) the other direction's volume
// flux.  The work arrays reuse the space of the last three once the first
// stage has read them.
template <typename T>
__device__ __forceinline__ T mom_limiter_value(T vdiffuw, T vdiffdw, T sigma, T width, T dx_dif) {
  T limiter = T(0.0);
  if (vdiffuw * vdiffdw > T(0.0)) {
    T auw = fabs(vdiffuw);
    T adw = fabs(vdiffdw);
    T wind = T(1.0);
    if (vdiffdw <= T(0.0)) wind = T(-1.0);
    limiter = wind * fmin(fmin(lim_div(width * (lim_div((T(2.0) - sigma) * adw, width) + lim_div((T(1.0) + sigma) * auw, dx_dif)), T(6.0)), auw), adw);
  }
  return limiter;
}

// The sum of four terms scaled by 0.25: node flux (four mass fluxes,
// src/serial/advec_mom.cpp:84-88 / :156-160) and node_mass_post (four cell
// masses density1 * post_vol, :93-96 / :165-168).
template <typename T> __device__ __forceinline__ T quarter_sum(T a, T b, T c, T d) { return T(0.25) * (a + b + c + d); }

// post_vol of a cell (:42-77): mom_sweep 1 vol + the y flux difference, 2
// vol + the x flux difference, 3 and 4 vol.
template <typename T> __device__ __forceinline__ T mom_post_vol(int mom_sweep, T vol, T lo, T hi) {
  return mom_sweep <= 2 ? vol + hi - lo : vol;
}

// node_mass_pre (:97-102 / :169-174) from node_mass_post and the node fluxes
// on the node's low and high side.
template <typename T> __device__ __forceinline__ T mom_node_mass_pre(T post, T nf_lo, T nf_hi) { return post - nf_lo + nf_hi; }

// sigma of a node's momentum flux (:120 / :192).
template <typename T> __device__ __forceinline__ T mom_sigma(T node_flux, T node_mass_pre_donor) {
  return sizeof(T) == sizeof(double) ? div_zero_num(fabs(node_flux), node_mass_pre_donor) : lim_div(fabs(node_flux), node_mass_pre_donor);
}

// Momentum flux of one velocity component (:121-133 / :193-205): vd, vu, vw
// the velocities at the donor, upwind and downwind nodes.
template <typename T> __device__ __forceinline__ T mom_flux_value(T sigma, T node_flux, T width, T dx_dif, T vd, T vu, T vw) {
  T lim = mom_limiter_value(vd - vu, vw - vd, sigma, width, dx_dif);
  return (vd + (T(1.0) - sigma) * lim) * node_flux;
}

// Velocity update (:139-144 / :211-216).
template <typename T> __device__ __forceinline__ T mom_update_value(T vel, T nm_pre, T nm_post, T mf_lo, T mf_hi) {
  return div_zero_num(vel * nm_pre + mf_lo - mf_hi, nm_post);
}

// xvel0 / yvel0 set: the sweep also does reset_field's node copy
// (src/serial/reset_field.cpp:42-49) of the velocities it writes, with its
// fold depth rfold -- the resident loop's second sweep, which then leaves
// xvel1 / yvel1 null: level 1 is not read again before the next step's
// accelerate rewrites it, and the loop restores it once at its end.
struct MomOut {
  void *xvel1, *yvel1;
  void *xvel0 = nullptr, *yvel0 = nullptr;
  int rfold = 0;
};

template <typename T, int DIR, int TY> struct MomLayout {
  static constexpr int LA = DIR == 1 ? TILE_X : TY; // nodes along the sweep
  static constexpr int LL = DIR == 1 ? TY : TILE_X; // lines across
  static constexpr int YH = DIR == 1 ? 1 : 2;       // staged rows above the tile
  static constexpr int BH = DIR == 1 ? TY + 2 : TY + 4;
  static constexpr int BOX = BOX_X * BH;
  static constexpr int BOXS = (BOX * (int)sizeof(T) + 127) / 128 * 128 / (int)sizeof(T); // 128-byte aligned stride
  static constexpr int NP = LA + 3;                  // positions 0 .. LA+2
  static constexpr int N_CM = NP * (LL + 1);         // cell masses: lines -1 .. LL-1
  static constexpr int N_W = NP * LL;                // node arrays
  static constexpr int SCRATCH = N_CM + 3 * N_W;    // cell masses, node flux, two momentum fluxes
  static constexpr int REGION = SCRATCH > 3 * BOXS ? SCRATCH : 3 * BOXS;
  static constexpr int GEO = 2 * BOXS + REGION; // the widths (fill_widths): celldx, then celldy
  static constexpr size_t SMEM = (size_t)(GEO + BOX_X + BH) * sizeof(T);
  // work-array indices: the thread-fastest coordinate is the contiguous one
  __device__ static constexpr int cm(int p, int lc) { return DIR == 1 ? lc * NP + p : p * (LL + 1) + lc; }
  __device__ static constexpr int w(int p, int l) { return DIR == 1 ? l * NP + p : p * LL + l; }
};

// EDGE = false: a tile whose every position lies inside the mesh's extents
// (no edge_tile), so the extent checks and the halo fold drop out.
// The tile's work once its boxes are staged at `sm` (L::SMEM bytes: the
// boxes, then the work arrays over the boxes the first stage consumes).
template <typename T, int DIR, int TY, bool EDGE, bool COMPACT = false>
__device__ __forceinline__ void advec_mom_compute(T *sm, const MomOut &out, const Mesh<T> &m, int vel_mask, int sweep, int fold, int bx,
                                                  int by) {
  using L = MomLayout<T, DIR, TY>;
  constexpr int LA = L::LA, LL = L::LL, NP = L::NP, YH = L::YH;
  const int mom_sweep = DIR + 2 * (sweep - 1);
  const int x0 = 2 + bx * TILE_X, y0 = 2 + by * TY;
  const T *U1 = sm, *V1 = sm + L::BOXS, *D1 = sm + 2 * L::BOXS, *MF = sm + 3 * L::BOXS, *VFO = sm + 4 * L::BOXS;
  T *region = sm + 2 * L::BOXS;
  T *s_cm = region, *s_nf = s_cm + L::N_CM, *s_mfu = s_nf + L::N_W, *s_mfv = s_mfu + L::N_W;
  const int na = DIR == 1 ? m.nx : m.ny, nlmax = DIR == 1 ? m.ny : m.nx;
  const int a0 = DIR == 1 ? x0 : y0, l0 = DIR == 1 ? y0 : x0;
  const int pitch = (int)m.pitch;
  constexpr int ST = DIR == 1 ? 1 : BOX_X; // box stride along the sweep
  constexpr int SL = DIR == 1 ? BOX_X : 1; // box stride across
  // box index of element (i, j)
  auto bidx = [&](int i, int j) { return (j - y0 + YH) * BOX_X + (i - x0 + HALO); };

  // (1) cell masses and node fluxes into registers, then into the region
  using ICM = Items<DIR, NP, LL + 1>; // cell masses: positions 0 .. LA+2, cell lines -1 .. LL-1
  using INF = Items<DIR, NP, LL>;     // node fluxes: positions 0 .. LA+2
  T r_cm[ICM::K] = {}, r_nf[INF::K] = {};
  ICM::each([&](int k, int p, int lc) {
    const int a = a0 - 2 + p, line = l0 - 1 + lc;
    if (!EDGE || (a >= 0 && a <= na + 3 && line >= 0 && line <= nlmax + 3)) {
      const int i = DIR == 1 ? a : line, j = DIR == 1 ? line : a;
      const int b = bidx(i, j);
      const T vol = sm[L::GEO + i - x0 + HALO] * sm[L::GEO + BOX_X + j - y0 + YH];
      // post_vol (:42-77): mom_sweep 1 vol + vfy difference, 2 vol + vfx difference, 3/4 vol
      const T pv = mom_sweep == 1 ? mom_post_vol(1, vol, VFO[b], VFO[b + BOX_X]) : mom_sweep == 2 ? mom_post_vol(2, vol, VFO[b], VFO[b + 1]) : vol;
      r_cm[k] = D1[b] * pv;
    }
  });
  INF::each([&](int k, int p, int l) {
    const int a = a0 - 2 + p, line = l0 + l;
    if (!EDGE || (line < nlmax + 3 && a >= 0 && a <= na + 3)) {
      const int b = DIR == 1 ? bidx(a, line) : bidx(line, a);
      // (:84-88 / :156-160) dir 1: mf(a, j-1) + mf(a, j) + mf(a+1, j-1) + mf(a+1, j); dir 2: mf(i-1, a) + mf(i, a) + mf(i-1, a+1) + mf(i, a+1)
      r_nf[k] = quarter_sum(MF[b - SL], MF[b], MF[b + ST - SL], MF[b + ST]);
    }
  });
  __syncthreads(); // density1, mass flux and volume flux boxes are dead from here on
  ICM::each([&](int k, int p, int lc) { s_cm[L::cm(p, lc)] = r_cm[k]; });
  INF::each([&](int k, int p, int l) { s_nf[L::w(p, l)] = r_nf[k]; });
  __syncthreads();

  // node_mass_post (:93-96 / :165-168) of node (p, l): cells (i, j-1), (i, j), (i-1, j-1), (i-1, j)
  auto node_mass_post = [&](int p, int l) -> T {
    if (DIR == 1) return quarter_sum(s_cm[L::cm(p, l)], s_cm[L::cm(p, l + 1)], s_cm[L::cm(p - 1, l)], s_cm[L::cm(p - 1, l + 1)]);
    return quarter_sum(s_cm[L::cm(p - 1, l + 1)], s_cm[L::cm(p, l + 1)], s_cm[L::cm(p - 1, l)], s_cm[L::cm(p, l)]);
  };

  // node_mass_pre (:97-102 / :169-174) of node (p, l), formed where it is
  // read (the donor of a momentum flux, the node of an update) rather than
  // stored: one barrier and one work array fewer
  auto node_mass_pre = [&](int p, int l) -> T { return mom_node_mass_pre(node_mass_post(p, l), s_nf[L::w(p - 1, l)], s_nf[L::w(p, l)]); };

  // (3) mom_flux (:108-133 / :180-205) over positions 1 .. LA+1
  // the sweep direction's cell widths: position a at celld[a]
  const T *celld = DIR == 1 ? sm + L::GEO + HALO - x0 : sm + L::GEO + BOX_X + YH - y0;
  Items<DIR, LA + 1, LL>::template each<!COMPACT>([&](int, int p, int l) {
    p += 1;
    const int a = a0 - 2 + p, line = l0 + l;
    if (EDGE && (line >= nlmax + 3 || a < 1 || a > na + 2)) return;
    const T nfv = s_nf[L::w(p, l)];
    int upwind, donor, downwind, dif;
    if (nfv < T(0.0)) {
      upwind = a + 2; donor = a + 1; downwind = a; dif = donor;
    } else {
      upwind = a - 1; donor = a; downwind = a + 1; dif = upwind;
    }
    const T sigma = mom_sigma(nfv, node_mass_pre(p + (donor - a), l));
    const T width = celld[a];
    const T dxd = celld[dif];
    const int b = DIR == 1 ? bidx(a, line) : bidx(line, a);
    const int bd = b + (donor - a) * ST, bu = b + (upwind - a) * ST, bw = b + (downwind - a) * ST;
    if (vel_mask & 1) s_mfu[L::w(p, l)] = mom_flux_value(sigma, nfv, width, dxd, U1[bd], U1[bu], U1[bw]);
    if (vel_mask & 2) s_mfv[L::w(p, l)] = mom_flux_value(sigma, nfv, width, dxd, V1[bd], V1[bu], V1[bw]);
  });
  __syncthreads();

  // (4) velocity update (:139-144 / :211-216) over positions 2 .. LA+1
  const bool do_fold = EDGE && fold;
  Items<DIR, LA, LL>::template each<!COMPACT>([&](int, int p, int l) {
    p += 2;
    const int a = a0 - 2 + p, line = l0 + l;
    if (EDGE && (line > nlmax + 2 || a > na + 2)) return;
    const int i = DIR == 1 ? a : line, j = DIR == 1 ? line : a;
    const int b = bidx(i, j);
    const T nmpost = node_mass_post(p, l), nmpre = mom_node_mass_pre(nmpost, s_nf[L::w(p - 1, l)], s_nf[L::w(p, l)]);
    const int g = gidx(pitch, i, j);
    if (vel_mask & 1) {
      T v = mom_update_value(U1[b], nmpre, nmpost, s_mfu[L::w(p - 1, l)], s_mfu[L::w(p, l)]);
      if (out.xvel1) {
        ((T *)out.xvel1)[g] = v;
        if (do_fold) fold_halo((T *)out.xvel1, m, halo_rule(XVEL1), fold, i, j, v);
      }
      if (out.xvel0) {
        ((T *)out.xvel0)[g] = v;
        if (EDGE && out.rfold) fold_halo((T *)out.xvel0, m, halo_rule(XVEL0), out.rfold, i, j, v);
      }
    }
    if (vel_mask & 2) {
      T v = mom_update_value(V1[b], nmpre, nmpost, s_mfv[L::w(p - 1, l)], s_mfv[L::w(p, l)]);
      if (out.yvel1) {
        ((T *)out.yvel1)[g] = v;
        if (do_fold) fold_halo((T *)out.yvel1, m, halo_rule(YVEL1), fold, i, j, v);
      }
      if (out.yvel0) {
        ((T *)out.yvel0)[g] = v;
        if (EDGE && out.rfold) fold_halo((T *)out.yvel0, m, halo_rule(YVEL0), out.rfold, i, j, v);
      }
    }
  });
}

// Fields the momentum sweep stages: the other direction's volume flux only for mom_sweep 1 and 2.
template <int DIR> __device__ __forceinline__ int mom_staged(int sweep) { return DIR + 2 * (sweep - 1) <= 2 ? 5 : 4; }

// One tile: staging, then the work (an edge tile keeps the extent checks;
// ALL_EDGE as for advec_cell_tile).
template <typename T, int DIR, int TY, bool ALL_EDGE = false>
__device__ __forceinline__ bool advec_mom_tile(TileCtx &cx, T *sm, const MapSet &ms, const MomOut &out, const Mesh<T> &m, int off,
                                               int vel_mask, int sweep, int fold, int bx, int by) {
  using L = MomLayout<T, DIR, TY>;
  const int x0 = 2 + bx * TILE_X, y0 = 2 + by * TY;
  stage_issue(cx, sm, ms, mom_staged<DIR>(sweep), L::BOXS, L::BH, off + x0 - HALO, y0 - L::YH);
  fill_widths<T>(m, x0, y0, L::YH, L::BH, DIR, sm + L::GEO, sm + L::GEO + BOX_X, nullptr, nullptr);
  if (!stage_wait(cx)) return false;
  if (ALL_EDGE || edge_tile(m.nx, m.ny, x0, y0, TY))
    advec_mom_compute<T, DIR, TY, true, ALL_EDGE>(sm, out, m, vel_mask, sweep, fold, bx, by);
  else
    advec_mom_compute<T, DIR, TY, false>(sm, out, m, vel_mask, sweep, fold, bx, by);
  return true;
}

template <typename T, int DIR, int TY>
__global__ void __launch_bounds__(256) kt_advec_mom(const __grid_constant__ Maps maps, MomOut out, Mesh<T> m, int off, int vel_mask,
                                                    int sweep, int fold, int *err) {
  extern __shared__ __align__(128) unsigned char smraw[];
  __shared__ uint64_t bar;
  TileCtx cx = tile_ctx(&bar, err);
  advec_mom_tile<T, DIR, TY>(cx, reinterpret_cast<T *>(smraw), map_set(maps, 5), out, m, off, vel_mask, sweep, fold, blockIdx.x, blockIdx.y);
}

} // namespace cb
