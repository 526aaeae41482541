// cb_batch_impl.cuh -- the persistent ensemble kernel (declared in
// cb_batch.h).  Included only by cb_fp64.cu and cb_fp32.cu, after
// cb_ops_impl.cuh, so the batch kernel is compiled with the same flags as
// the one-launch kernels of its precision and calls the same tile bodies:
// a deck advanced here is bit-identical to the same deck advanced by the
// one-launch kernels through the C ABI.
//
// Per deck, a lane does what HydroRun / the reference driver does for one
// chunk (driver/start.cpp:43-138, driver/hydro.cpp:46-223,
// driver/timestep.cpp:37-109, driver/advection.cpp:29-105), with every halo
// folded into its producer (meshes of at least 8 cells per side):
//   build_field, generate_chunk, ideal_gas, update_halo(10 fields, depth 2),
//   field_summary; then per step ideal_gas + viscosity + calc_dt as one pass
//   (lane-wide minimum), PdV predictor (+ ideal_gas, pressure halo, revert),
//   accelerate, PdV corrector, flux_calc, advec_cell / advec_mom (two sweeps,
//   the second writing reset_field's level-0 copies as it stores), and
//   field_summary every summary_frequency steps and at the end.
#pragma once

#include "cb_batch.h"
#include "cb_ops_impl.cuh"
#include "cb_sync.cuh"

namespace cb {

// Tile shapes of the batch kernel variants: the rows per tile of accelerate
// and flux_calc (the phases with the largest staged boxes) set the shared
// memory per CTA and with it the CTAs per SM.
// Rows per advection tile in both precisions: the decks are small, and more,
// smaller tiles spread a deck's phase more evenly over its lane.
constexpr int BATCH_ADV_TY = 8;
// Rows per tile of the fused ideal_gas + viscosity + calc_dt pass.
constexpr int BATCH_IVD_TY = 8;

template <int V> struct BatchTune;
template <> struct BatchTune<0> {
  static constexpr int ACC = 16, FLUX = 16, MINB = 3;
};
template <> struct BatchTune<1> {
  static constexpr int ACC = 8, FLUX = 8, MINB = 4;
};

template <typename T, int V> constexpr size_t batch_smem() {
  using BT = BatchTune<V>;
  auto mx = [](size_t a, size_t b) { return a > b ? a : b; };
  size_t s = ((size_t)4 * Box1<T, BATCH_IVD_TY>::BOXS + (sizeof(T) == sizeof(double) ? REST_MEMO_ELEMS : 0)) * sizeof(T);
  s = mx(s, pdv_smem<T>());
  s = mx(s, acc_smem<T, BT::ACC>());
  s = mx(s, flux_smem<T, BT::FLUX>());
  s = mx(s, CellLayout<T, 1, BATCH_ADV_TY>::SMEM);
  s = mx(s, CellLayout<T, 2, BATCH_ADV_TY>::SMEM);
  s = mx(s, MomLayout<T, 1, BATCH_ADV_TY>::SMEM);
  s = mx(s, MomLayout<T, 2, BATCH_ADV_TY>::SMEM);
  s = mx(s, (size_t)5 * 256 * sizeof(double)); // the summary's block reduction
  return s;
}

// Buffers of the double-buffered pairs during a step: advec_cell writes the
// updated density1/energy1 to the spares and the pair swaps, twice per step
// (so each step starts and ends with the identity mapping); advec_mom does
// the same for xvel1/yvel1.
struct BufMap {
  bool cell_swapped = false, mom_swapped = false;
  __device__ int of(int f) const {
    if (cell_swapped && f == DENSITY1) return 15;
    if (cell_swapped && f == ENERGY1) return 16;
    if (mom_swapped && f == XVEL1) return 17;
    if (mom_swapped && f == YVEL1) return 18;
    return f;
  }
  __device__ int spare(int s) const { // spare s of the pair (0, 1 cell; 2, 3 mom)
    if (s < 2) return cell_swapped ? (s == 0 ? DENSITY1 : ENERGY1) : 15 + s;
    return mom_swapped ? (s == 2 ? XVEL1 : YVEL1) : 15 + s;
  }
};

// The deck a lane works on, kept in shared memory (one copy per CTA, written
// by thread 0): the phases read it there instead of holding it in registers.
template <typename T> struct DeckCtx {
  const BatchDeck *D;
  Mesh<T> m;
  int rank, w;
  BufMap bm;
  MapSet ms; // tensor maps of the current phase (read by the staging thread only)
  Fields<T> F; // field pointers under the current buffer map (set_fields)

  __device__ T *base(int b) const { return (T *)D->buf[b] + D->off; }
  __device__ T *field(int f) const { return base(bm.of(f)); }
  __device__ void set_fields() {
    for (int f = 0; f < NUM_FIELDS; ++f) F.f[f] = f < 15 ? field(f) : nullptr;
  }
  // Sets ms to the maps of fields fl[0..n) (called by thread 0 before a phase's tiles).
  template <int H> __device__ void set_maps(int n, const int *fl) {
#pragma unroll
    for (int k = 0; k < 8; ++k) ms.m[k] = k < n ? &D->maps[bm.of(fl[k]) * NUM_BOX_H + box_slot<H>()] : nullptr;
  }
};

// The lane's share of a phase over nt tiles: tiles rank, rank + w, ...
#define CB_LANE_TILES(ctx, nt, tx_, body)                                                                                                    \
  for (int _t = (ctx).rank; _t < (nt); _t += (ctx).w) {                                                                                     \
    const int bx = _t % (tx_), by = _t / (tx_);                                                                                              \
    if (!(body)) return false;                                                                                                               \
  }

// The advection phases and the summary are called, not inlined: each gets
// its own register allocation instead of sharing the whole kernel's, which
// spills less (measured 2 % faster on the 512-deck ensemble).
//
// Code size: the kernel holds every phase, and its code outgrew the
// instruction caches (ncu: "no instruction" the second stall).  So the
// advection tiles are compiled in their edge form only (ALL_EDGE; 512-deck
// ensemble 279 -> 241 ms FP64, 193 -> 168 ms FP32), their item loops and the
// row loops of ideal_gas + viscosity + calc_dt, accelerate and flux_calc are
// kept as loops instead of unrolled (then 187 ms / 129 ms with the autotuner's
// wider choice of cells per CTA).
template <typename T, int DIR>
__device__ __noinline__ bool batch_advec_cell(TileCtx &cx, T *sm, DeckCtx<T> &d, int sweep, bool reset = false) {
  constexpr int TY = BATCH_ADV_TY;
  using L = CellLayout<T, DIR, TY>;
  const int fl[4] = {DENSITY1, ENERGY1, VOL_FLUX_X, VOL_FLUX_Y};
  if (threadIdx.x == 0 && threadIdx.y == 0) d.template set_maps<L::BH>(4, fl);
  const MapSet &ms = d.ms;
  CellOut out{d.base(d.bm.spare(0)), d.base(d.bm.spare(1)), d.field(DIR == 1 ? MASS_FLUX_X : MASS_FLUX_Y)};
  if (reset) { out.density0 = d.field(DENSITY0); out.energy0 = d.field(ENERGY0); out.rfold = 1; }
  const int tx = (d.m.nx + TILE_X - 1) / TILE_X, nt = tx * ((d.m.ny + TY - 1) / TY);
  CB_LANE_TILES(d, nt, tx, (advec_cell_tile<T, DIR, TY, true>(cx, sm, ms, out, d.m, d.D->off, sweep, 2, bx, by)));
  return true;
}

template <typename T, int DIR>
__device__ __noinline__ bool batch_advec_mom(TileCtx &cx, T *sm, DeckCtx<T> &d, int sweep, int fold, bool reset = false) {
  constexpr int TY = BATCH_ADV_TY;
  using L = MomLayout<T, DIR, TY>;
  const int mom_sweep = DIR + 2 * (sweep - 1);
  const int mf = DIR == 1 ? MASS_FLUX_X : MASS_FLUX_Y;
  const int fl[5] = {XVEL1, YVEL1, DENSITY1, mf, mom_sweep == 1 ? VOL_FLUX_Y : VOL_FLUX_X};
  if (threadIdx.x == 0 && threadIdx.y == 0) d.template set_maps<L::BH>(mom_sweep <= 2 ? 5 : 4, fl);
  const MapSet &ms = d.ms;
  MomOut out{d.base(d.bm.spare(2)), d.base(d.bm.spare(3))};
  if (reset) { out.xvel0 = d.field(XVEL0); out.yvel0 = d.field(YVEL0); out.rfold = 1; }
  const int tx = (d.m.nx + 1 + TILE_X - 1) / TILE_X, nt = tx * ((d.m.ny + 1 + TY - 1) / TY);
  CB_LANE_TILES(d, nt, tx, (advec_mom_tile<T, DIR, TY, true>(cx, sm, ms, out, d.m, d.D->off, 3, sweep, fold, bx, by)));
  return true;
}

// field_summary (src/serial/field_summary.cpp:44-104): the lane's cells in
// 32 x 8 tiles, a fixed-order block reduction, one partial per CTA, and the
// lane's first CTA adds the partials in CTA order into the record.
template <typename T>
__device__ __noinline__ bool batch_summary(T *sm, DeckCtx<T> &d, unsigned *ctr, int *abort, int step, double time, int &nsum) {
  const int tid = threadIdx.y * blockDim.x + threadIdx.x;
  const Fields<T> &F = d.F;
  const T gm1 = (T)d.D->gm1;
  double s[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
  const int tx = (d.m.nx + PW_X - 1) / PW_X, nt = tx * ((d.m.ny + PW_Y - 1) / PW_Y);
  for (int t = d.rank; t < nt; t += d.w) {
    const int i = 2 + (t % tx) * PW_X + (tid & 31), j = 2 + (t / tx) * PW_Y + (tid >> 5);
    if (i < d.m.nx + 2 && j < d.m.ny + 2) summary_cell(F, d.m, gm1, i, j, s);
  }
  double *red = reinterpret_cast<double *>(sm);
  __syncthreads(); // sm may still hold the previous phase's boxes
  for (int q = 0; q < 5; ++q) red[q * 256 + tid] = s[q];
  __syncthreads();
  for (int h = 128; h > 0; h >>= 1) {
    if (tid < h)
      for (int q = 0; q < 5; ++q) red[q * 256 + tid] += red[q * 256 + tid + h];
    __syncthreads();
  }
  if (tid == 0)
    for (int q = 0; q < 5; ++q) d.D->partials[d.rank * 5 + q] = red[q * 256];
  if (!lane_sync(ctr, d.w, abort)) return false;
  if (d.rank == 0 && tid == 0) {
    double tot[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
    for (int r = 0; r < d.w; ++r)
      for (int q = 0; q < 5; ++q) tot[q] += ((volatile double *)d.D->partials)[r * 5 + q];
    if (nsum < d.D->max_summaries) {
      double *rec = d.D->summaries + (size_t)nsum * BATCH_RECORD;
      rec[0] = step;
      rec[1] = time;
      for (int q = 0; q < 5; ++q) rec[2 + q] = tot[q];
    }
  }
  ++nsum;
  return true;
}

// One deck from build_field to its end.  Returns false when a wait gave up
// (the lane then stops); a deck that ends early for physical reasons (dt
// below dtmin) returns true with its status set.
template <typename T, int V>
__device__ __forceinline__ bool batch_run_deck(TileCtx &cx, T *sm, BatchDeck *D, int rank, int w, unsigned *ctr, int *abort) {
  using BT = BatchTune<V>;
  constexpr int N = Vec16<T>::N;
  __shared__ DeckCtx<T> d;
  const int tid = threadIdx.y * blockDim.x + threadIdx.x;
  __syncthreads(); // the previous deck's readers are done with d
  if (tid == 0) {
  d.D = D;
  d.rank = rank;
  d.w = w;
  d.bm = BufMap{};
  d.m.nx = D->nx;
  d.m.ny = D->ny;
  d.m.pitch = D->pitch;
  d.m.celldx = D->geom_d[CELLDX];
  d.m.celldy = D->geom_d[CELLDY];
  d.m.vertexdx = D->geom_d[VERTEXDX];
  d.m.vertexdy = D->geom_d[VERTEXDY];
  d.m.celldx_t = (const T *)D->geom_t[CELLDX];
  d.m.celldy_t = (const T *)D->geom_t[CELLDY];
  d.m.rcelldx = D->rgeom;
  d.m.rcelldy = D->rgeom + D->geom_len;
  d.m.rvertexdx = D->rgeom + 2 * D->geom_len;
  d.m.rvertexdy = D->rgeom + 3 * D->geom_len;
  d.set_fields();
  }
  __syncthreads();
  const Mesh<T> &m = d.m;
  const int off = D->off;
  const T gm1 = (T)D->gm1;
  const int ptx = tid & 31, pty = tid >> 5; // thread of a 32 x 8 pointwise block
  const int lt = rank * 256 + tid, lstride = w * 256;
  int status = DECK_PENDING;
  auto finish = [&](int st, int steps, double time, int nsum) {
    if (rank == 0 && tid == 0) {
      D->status = st;
      D->steps = steps;
      D->time = time;
      D->nsummaries = nsum;
    }
  };
#define CB_SYNC()                                                                                                                            \
  do {                                                                                                                                       \
    if (!lane_sync(ctr, w, abort)) {                                                                                                         \
      finish(DECK_SYNC_FAIL, step, time, nsum);                                                                                              \
      return false;                                                                                                                          \
    }                                                                                                                                        \
  } while (0)
#define CB_PHASE(expr)                                                                                                                       \
  do {                                                                                                                                       \
    if (!(expr)) {                                                                                                                           \
      finish(DECK_STAGE_FAIL, step, time, nsum);                                                                                             \
      return false;                                                                                                                          \
    }                                                                                                                                        \
  } while (0)
  int step = 0, nsum = 0;
  double time = 0.0;

  // build_field (src/serial/build_field.cpp:29-180): every buffer to zero
  {
    const size_t nv = D->buf_bytes / 16;
    for (int b = 0; b < BATCH_BUF; ++b) {
      uint4 *p = (uint4 *)D->buf[b];
      for (size_t e = lt; e < nv; e += lstride) p[e] = make_uint4(0u, 0u, 0u, 0u);
    }
    if (rank == 0 && tid < 3) D->dt_slots[tid] = (unsigned long long)__double_as_longlong(g_big);
  }
  CB_SYNC();
  // generate_chunk over the full extents, then ideal_gas on level 0
  {
    const Fields<T> &F = d.F;
    const int ex = m.nx + 5, ey = m.ny + 5;
    for (int e = lt; e < ex * ey; e += lstride)
      generate_element(F, m, D->states, D->nstates, D->geom_d[CELLX], D->geom_d[CELLY], D->geom_d[VERTEXX], D->geom_d[VERTEXY], e % ex,
                       e / ex);
  }
  CB_SYNC();
  {
    const Fields<T> &F = d.F;
    const int gx = ((m.nx + N - 1) / N + PW_X - 1) / PW_X, gy = (m.ny + PW_Y - 1) / PW_Y;
    for (int vb = rank; vb < gx * gy; vb += w) ideal_gas_block(F, m, 0, gm1, 0, vb % gx, vb / gx, ptx, pty);
  }
  CB_SYNC();
  // update_halo of density0/1, energy0/1, pressure, viscosity, xvel0/1, yvel0/1 at depth 2 (driver/start.cpp:103-118):
  // bottom/top of every column, then left/right of every row
  {
    const int hf[10] = {DENSITY0, ENERGY0, PRESSURE, VISCOSITY, DENSITY1, ENERGY1, XVEL0, YVEL0, XVEL1, YVEL1};
    const Fields<T> &F = d.F;
    const int len = (m.nx > m.ny ? m.nx : m.ny) + 5 + 4;
    for (int pass = 0; pass < 2; ++pass) {
      for (int e = lt; e < 10 * len; e += lstride) halo_fill(F, m, hf[e / len], 2, pass, e % len);
      CB_SYNC();
    }
  }
  if (!batch_summary(sm, d, ctr, abort, 0, 0.0, nsum)) {
    finish(DECK_SYNC_FAIL, step, time, nsum);
    return false;
  }

  double dt = D->dtinit, dtold = D->dtinit;
  bool advect_x = true;
  while (true) {
    ++step;
    unsigned long long *slot = D->dt_slots + step % 3;
    {
      constexpr int TY = BATCH_IVD_TY;
      const int fl[4] = {DENSITY0, ENERGY0, XVEL0, YVEL0};
      if (tid == 0) d.template set_maps<Box1<T, TY>::BH>(4, fl);
      const MapSet &ms = d.ms;
      const int tx = (m.nx + TILE_X - 1) / TILE_X, nt = tx * ((m.ny + TY - 1) / TY);
      double vmin = g_big;
      // the at-rest memo: FP64 in shared memory after the staged boxes (in registers it spills), FP32 in registers
      using Memo = std::conditional_t<sizeof(T) == sizeof(double), RestMemoShared<T>, RestMemo<T>>;
      Memo memo = make_memo<Memo>(sm + 4 * Box1<T, TY>::BOXS);
      for (int t = rank; t < nt; t += w)
        CB_PHASE((ig_visc_dt_tile<T, Memo, TY, true>(cx, sm, ms, d.field(PRESSURE), d.field(SOUNDSPEED), d.field(VISCOSITY), m, off, D->k,
                                                      gm1, 1, 1, t % tx, t / tx, vmin, memo)));
      block_min_to(vmin, slot);
    }
    CB_SYNC();
    const double dtlp = __longlong_as_double((long long)*(volatile unsigned long long *)slot);
    if (rank == 0 && tid == 0) D->dt_slots[(step + 1) % 3] = (unsigned long long)__double_as_longlong(g_big);
    dt = g_big;
    if (dtlp <= dt) dt = dtlp;
    double mm = dtold * D->dtrise;
    mm = mm < dt ? mm : dt;
    dt = D->dtmax < mm ? D->dtmax : mm;
    if (rank == 0 && tid == 0 && step - 1 < D->max_steps) D->dt_trace[step - 1] = dt;
    if (dt < D->dtmin) {
      status = DECK_SMALL_DT;
      break;
    }
    dtold = dt;
    // PdV predictor with ideal_gas, the pressure halo and revert (src/serial/PdV.cpp:92-133)
    {
      const int fl[4] = {XVEL0, YVEL0, XVEL1, YVEL1};
      if (tid == 0) d.template set_maps<Box1<T, PDV_TY>::BH>(2, fl);
      const MapSet &ms = d.ms;
      const PdvIn in{d.field(DENSITY0), d.field(ENERGY0), d.field(PRESSURE), d.field(VISCOSITY)};
      const PdvOut out{d.field(DENSITY1), d.field(ENERGY1), d.field(PRESSURE), d.field(SOUNDSPEED)};
      const int tx = (m.nx + TILE_X - 1) / TILE_X, nt = tx * ((m.ny + PDV_TY - 1) / PDV_TY);
      for (int t = rank; t < nt; t += w) CB_PHASE(pdv_tile(cx, sm, ms, in, out, m, off, 1, (T)dt, 1, gm1, 1, t % tx, t / tx));
    }
    CB_SYNC();
    {
      const int fl[5] = {DENSITY0, PRESSURE, VISCOSITY, XVEL0, YVEL0};
      if (tid == 0) d.template set_maps<Box1<T, BT::ACC>::BH>(5, fl);
      const MapSet &ms = d.ms;
      const int tx = (m.nx + 1 + TILE_X - 1) / TILE_X, nt = tx * ((m.ny + 1 + BT::ACC - 1) / BT::ACC);
      for (int t = rank; t < nt; t += w)
        CB_PHASE((accelerate_tile<T, BT::ACC, true>(cx, sm, ms, d.field(XVEL1), d.field(YVEL1), m, off, (T)dt, 2, t % tx, t / tx)));
    }
    CB_SYNC();
    {
      const int fl[4] = {XVEL0, YVEL0, XVEL1, YVEL1};
      if (tid == 0) d.template set_maps<Box1<T, PDV_TY>::BH>(4, fl);
      const MapSet &ms = d.ms;
      const PdvIn in{d.field(DENSITY0), d.field(ENERGY0), d.field(PRESSURE), d.field(VISCOSITY)};
      const PdvOut out{d.field(DENSITY1), d.field(ENERGY1), d.field(PRESSURE), d.field(SOUNDSPEED)};
      const int tx = (m.nx + TILE_X - 1) / TILE_X, nt = tx * ((m.ny + PDV_TY - 1) / PDV_TY);
      for (int t = rank; t < nt; t += w) CB_PHASE(pdv_tile(cx, sm, ms, in, out, m, off, 0, (T)dt, 0, gm1, 2, t % tx, t / tx));
    }
    CB_SYNC();
    {
      const int fl[4] = {XVEL0, YVEL0, XVEL1, YVEL1};
      if (tid == 0) d.template set_maps<Box1<T, BT::FLUX>::BH>(4, fl);
      const MapSet &ms = d.ms;
      const int tx = (m.nx + 1 + TILE_X - 1) / TILE_X, nt = tx * ((m.ny + 1 + BT::FLUX - 1) / BT::FLUX);
      for (int t = rank; t < nt; t += w)
        CB_PHASE((flux_calc_tile<T, BT::FLUX, true>(cx, sm, ms, d.field(VOL_FLUX_X), d.field(VOL_FLUX_Y), m, off, (T)dt, 2, t % tx, t / tx)));
    }
    CB_SYNC();
    // advection (driver/advection.cpp:29-105): the two advec_mom calls of a sweep in one pass
    const int dir1 = advect_x ? 1 : 2, dir2 = advect_x ? 2 : 1;
    // the buffer map changes after each lane barrier, by thread 0, before anyone reads it again
    CB_PHASE((dir1 == 1 ? batch_advec_cell<T, 1>(cx, sm, d, 1) : batch_advec_cell<T, 2>(cx, sm, d, 1)));
    CB_SYNC();
    if (tid == 0) d.bm.cell_swapped = true, d.set_fields();
    __syncthreads();
    CB_PHASE((dir1 == 1 ? batch_advec_mom<T, 1>(cx, sm, d, 1, 2) : batch_advec_mom<T, 2>(cx, sm, d, 1, 2)));
    CB_SYNC();
    if (tid == 0) d.bm.mom_swapped = true, d.set_fields();
    __syncthreads();
    // the second sweep also stores reset_field's level-0 copies (src/serial/reset_field.cpp:27-70), halo folded
    CB_PHASE((dir2 == 1 ? batch_advec_cell<T, 1>(cx, sm, d, 2, true) : batch_advec_cell<T, 2>(cx, sm, d, 2, true)));
    CB_SYNC();
    if (tid == 0) d.bm.cell_swapped = false, d.set_fields();
    __syncthreads();
    CB_PHASE((dir2 == 1 ? batch_advec_mom<T, 1>(cx, sm, d, 2, 0, true) : batch_advec_mom<T, 2>(cx, sm, d, 2, 0, true)));
    CB_SYNC();
    if (tid == 0) d.bm.mom_swapped = false, d.set_fields();
    __syncthreads();
    // driver/hydro.cpp:87-111
    advect_x = !advect_x;
    time += dt;
    const bool done = time + g_small > D->end_time || step >= D->end_step;
    if (D->summary_frequency != 0 && step % D->summary_frequency == 0)
      if (!batch_summary(sm, d, ctr, abort, step, time, nsum)) {
        finish(DECK_SYNC_FAIL, step, time, nsum);
        return false;
      }
    if (done) {
      if (!batch_summary(sm, d, ctr, abort, step, time, nsum)) {
        finish(DECK_SYNC_FAIL, step, time, nsum);
        return false;
      }
      status = DECK_DONE;
      break;
    }
  }
#undef CB_SYNC
#undef CB_PHASE
  finish(status, step, time, nsum);
  return true;
}

template <typename T, int V>
__global__ void __launch_bounds__(256, BatchTune<V>::MINB) kb_ensemble(const __grid_constant__ BatchLaunch a) {
  extern __shared__ __align__(128) unsigned char smraw[];
  __shared__ uint64_t bar;
  T *sm = reinterpret_cast<T *>(smraw);
  TileCtx cx = tile_ctx(&bar, a.err);
  const bool lead = threadIdx.x == 0 && threadIdx.y == 0;
  for (int k = 0; k < a.nlevels; ++k) {
    const int W = a.level[4 * k], q0 = a.level[4 * k + 1], nq = a.level[4 * k + 2], s0 = a.level[4 * k + 3];
    const int lane = (int)blockIdx.x / W, rank = (int)blockIdx.x % W;
    if (lane >= (int)gridDim.x / W) continue; // no full lane of this width here
    unsigned *ctr = a.lane_sync + s0 + lane;
    volatile int *slot = a.lane_deck + s0 + lane;
    while (true) {
      // the lane's first CTA takes the next deck of the queue; the others read it after the barrier
      // (every CTA of the lane has passed at least one lane barrier since it read the previous one)
      if (rank == 0 && lead) *slot = (int)atomicAdd(a.next + k, 1u);
      if (!lane_sync(ctr, W, a.abort)) return;
      const int q = *slot;
      if (q >= nq) break;
      if (!batch_run_deck<T, V>(cx, sm, a.decks + a.queue[q0 + q], rank, W, ctr, a.abort)) return;
    }
  }
}

template <typename T> size_t BatchOps<T>::smem_bytes(int variant) { return variant == 0 ? batch_smem<T, 0>() : batch_smem<T, 1>(); }

template <typename T> cudaError_t BatchOps<T>::occupancy(int variant, int *per_sm) {
  const size_t smem = smem_bytes(variant);
  cudaError_t e;
  if (variant == 0) {
    if ((e = cudaFuncSetAttribute(kb_ensemble<T, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem)) != cudaSuccess) return e;
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(per_sm, kb_ensemble<T, 0>, 256, smem);
  }
  if ((e = cudaFuncSetAttribute(kb_ensemble<T, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem)) != cudaSuccess) return e;
  return cudaOccupancyMaxActiveBlocksPerMultiprocessor(per_sm, kb_ensemble<T, 1>, 256, smem);
}

template <typename T> cudaError_t BatchOps<T>::launch(int variant, const BatchLaunch &a, int grid, cudaStream_t s) {
  const size_t smem = smem_bytes(variant);
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)grid);
  cfg.blockDim = dim3(64, 4);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative; // every CTA of a lane must be resident while the others wait for it
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  if (variant == 0) return cudaLaunchKernelEx(&cfg, kb_ensemble<T, 0>, a);
  return cudaLaunchKernelEx(&cfg, kb_ensemble<T, 1>, a);
}

} // namespace cb
