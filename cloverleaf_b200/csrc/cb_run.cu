// cb_run.cu -- cb_run: the hydro loop of driver/hydro.cpp:53-111 for one
// chunk, resident on the device from its first step to its last.
//
// The loop is one CUDA graph: a WHILE conditional node whose body is one
// hydro step -- the phase launches the C ABI makes for the driver's call
// sequence (driver/timestep.cpp:37-109, driver/advection.cpp:29-105,
// src/serial/PdV.cpp:92-133) -- with dt computed, clamped and kept on the
// device.  The body's advection is a two-way IF node (x sweep first or y
// sweep first, as advect_x says), and a second IF node records the field
// summary every summary_frequency steps and at the end.  Four one-thread
// kernels carry the driver's scalar logic (the dt clamp of
// driver/timestep.cpp:75-96; time, the end test and the summaries of
// driver/hydro.cpp:87-111) and set the conditions from the device.  The
// host waits once, at the end.
//
// The run's entry state and constants live in device memory (RunParams),
// written before each launch, so the instantiated graph is kept by the
// chunk and launched again by the next cb_run that finds the chunk as the
// graph was captured for (RunKey: the buffer map, the halo freshness, the
// options and the constants its launches carry).
//
// The update_halo calls of the sequence follow the chunk's halo freshness
// exactly as cb_update_halo does.  The body is captured from the state the
// freshness settles in after the first steps; a pass that the first step
// would make and the settled body does not (a mass flux that no sweep has
// written yet) runs once before the loop, which is exact because nothing
// writes that field between the loop's start and the pass.
//
// Compiled with -fmad=false like the FP64 kernels: the dt clamp and the time
// sum round exactly as the host-driven loop's.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstddef>
#include <cstring>
#include <initializer_list>
#include <memory>
#include <new>
#include <string>
#include <vector>

#include "../../include/cloverb200.h"
#include "cb_chunk.h"
#include "cb_ops.h"

namespace cb {
int set_last_error(int code, const std::string &msg);
// Defined in cb_api.cu: runs the phase calls call fusion holds back.
cudaError_t run_pending_calls(cb_chunk *c);
} // namespace cb

using namespace cb;

namespace {

int fail(int code, const std::string &m) { return set_last_error(code, m); }

int cuda_fail(cudaError_t e, const char *where) {
  return fail(CB_ECUDA, std::string(where) + ": " + cudaGetErrorName(e) + ": " + cudaGetErrorString(e));
}

// ---------------------------------------------------------------------------
// device side: the scalar state of the run and its one-thread kernels

struct RunState {
  double dt, dtold, time;
  int step, nsum, sum_runs, small, advect_x, records_due;
  int last; // the step under way is the run's last (k_run_end will stop the loop)
};

struct RunConsts {
  double dtmin, dtmax, dtrise, end_time;
  int end_step, summary_frequency, last_step, step0, max_records;
};

// What a launch of the run's graph starts from: the constants and the entry
// state, copied to the device before each launch.
struct RunParams {
  RunConsts k;
  double time, dtold;
  int step, advect_x;
};

constexpr int RUN_KERNELS_PER_STEP = 3; // k_run_begin, k_run_dt, k_run_end

__global__ void k_run_init(RunState *s, const RunParams *p) {
  s->dt = p->dtold;
  s->dtold = p->dtold;
  s->time = p->time;
  s->step = p->step;
  s->nsum = 0;
  s->sum_runs = 0;
  s->small = 0;
  s->advect_x = p->advect_x;
  s->records_due = 0;
}

// Start of a step: the step counter, and calc_dt's minimum set to g_big.
__global__ void k_run_begin(RunState *s, unsigned long long *dt_bits) {
  s->step += 1;
  *dt_bits = (unsigned long long)__double_as_longlong(g_big);
}

// dt of the step from calc_dt's minimum (driver/timestep.cpp:75-96), kept on
// the device for the phases that read it; the advection branch of the step.
__global__ void k_run_dt(RunState *s, const unsigned long long *dt_bits, const RunParams *p, double *dt_dev, double *trace,
                         cudaGraphConditionalHandle hadv) {
  const RunConsts &k = p->k;
  const double dtlp = __longlong_as_double((long long)*dt_bits);
  double dt = g_big;
  if (dtlp <= dt) dt = dtlp;
  double m = s->dtold * k.dtrise;
  m = m < dt ? m : dt;
  dt = k.dtmax < m ? k.dtmax : m;
  if (dt < k.dtmin) s->small = 1;
  // k_run_end's stop test, with the same time sum
  s->last = s->time + dt + g_small > k.end_time || s->step >= k.end_step || s->step >= k.last_step || s->small;
  s->dt = dt;
  s->dtold = dt;
  *dt_dev = dt;
  trace[s->step - k.step0 - 1] = dt; // step0 < step <= last_step = step0 + (trace length)
  cudaGraphSetConditional(hadv, s->advect_x ? 1u : 0u);
}

// End of a step (driver/hydro.cpp:87-111): direction toggle, time, the end
// test, the summaries due, and whether the loop goes on.
__global__ void k_run_end(RunState *s, const RunParams *p, cudaGraphConditionalHandle hsum, cudaGraphConditionalHandle hloop) {
  const RunConsts &k = p->k;
  s->advect_x = !s->advect_x;
  s->time += s->dt;
  const bool complete = s->time + g_small > k.end_time || s->step >= k.end_step;
  const bool stop = complete || s->step >= k.last_step || s->small;
  int due = 0;
  if (!s->small) {
    if (k.summary_frequency != 0 && s->step % k.summary_frequency == 0) ++due;
    if (complete) ++due;
  }
  s->records_due = due;
  cudaGraphSetConditional(hsum, due > 0 ? 1u : 0u);
  cudaGraphSetConditional(hloop, stop ? 0u : 1u);
}

// The summary record(s) of the step: step, time and the five sums
// (the report line of driver/field_summary.cpp).
__global__ void k_run_record(RunState *s, const double *sums, double *records, const RunParams *p) {
  const RunConsts &k = p->k;
  for (int r = 0; r < s->records_due; ++r) {
    if (s->nsum < k.max_records) {
      double *rec = records + 7 * (size_t)s->nsum;
      rec[0] = s->step;
      rec[1] = s->time;
      for (int q = 0; q < 5; ++q) rec[2 + q] = sums[q];
    }
    s->nsum += 1;
  }
  s->sum_runs += 1;
}

// ---------------------------------------------------------------------------
// host side: the step's call sequence, as launches or as a freshness model

enum : int { D0 = DENSITY0, D1 = DENSITY1, E0 = ENERGY0, E1 = ENERGY1, P = PRESSURE, Q = VISCOSITY, SS = SOUNDSPEED };
enum : int { U0 = XVEL0, U1 = XVEL1, V0 = YVEL0, V1 = YVEL1, VFX = VOL_FLUX_X, VFY = VOL_FLUX_Y, MFX = MASS_FLUX_X, MFY = MASS_FLUX_Y };

struct Pass {
  int pos, field, depth;
  unsigned written_before; // fields the step had written when the pass ran
  bool operator==(const Pass &o) const { return pos == o.pos && field == o.field && depth == o.depth; }
};

// One step's C-ABI call sequence (the calls of HydroRun.hydro_step in
// cloverleaf_b200/hydro.py and of the C++ model glue).  With emit set the
// phases are launched on c.stream; either way the halo freshness moves as
// cb_api.cu's bookkeeping moves it, the host buffer map swaps as the
// double-buffered phases swap it, and every update_halo pass is logged.
template <typename T> struct Seq {
  Chunk &c;
  bool emit;
  bool fold;
  DtConsts dk;
  int fresh[15];
  int pos = 0;
  unsigned written = 0;
  std::vector<Pass> passes;
  cudaError_t err = cudaSuccess;
  // fused emission (only with every producer folding): ideal_gas +
  // viscosity + calc_dt in one pass, the PdV predictor + accelerate + the
  // PdV corrector + flux_calc in one pass, and reset_field done by the
  // second sweeps; the freshness moves exactly as unfused
  bool fuse = false;
  // fused: the run's last-step flag on the device; the Lagrangian pass
  // stores the predicted pressure and soundspeed in that step only, the
  // fused x sweep the mass flux of the tiles the edge strip does not read
  // (all rewritten unread otherwise); the fused ideal_gas pass stores
  // neither pressure nor soundspeed: the Lagrangian pass forms the pressure
  // from density0 and energy0 as the ideal_gas pass would store it
  const int *last_flag = nullptr;

  Seq(Chunk &ch, bool e, bool f, const DtConsts &k) : c(ch), emit(e), fold(f), dk(k) { std::memcpy(fresh, ch.halo_fresh, sizeof fresh); }

  int dep(int d) const { return fold ? d : 0; }    // the halo_depth argument of a folding producer
  int eff(int d) const { return c.can_fold() ? d : 0; } // effective_fold of cb_api.cu
  void run(cudaError_t e) {
    if (err == cudaSuccess && e != cudaSuccess) err = e;
  }
  void wrote(std::initializer_list<int> fs, int depth) {
    for (int f : fs) {
      fresh[f] = depth;
      written |= 1u << f;
    }
    ++pos;
  }
  // cb_update_halo
  void halo(std::initializer_list<int> fs, int depth) {
    HaloJob job{};
    for (int f : fs) {
      if (c.can_fold() && fresh[f] >= depth) continue;
      job.field[job.nfields++] = f;
    }
    for (int k = 0; k < job.nfields; ++k) {
      passes.push_back(Pass{pos, job.field[k], depth, written});
      fresh[job.field[k]] = std::max(fresh[job.field[k]], depth);
    }
    ++pos;
    if (emit && job.nfields) run(Ops<T>::update_halo(c, job, depth));
  }
  // driver/timestep.cpp:37-73 up to calc_dt
  void timestep_front() {
    const int fi = eff(dep(1));
    if (emit && !fuse) run(Ops<T>::ideal_gas(c, 0, fi));
    wrote({P}, fi);
    wrote({SS}, 0);
    halo({P, E0, D0, U0, V0}, 1);
    const int fv = eff(dep(1));
    if (emit && !fuse) run(Ops<T>::viscosity(c, fv));
    wrote({Q}, fv);
    halo({Q}, 1); // (no pass when fused: q is fresh to depth 1)
    // fused: ideal_gas, viscosity and calc_dt in one pass here (the halo
    // passes between them are none: density0 / energy0 and q are fresh),
    // the pressure written to its second buffer (see lagrange)
    if (fuse) swap_pressure();
    if (emit) run(fuse ? Ops<T>::ig_visc_dt(c, dk, fi, fv, last_flag == nullptr, last_flag == nullptr) : Ops<T>::calc_dt(c, dk));
    ++pos;
  }
  // Fused, the predicted pressure goes to the other of two buffers: the pass
  // that makes it reads the previous pressure of cells other tiles predict.
  // ideal_gas swaps as well, so a step leaves the buffer map as it found it.
  void swap_pressure() { std::swap(c.fbuf[P], c.sbuf[4]); }
  // driver/hydro.cpp:69-75 and src/serial/PdV.cpp:92-133, dt from the device
  void lagrange() {
    const int fp = eff(1); // the predictor makes its own pressure halo
    const int fa = eff(dep(2));
    const int fc = eff(dep(2));
    const int ff = eff(dep(2));
    if (fuse) {
      // fused: the whole Lagrangian step in one pass
      if (emit) run(Ops<T>::lagrange(c, c.spare_base(4), 0.0, fp, fa, fc, ff, false, last_flag, last_flag != nullptr));
      swap_pressure();
    } else if (emit) {
      run(Ops<T>::pdv(c, 1, 0.0, 1, fp));
      if (fp == 0) {
        HaloJob job{};
        job.nfields = 1;
        job.field[0] = P;
        run(Ops<T>::update_halo(c, job, 1));
      }
    }
    wrote({P}, fp);
    wrote({SS, D1, E1}, 0);
    if (emit && !fuse) run(Ops<T>::accelerate(c, 0.0, fa));
    wrote({U1, V1}, fa);
    if (emit && !fuse) run(Ops<T>::pdv(c, 0, 0.0, 0, fc));
    wrote({D1, E1}, fc);
    if (emit && !fuse) run(Ops<T>::flux_calc(c, 0.0, ff));
    wrote({VFX, VFY}, ff);
  }
  // fold depth of reset_field, which a fused second sweep does
  int reset_tail(bool last) const { return fuse && last ? eff(dep(1)) : -1; }
  // cb_advec_cell with its buffer swap.  A fused second sweep writes the new
  // energy to energy0 only: energy1 is next read after the following step's
  // PdV has rewritten it, and the loop restores it at its end
  // (restore_level1); the swap still renames the buffers, so the body leaves
  // the buffer map as it found it.
  void cell(int sweep, int dir, bool last = false) {
    const int f = eff(dep(2));
    if (emit) run(Ops<T>::advec_cell(c, sweep, dir, f, c.spare_base(0), fuse && last ? nullptr : c.spare_base(1), reset_tail(last)));
    std::swap(c.fbuf[DENSITY1], c.sbuf[0]);
    std::swap(c.fbuf[ENERGY1], c.sbuf[1]);
    wrote({D1, E1, dir == 1 ? MFX : MFY}, f);
  }
  // cb_advec_mom of both velocities with its buffer swaps; a fused second
  // sweep writes the velocities to level 0 only (as the energy above)
  void mom(int sweep, int dir, int depth, bool last = false) {
    const int f = eff(depth);
    const bool lvl0 = fuse && last;
    if (emit)
      run(Ops<T>::advec_mom(c, 3, sweep, dir, f, lvl0 ? nullptr : c.spare_base(2), lvl0 ? nullptr : c.spare_base(3), reset_tail(last)));
    std::swap(c.fbuf[XVEL1], c.sbuf[2]);
    std::swap(c.fbuf[YVEL1], c.sbuf[3]);
    wrote({U1, V1}, f);
  }
  // One sweep: advec_cell, the halo exchange, advec_mom.  Fused, an x sweep
  // whose exchange has nothing to do (the velocities and the y mass flux
  // already fresh; the cell sweep makes its own outputs fresh) runs as one
  // pass over the tiles away from the edge (Ops::advec_sweep_x).
  void sweep_pair(int sweep, int dir, int mom_depth, bool last) {
    const bool fused = fuse && dir == 1 && Ops<T>::sweep_x_fusable(c) && fresh[U1] >= 2 && fresh[V1] >= 2 && fresh[MFY] >= 2;
    if (!fused) {
      cell(sweep, dir, last);
      halo({D1, E1, U1, V1, MFX, MFY}, 2);
      mom(sweep, dir, mom_depth, last);
      return;
    }
    const int f = eff(dep(2)), fm = eff(mom_depth);
    if (emit) run(Ops<T>::advec_sweep_x(c, sweep, f, fm, reset_tail(last), last, last_flag));
    std::swap(c.fbuf[DENSITY1], c.sbuf[0]);
    std::swap(c.fbuf[ENERGY1], c.sbuf[1]);
    wrote({D1, E1, MFX}, f);
    halo({D1, E1, U1, V1, MFX, MFY}, 2); // (no pass: every field is fresh)
    std::swap(c.fbuf[XVEL1], c.sbuf[2]);
    std::swap(c.fbuf[YVEL1], c.sbuf[3]);
    wrote({U1, V1}, fm);
  }
  // driver/advection.cpp:29-105; the two advec_mom calls of a sweep run as one pass
  void advection(bool x_first) {
    const int d1 = x_first ? 1 : 2, d2 = x_first ? 2 : 1;
    halo({E1, D1, VFX, VFY}, 2);
    sweep_pair(1, d1, dep(2), false);
    sweep_pair(2, d2, 0, true);
  }
  void reset() {
    const int f = eff(dep(1));
    if (emit && !fuse) run(Ops<T>::reset_field(c, f));
    wrote({D0, E0, U0, V0}, f);
  }
  // cb_field_summary
  void summary() {
    if (emit) run(Ops<T>::field_summary(c, last_flag)); // its pressure and soundspeed are read by no later phase
    fresh[P] = 0;
    fresh[SS] = 0;
    ++pos;
  }
  // one whole step as a freshness model (a summary at its end: the pressure
  // halo it marks stale is rewritten by the next step's first phase either way)
  void model_step(bool x_first) {
    pos = 0;
    written = 0;
    timestep_front();
    lagrange();
    advection(x_first);
    reset();
    summary();
  }
};

bool same_fresh(const int *a, const int *b) { return std::memcmp(a, b, sizeof(int) * 15) == 0; }

// Adds a conditional node at the capture position of stream s; the capture
// continues after it.  Returns the node's body graphs (owned by the node).
cudaError_t add_conditional(cudaStream_t s, cudaGraphConditionalHandle h, cudaGraphConditionalNodeType type, unsigned size,
                            cudaGraph_t *bodies) {
  cudaStreamCaptureStatus st;
  cudaGraph_t g = nullptr;
  const cudaGraphNode_t *deps = nullptr;
  size_t ndeps = 0;
  cudaError_t e = cudaStreamGetCaptureInfo(s, &st, nullptr, &g, &deps, &ndeps);
  if (e != cudaSuccess) return e;
  if (st != cudaStreamCaptureStatusActive) return cudaErrorStreamCaptureInvalidated;
  cudaGraphNodeParams p = {};
  p.type = cudaGraphNodeTypeConditional;
  p.conditional.handle = h;
  p.conditional.type = type;
  p.conditional.size = size;
  cudaGraphNode_t node;
  if ((e = cudaGraphAddNode(&node, g, deps, ndeps, &p)) != cudaSuccess) return e;
  if ((e = cudaStreamUpdateCaptureDependencies(s, &node, 1, cudaStreamSetCaptureDependencies)) != cudaSuccess) return e;
  for (unsigned k = 0; k < size; ++k) bodies[k] = p.conditional.phGraph_out[k];
  return cudaSuccess;
}

// Device buffers of a run's graph: its scalar state, parameters, dt, and
// room for trace_cap dt values and rec_cap summary records.
struct RunBufs {
  RunState *st = nullptr;
  RunParams *par = nullptr;
  double *dt_dev = nullptr, *trace = nullptr, *records = nullptr;
  int trace_cap = 0, rec_cap = 0;
  ~RunBufs() {
    cudaFree(st);
    cudaFree(par);
    cudaFree(dt_dev);
    cudaFree(trace);
    cudaFree(records);
  }
  cudaError_t alloc(int ntrace, int nrec) {
    cudaError_t e;
    if ((e = cudaMalloc(&st, sizeof(RunState))) != cudaSuccess) return e;
    if ((e = cudaMalloc(&par, sizeof(RunParams))) != cudaSuccess) return e;
    if ((e = cudaMalloc(&dt_dev, sizeof(double))) != cudaSuccess) return e;
    if ((e = cudaMalloc(&trace, sizeof(double) * (size_t)ntrace)) != cudaSuccess) return e;
    if ((e = cudaMalloc(&records, sizeof(double) * 7 * (size_t)nrec)) != cudaSuccess) return e;
    trace_cap = ntrace;
    rec_cap = nrec;
    return cudaSuccess;
  }
};

// Library kernels per step body, advection branch and summary branch.
struct Counts {
  long long body = 0, adv[2] = {0, 0}, sum = 0;
};

// Everything a captured run bakes into its launches besides the device
// buffers it owns: a graph is launched again only for an equal key.
struct RunKey {
  const void *buf[NUM_BUF];
  const void *geom[NUM_GEOM], *geom_t[NUM_GEOM];
  const void *rgeom;
  int fbuf[15], sbuf[NUM_SPARE], fresh[15];
  int precision, fold, fuse, can_fold, faces;
  double gamma, dtc_safe, dtu_safe, dtv_safe, dtdiv_safe;
};

// The instantiated graph of a chunk's last run (Chunk::run_cache).
struct RunCache {
  RunKey key;
  RunBufs rb;
  Counts n;
  bool fuse = false;
  cudaGraph_t g = nullptr;
  cudaGraphExec_t x = nullptr;
  RunParams *h_par = nullptr; // pinned: the parameters of the next launch
  ~RunCache() {
    if (x) cudaGraphExecDestroy(x);
    if (g) cudaGraphDestroy(g);
    if (h_par) cudaFreeHost(h_par);
  }
};

// Captures the loop into *g: init, then WHILE { step }.  Every capture this
// function began has ended when it returns; *g is set only once the
// top-level capture has ended, and the caller owns it from then on.
template <typename T>
cudaError_t capture_run(Chunk &c, Seq<T> &q, const RunBufs &rb, cudaStream_t s0, cudaStream_t s1, cudaGraph_t *g, Counts &n,
                        std::string &why) {
  const cudaStreamCaptureMode mode = cudaStreamCaptureModeRelaxed;
  bool top_open = false;
  auto abandon = [&](cudaError_t err) {
    for (cudaStream_t s : {s0, s1}) {
      cudaStreamCaptureStatus st;
      if (cudaStreamIsCapturing(s, &st) != cudaSuccess || st == cudaStreamCaptureStatusNone) continue;
      cudaGraph_t junk = nullptr;
      cudaStreamEndCapture(s, &junk);
      if (junk && s == s0 && top_open) cudaGraphDestroy(junk); // body graphs belong to their nodes
    }
    cudaGetLastError();
    return err;
  };
  cudaError_t e;
  if ((e = cudaStreamBeginCapture(s0, mode)) != cudaSuccess) return abandon(e);
  top_open = true;
  k_run_init<<<1, 1, 0, s0>>>(rb.st, rb.par);
  if ((e = cudaGetLastError()) != cudaSuccess) return abandon(e);
  cudaGraph_t top = nullptr;
  {
    cudaStreamCaptureStatus cs;
    if ((e = cudaStreamGetCaptureInfo(s0, &cs, nullptr, &top, nullptr, nullptr)) != cudaSuccess) return abandon(e);
  }
  cudaGraphConditionalHandle hloop;
  if ((e = cudaGraphConditionalHandleCreate(&hloop, top, 1, cudaGraphCondAssignDefault)) != cudaSuccess) return abandon(e);
  cudaGraph_t body;
  if ((e = add_conditional(s0, hloop, cudaGraphCondTypeWhile, 1, &body)) != cudaSuccess) return abandon(e);
  if ((e = cudaStreamEndCapture(s0, g)) != cudaSuccess) return abandon(e);
  top_open = false;

  // the body: one step, captured on s0 into the loop's body graph
  c.stream = s0;
  const long long l0 = c.launches;
  if ((e = cudaStreamBeginCaptureToGraph(s0, body, nullptr, nullptr, 0, mode)) != cudaSuccess) return abandon(e);
  cudaGraphConditionalHandle hadv, hsum;
  if ((e = cudaGraphConditionalHandleCreate(&hadv, body, 0, cudaGraphCondAssignDefault)) != cudaSuccess) return abandon(e);
  if ((e = cudaGraphConditionalHandleCreate(&hsum, body, 0, cudaGraphCondAssignDefault)) != cudaSuccess) return abandon(e);
  q.pos = 0;
  q.written = 0;
  k_run_begin<<<1, 1, 0, s0>>>(rb.st, c.d_dt_bits);
  q.run(cudaGetLastError());
  q.timestep_front();
  k_run_dt<<<1, 1, 0, s0>>>(rb.st, c.d_dt_bits, rb.par, rb.dt_dev, rb.trace, hadv);
  q.run(cudaGetLastError());
  q.lagrange();
  if (q.err != cudaSuccess) return abandon(q.err);
  cudaGraph_t adv[2];
  if ((e = add_conditional(s0, hadv, cudaGraphCondTypeIf, 2, adv)) != cudaSuccess) return abandon(e);
  // the two advection orders from the same state; body 0 runs when advect_x is set
  int fresh0[15], fresh1[15];
  std::memcpy(fresh0, q.fresh, sizeof fresh0);
  const int pos0 = q.pos;
  const unsigned written0 = q.written;
  for (int b = 0; b < 2; ++b) {
    std::memcpy(q.fresh, fresh0, sizeof fresh0);
    q.pos = pos0;
    q.written = written0;
    const long long la = c.launches;
    c.stream = s1;
    if ((e = cudaStreamBeginCaptureToGraph(s1, adv[b], nullptr, nullptr, 0, mode)) != cudaSuccess) return abandon(e);
    q.advection(b == 0);
    cudaGraph_t got = nullptr;
    e = cudaStreamEndCapture(s1, &got);
    c.stream = s0;
    if (q.err != cudaSuccess) return abandon(q.err);
    if (e != cudaSuccess) return abandon(e);
    n.adv[b] = c.launches - la;
    if (b == 0) {
      std::memcpy(fresh1, q.fresh, sizeof fresh1);
    } else if (!same_fresh(fresh1, q.fresh) || n.adv[0] != n.adv[1]) {
      why = "the two advection orders leave different halo states";
      return abandon(cudaErrorNotSupported);
    }
  }
  q.reset();
  k_run_end<<<1, 1, 0, s0>>>(rb.st, rb.par, hsum, hloop);
  q.run(cudaGetLastError());
  if (q.err != cudaSuccess) return abandon(q.err);
  cudaGraph_t sum;
  if ((e = add_conditional(s0, hsum, cudaGraphCondTypeIf, 1, &sum)) != cudaSuccess) return abandon(e);
  {
    cudaGraph_t got = nullptr;
    if ((e = cudaStreamEndCapture(s0, &got)) != cudaSuccess) return abandon(e);
  }
  n.body = c.launches - l0 - n.adv[0] - n.adv[1];
  // the summary branch
  const long long ls = c.launches;
  if ((e = cudaStreamBeginCaptureToGraph(s0, sum, nullptr, nullptr, 0, mode)) != cudaSuccess) return abandon(e);
  q.summary();
  k_run_record<<<1, 1, 0, s0>>>(rb.st, c.d_sums, rb.records, rb.par);
  q.run(cudaGetLastError());
  {
    cudaGraph_t got = nullptr;
    e = cudaStreamEndCapture(s0, &got);
  }
  n.sum = c.launches - ls;
  if (q.err != cudaSuccess) return abandon(q.err);
  if (e != cudaSuccess) return abandon(e);
  return cudaSuccess;
}

template <typename T>
int run_impl(cb_chunk *c, const cb_run_params *p, cb_run_state *state, int max_steps, double *dt_trace, double *summaries,
             int max_summaries, int *nsummaries) {
  const DtConsts dk{p->dtc_safe, p->dtu_safe, p->dtv_safe, p->dtdiv_safe};
  const bool fold = p->fold != 0;
  const bool x0 = state->advect_x != 0;

  // the halo freshness over the first steps, from the chunk's present state
  int fbuf0[15], sbuf0[NUM_SPARE];
  std::memcpy(fbuf0, c->fbuf, sizeof fbuf0);
  std::memcpy(sbuf0, c->sbuf, sizeof sbuf0);
  Seq<T> m(*c, false, fold, dk);
  std::vector<Pass> first[2];
  int settled[4][15];
  for (int s = 0; s < 5; ++s) {
    m.passes.clear();
    m.model_step(s % 2 == 0 ? x0 : !x0);
    if (s < 2) first[s] = m.passes;
    if (s >= 1) std::memcpy(settled[s - 1], m.fresh, sizeof settled[0]);
  }
  if (std::memcmp(fbuf0, c->fbuf, sizeof fbuf0) != 0) return fail(CB_ESTATE, "cb_run: internal: the buffer map did not return after a step");
  if (!same_fresh(settled[1], settled[2]) || !same_fresh(settled[2], settled[3]))
    return fail(CB_ESTATE, "cb_run: the chunk's halo state does not settle; run one step through the phase calls first");

  // passes the first two steps make that the settled body does not: allowed
  // in the first step only, for a field the step has not written before the pass
  HaloJob pro[2] = {}; // depth 1, depth 2
  for (int s = 0; s < 2; ++s) {
    Seq<T> b(*c, false, fold, dk);
    std::memcpy(b.fresh, settled[3], sizeof b.fresh);
    b.model_step(s == 0 ? x0 : !x0);
    for (const Pass &pa : first[s]) {
      if (std::find(b.passes.begin(), b.passes.end(), pa) != b.passes.end()) continue;
      if (s == 1 || (pa.written_before >> pa.field & 1u))
        return fail(CB_ESTATE, "cb_run: the chunk's halo state needs a pass inside the first steps; run one step through the phase calls first");
      HaloJob &job = pro[pa.depth - 1];
      job.field[job.nfields++] = pa.field;
    }
  }

  // what the captured graph bakes in: a kept graph with the same key is launched again
  const int max_records = std::max(max_summaries, 0);
  RunKey key;
  std::memset(&key, 0, sizeof key);
  for (int b = 0; b < NUM_BUF; ++b) key.buf[b] = c->buf[b];
  for (int g = 0; g < NUM_GEOM; ++g) {
    key.geom[g] = c->geom_d[g];
    key.geom_t[g] = c->geom_t[g];
  }
  key.rgeom = c->rgeom_d;
  std::memcpy(key.fbuf, fbuf0, sizeof key.fbuf);
  std::memcpy(key.sbuf, sbuf0, sizeof key.sbuf);
  std::memcpy(key.fresh, settled[3], sizeof key.fresh);
  key.precision = c->precision;
  key.fold = fold ? 1 : 0;
  key.fuse = p->fuse != 0 ? 1 : 0;
  key.can_fold = c->can_fold() ? 1 : 0;
  key.faces = c->external_faces; // the reflective fill's faces
  key.gamma = c->gamma;
  key.dtc_safe = dk.dtc_safe;
  key.dtu_safe = dk.dtu_safe;
  key.dtv_safe = dk.dtv_safe;
  key.dtdiv_safe = dk.dtdiv_safe;
  RunCache *rc = static_cast<RunCache *>(c->run_cache);
  if (rc && (std::memcmp(&rc->key, &key, sizeof key) != 0 || rc->rb.trace_cap < max_steps || rc->rb.rec_cap < std::max(max_records, 1))) {
    run_cache_free(*c);
    rc = nullptr;
  }
  cudaError_t e;
  if (!rc) {
    // the loop's graph, its body captured from the settled freshness
    std::unique_ptr<RunCache> nc(new (std::nothrow) RunCache);
    if (!nc) return fail(CB_ECUDA, "cb_run: out of host memory");
    nc->key = key;
    if ((e = nc->rb.alloc(std::max(max_steps, 1024), std::max(max_records, 256))) != cudaSuccess) return cuda_fail(e, "cb_run");
    if ((e = cudaMallocHost(&nc->h_par, sizeof(RunParams))) != cudaSuccess) return cuda_fail(e, "cb_run");
    cudaStream_t s0 = nullptr, s1 = nullptr;
    if ((e = cudaStreamCreateWithFlags(&s0, cudaStreamNonBlocking)) != cudaSuccess) return cuda_fail(e, "cb_run");
    if ((e = cudaStreamCreateWithFlags(&s1, cudaStreamNonBlocking)) != cudaSuccess) {
      cudaStreamDestroy(s0);
      return cuda_fail(e, "cb_run");
    }
    Seq<T> q(*c, true, fold, dk);
    q.fuse = p->fuse != 0 && fold && c->can_fold();
    if (q.fuse) q.last_flag = reinterpret_cast<const int *>(reinterpret_cast<const char *>(nc->rb.st) + offsetof(RunState, last));
    std::memcpy(q.fresh, settled[3], sizeof q.fresh);
    const cudaStream_t user = c->stream;
    const long long launches0 = c->launches;
    c->dt_dev = nc->rb.dt_dev;
    std::string why;
    e = capture_run<T>(*c, q, nc->rb, s0, s1, &nc->g, nc->n, why);
    c->dt_dev = nullptr;
    c->stream = user;
    c->launches = launches0;
    std::memcpy(c->fbuf, fbuf0, sizeof fbuf0); // (a capture that stopped midway may leave a sweep's swap undone)
    std::memcpy(c->sbuf, sbuf0, sizeof sbuf0);
    if (e == cudaSuccess) e = cudaGraphInstantiate(&nc->x, nc->g, 0);
    cudaStreamDestroy(s0);
    cudaStreamDestroy(s1);
    if (e != cudaSuccess) {
      if (!why.empty()) return fail(CB_ESTATE, "cb_run: " + why);
      return cuda_fail(e, "cb_run");
    }
    nc->fuse = q.fuse;
    rc = nc.release();
    c->run_cache = rc;
  }
  const RunBufs &rb = rc->rb;
  const Counts &n = rc->n;

  // this launch's constants and entry state
  RunParams &hp = *rc->h_par;
  hp.k = RunConsts{};
  hp.k.dtmin = p->dtmin;
  hp.k.dtmax = p->dtmax;
  hp.k.dtrise = p->dtrise;
  hp.k.end_time = p->end_time;
  hp.k.end_step = p->end_step;
  hp.k.summary_frequency = p->summary_frequency;
  hp.k.step0 = state->step;
  hp.k.last_step = state->step + max_steps;
  hp.k.max_records = max_records;
  hp.time = state->time;
  hp.dtold = state->dtold;
  hp.step = state->step;
  hp.advect_x = x0 ? 1 : 0;
  long long restore_launches = 0;
  e = cudaMemcpyAsync(rb.par, &hp, sizeof hp, cudaMemcpyHostToDevice, c->stream);
  for (int d = 0; d < 2 && e == cudaSuccess; ++d)
    if (pro[d].nfields) e = Ops<T>::update_halo(*c, pro[d], d + 1);
  if (e == cudaSuccess) e = cudaGraphLaunch(rc->x, c->stream);
  if (e == cudaSuccess && rc->fuse) {
    // the fused second sweeps left energy1 / xvel1 / yvel1 stale: rebuild
    // them as the phase-by-phase step leaves them (the last first sweep's
    // momentum output, in the spares, gives the velocities' halo ring)
    const long long l = c->launches;
    e = Ops<T>::restore_level1(*c, c->spare_base(2), c->spare_base(3));
    restore_launches = c->launches - l;
    c->launches = l;
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  if (e != cudaSuccess) {
    run_cache_free(*c);
    return cuda_fail(e, "cb_run");
  }

  RunState h{};
  if ((e = cudaMemcpy(&h, rb.st, sizeof h, cudaMemcpyDeviceToHost)) != cudaSuccess) return cuda_fail(e, "cb_run");
  int derr = 0;
  if ((e = cudaMemcpy(&derr, c->d_err, sizeof derr, cudaMemcpyDeviceToHost)) != cudaSuccess) return cuda_fail(e, "cb_run");
  const int steps = h.step - state->step;
  if (dt_trace && steps > 0)
    if ((e = cudaMemcpy(dt_trace, rb.trace, sizeof(double) * (size_t)steps, cudaMemcpyDeviceToHost)) != cudaSuccess)
      return cuda_fail(e, "cb_run");
  const int nrec = std::min(h.nsum, max_records);
  if (summaries && nrec > 0)
    if ((e = cudaMemcpy(summaries, rb.records, sizeof(double) * 7 * (size_t)nrec, cudaMemcpyDeviceToHost)) != cudaSuccess)
      return cuda_fail(e, "cb_run");
  if (nsummaries) *nsummaries = h.nsum;
  // (the passes before the loop counted themselves)
  c->launches += 1 + (long long)steps * (n.body + RUN_KERNELS_PER_STEP + n.adv[0]) + (long long)h.sum_runs * (n.sum + 1) + restore_launches;
  std::memcpy(c->halo_fresh, settled[3], sizeof c->halo_fresh);
  state->step = h.step;
  state->time = h.time;
  state->dt = h.dt;
  state->dtold = h.dtold;
  state->advect_x = h.advect_x;
  state->done = (h.time + g_small > p->end_time || h.step >= p->end_step) ? 1 : 0;
  if (derr) return fail(CB_ECUDA, "cb_run: a kernel's tile staging did not complete (TMA wait limit reached)");
  if (h.small) return fail(CB_ESTATE, "cb_run: small timestep " + std::to_string(h.dt) + " at step " + std::to_string(h.step));
  return CB_OK;
}

} // namespace

namespace cb {
void run_cache_free(Chunk &c) {
  delete static_cast<RunCache *>(c.run_cache);
  c.run_cache = nullptr;
}
} // namespace cb

namespace {

cudaError_t select_device(const cb_chunk *c) {
  int cur = -1;
  cudaError_t e = cudaGetDevice(&cur);
  if (e != cudaSuccess) return e;
  if (cur != c->device) return cudaSetDevice(c->device);
  return cudaSuccess;
}

} // namespace

extern "C" int cb_run(cb_chunk *c, const cb_run_params *p, cb_run_state *state, int max_steps, double *dt_trace, double *summaries,
                      int max_summaries, int *nsummaries) {
  if (!c || !p || !state) return fail(CB_EINVAL, "cb_run: null argument");
  if (max_steps < 1) return fail(CB_EINVAL, "cb_run: max_steps must be at least 1");
  if (max_summaries > 0 && !summaries) return fail(CB_EINVAL, "cb_run: null summaries with max_summaries > 0");
  if (!(p->dtrise > 0.0) || !(p->dtmax > 0.0)) return fail(CB_EINVAL, "cb_run: dtrise and dtmax must be positive");
  if (state->step < 0 || !(state->dtold > 0.0)) return fail(CB_EINVAL, "cb_run: the entry state needs step >= 0 and dtold > 0");
  if ((long long)state->step + max_steps > 0x7fffffffll) return fail(CB_EINVAL, "cb_run: the step count overflows");
  cudaError_t e = select_device(c);
  if (e != cudaSuccess) return cuda_fail(e, "cb_run");
  if ((e = run_pending_calls(c)) != cudaSuccess) return cuda_fail(e, "cb_run");
  if (c->precision == CB_FP64) return run_impl<double>(c, p, state, max_steps, dt_trace, summaries, max_summaries, nsummaries);
  return run_impl<float>(c, p, state, max_steps, dt_trace, summaries, max_summaries, nsummaries);
}
