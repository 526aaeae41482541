// cb_chunk.h -- host-side state of one mesh chunk owned by the C-ABI library.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>
#include <string>

#include "cb_mesh.cuh"

namespace cb {

// second buffers of the double-buffered phases: 0 density1, 1 energy1,
// 2 xvel1, 3 yvel1 (advection), 4 pressure (the resident loop's fused step)
constexpr int NUM_SPARE = 5;
constexpr int NUM_BUF = 15 + NUM_SPARE; // device buffers of the 15 state fields + spares
constexpr int BATCH_BUF = 15 + 4;       // a batch deck's buffers: the state fields + the advection spares
constexpr int NUM_BOX_H = 6;            // staged box heights (rows) with a tensor map each
constexpr int BOX_HEIGHTS[NUM_BOX_H] = {10, 12, 16, 18, 20, 24};

// Slot of box height H in BOX_HEIGHTS; a height without a map does not compile.
template <int H> constexpr int box_slot() {
  constexpr int s = H == 10 ? 0 : H == 12 ? 1 : H == 16 ? 2 : H == 18 ? 3 : H == 20 ? 4 : H == 24 ? 5 : -1;
  static_assert(s >= 0, "no tensor map for this box height");
  return s;
}

// Phase calls held back under call fusion (CB_OPT_FUSE_CALLS): ideal_gas
// and viscosity wait for calc_dt (then one pass does the three), the PdV
// predictor, accelerate and the PdV corrector wait for flux_calc (the
// Lagrangian pass), the second advection sweeps wait for reset_field (which
// they then do), and the cell part of a first x sweep waits for its
// momentum part (the x sweep runs as one pass).  Any other call first runs
// what is held back, as called.
enum PendKind : int { PEND_NONE = 0, PEND_IG, PEND_IG_VISC, PEND_PDV1, PEND_PDV1_ACC, PEND_PDV1_ACC_PDV0, PEND_CELL, PEND_CELL_MOM };
struct Pending {
  int kind = PEND_NONE;
  int ig_fold = 0, visc_fold = 0;                  // ideal_gas, viscosity
  double dt = 0.0;                                 // the Lagrangian calls' dt
  int pdv1_fold = 0, acc_fold = 0, pdv0_fold = 0;  // predictor (pressure), accelerate, corrector
  int cell_sweep = 0, cell_dir = 0, cell_fold = 0; // a cell sweep
  int mom_fold = 0, mom_mask = 0;                  // its momentum sweep (the second sweep's)
};

// The Lagrangian pass run ahead (cb_set_dt_ahead): cb_calc_dt, with the
// driver's dt clamp in hand, also enqueues the pass with the clamped dt on
// the device, so the GPU keeps working while the host reads the minimum
// back; the four calls that follow are checked against it (dt and halo
// depths) and find their work done.  A call out of that sequence first
// enqueues the calls it already stood for.
struct DtAhead {
  bool armed = false;             // set for the next cb_calc_dt
  double dtold = 0.0, dtrise = 0.0, dtmax = 0.0;
  bool launched = false;          // the pass is enqueued
  double dt = 0.0;                // its dt: the host's clamp of the read-back minimum
  int folds[4] = {};              // predictor (pressure), accelerate, corrector, flux_calc
  int stage = 0;                  // calls matched: 1 predictor, 2 accelerate, 3 corrector
  long long launched_count = 0, used_count = 0; // passes run ahead / consumed
};

struct Chunk {
  int nx = 0, ny = 0;
  int precision = 0; // 0 FP64, 1 FP32
  int device = 0;
  size_t esize = 8;       // bytes per element
  long long pitch = 0;    // elements per row
  size_t off = 0;         // elements before logical (0, 0) in an allocation
  size_t alloc_elems = 0; // elements per allocation
  double gamma = 1.4;

  // Buffers: buf[b] is a raw allocation; field f currently lives in buffer
  // fbuf[f], spare s in sbuf[s].  Double-buffered phases swap indices.
  void *buf[NUM_BUF] = {};
  int fbuf[15] = {};
  int sbuf[NUM_SPARE] = {};
  // One TMA tensor map per buffer and staged box height (cb_tma.cuh).
  CUtensorMap tmap[NUM_BUF][NUM_BOX_H];
  bool tmap_ok = false;

  // geometry: FP64 on device for every precision, plus a copy in the storage type
  double *geom_d[NUM_GEOM] = {};
  void *geom_t[NUM_GEOM] = {};
  double *geom_h[NUM_GEOM] = {};
  double *rgeom_d = nullptr; // 1 / celldx, 1 / celldy, 1 / vertexdx, 1 / vertexdy (4 x geom_len, FP64)
  int geom_len = 0;

  cudaStream_t stream = nullptr;
  unsigned long long *d_dt_bits = nullptr;
  double *d_partials = nullptr;
  unsigned int *d_counter = nullptr;
  double *d_sums = nullptr;
  int *d_err = nullptr;        // set by a kernel whose staging wait gave up
  double *h_scalars = nullptr; // pinned: [0] dt init, [1] dt, [2..6] sums
  int summary_grid = 0;
  int sms = 148;

  int halo_fresh[15] = {};     // depth to which each field's halo matches update_halo
  int external_faces = 15;     // faces on the physical boundary (CB_FACE_* bits): the reflective fill's faces
  cudaEvent_t ev_order = nullptr; // orders a tile-halo copy between two chunks' streams
  bool fold_enabled = true;    // fold halos into producers when the mesh allows it
  bool fuse_calls = false;     // call fusion (CB_OPT_FUSE_CALLS), with folding producers
  Pending pend;                // calls held back by call fusion
  DtAhead ahead;               // the Lagrangian pass run ahead of its calls
  double *d_dt_ahead = nullptr; // its dt on the device
  cudaEvent_t ev_dt = nullptr;  // the dt read-back's completion

  long long launches = 0; // kernels launched for this chunk
  // When set, the phases that take dt (PdV, accelerate, flux_calc) read it
  // from this device address instead of their argument (cb_run's graph).
  const double *dt_dev = nullptr;
  // cb_run's instantiated graph of the last run and its device buffers,
  // launched again by a run that finds the chunk as it was captured for
  // (cb_run.cu); freed by run_cache_free.
  void *run_cache = nullptr;

  // folding writes reflected halos, so it needs every face on the physical boundary
  bool can_fold() const { return fold_enabled && nx >= 8 && ny >= 8 && external_faces == 15; }
  void *base(int f) const { return (char *)buf[fbuf[f]] + off * esize; }
  void *spare_base(int s) const { return (char *)buf[sbuf[s]] + off * esize; }
  template <int H> const CUtensorMap *map(int f) const { return &tmap[fbuf[f]][box_slot<H>()]; }
};

// Frees cb_run's kept graph (cb_run.cu).
void run_cache_free(Chunk &c);

} // namespace cb

// The C ABI's opaque handle (include/cloverb200.h) is the chunk itself.
struct cb_chunk : cb::Chunk {};
