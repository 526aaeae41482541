/*
 * cloverb200.h -- C ABI of the B200 CloverLeaf hydro library (libcloverb200.so).
 *
 * One opaque cb_chunk holds one mesh chunk resident in the memory of one
 * B200: every 2-D field of the reference's field_type
 * (driver/definitions.h:130-170), the 1-D geometry, a CUDA stream and the
 * scratch of the on-device reductions.  Each entry point below replaces one
 * routine of the reference's per-model interface (the driver/NAME.h
 * declarations every src/<model>/ implements); the comment names it.
 *
 * Conventions
 *  - Every function returns 0 on success and a nonzero CB_E* code on
 *    failure; cb_last_error() then describes the failure (per thread).
 *  - Indices follow the reference: interior cell (j, k) of the Fortran
 *    original is (i, j) = (j + 1, k + 1); arrays carry a 2-deep halo.
 *    Field extents are the reference's (driver/definitions.cpp:4-41):
 *    cell (nx+4)x(ny+4), vertex (nx+5)x(ny+5), x face (nx+5)x(ny+4),
 *    y face (nx+4)x(ny+5).
 *  - Calls are enqueued on the chunk's stream and return without waiting,
 *    except those that hand a value to the host (cb_calc_dt,
 *    cb_field_summary, cb_read_*), which wait for it.
 *  - halo_depth arguments (0, 1 or 2): besides its outputs, the phase also
 *    writes their reflective halo exactly as a following
 *    cb_update_halo(..., halo_depth) would, and the library remembers it, so
 *    that cb_update_halo skips those fields.  0 writes no halo.  Meshes
 *    smaller than 8 cells in either direction ignore halo_depth (there the
 *    reference's fill reads halo cells and is not idempotent, so every
 *    cb_update_halo runs as called), except cb_pdv(full = 1), whose halo
 *    update is part of the routine it replaces.
 *  - Host buffers are plain double arrays; in the FP32 form values are
 *    converted on the way in and out.
 */
#ifndef CLOVERB200_H
#define CLOVERB200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct cb_chunk cb_chunk;

/* Field ids; 0..14 are driver/definitions.h:61-77 (field_parameter). */
enum {
  CB_DENSITY0 = 0, CB_DENSITY1 = 1, CB_ENERGY0 = 2, CB_ENERGY1 = 3, CB_PRESSURE = 4, CB_VISCOSITY = 5,
  CB_SOUNDSPEED = 6, CB_XVEL0 = 7, CB_XVEL1 = 8, CB_YVEL0 = 9, CB_YVEL1 = 10, CB_VOL_FLUX_X = 11,
  CB_VOL_FLUX_Y = 12, CB_MASS_FLUX_X = 13, CB_MASS_FLUX_Y = 14,
  CB_WORK_ARRAY1 = 15, CB_WORK_ARRAY7 = 21, CB_VOLUME = 22, CB_XAREA = 23, CB_YAREA = 24,
  CB_NUM_FIELDS = 25
};
/* 1-D geometry ids (driver/definitions.h:156-163). */
enum { CB_CELLX = 0, CB_CELLY, CB_CELLDX, CB_CELLDY, CB_VERTEXX, CB_VERTEXY, CB_VERTEXDX, CB_VERTEXDY, CB_NUM_GEOM };
enum { CB_FP64 = 0, CB_FP32 = 1 };
/* Host layouts for cb_read_field / cb_write_field: row-major with x fastest,
 * or the reference Buffer2D order data[j + i * sizeY] (src/serial/context.h:73). */
enum { CB_LAYOUT_XFAST = 0, CB_LAYOUT_YFAST = 1 };
/* Options for cb_set_option.
 * CB_OPT_FOLD_HALO (default 1): producers write the halo the driver's next
 *   update_halo asks for, which then has nothing left to do.
 * CB_OPT_FUSE_CALLS (default 0): with folding on, the phase calls of the
 *   reference driver's step run as the fused passes of cb_run's fuse = 1 --
 *   cb_ideal_gas(predict 0) and cb_viscosity are held back until cb_calc_dt,
 *   which does all three in one pass; cb_pdv(predictor), cb_accelerate and
 *   cb_pdv(corrector) until cb_flux_calc (one Lagrangian pass, as
 *   cb_lagrangian); the second sweeps' cb_advec_cell and cb_advec_mom until
 *   cb_reset_field, which they then do.  Results are those of the calls made
 *   one by one (FP64 to the bit).  A held-back call's kernels are enqueued
 *   when its group completes or when any other call on the chunk is made
 *   (cb_launch_count and cb_get_stream excepted): work enqueued directly on
 *   the chunk's stream after a held-back call may run before it. */
enum { CB_OPT_FOLD_HALO = 1, CB_OPT_FUSE_CALLS = 3 };
/* Faces of a chunk (cb_set_external_faces, cb_copy_tile_halo). */
enum { CB_FACE_LEFT = 1, CB_FACE_RIGHT = 2, CB_FACE_BOTTOM = 4, CB_FACE_TOP = 8 };
/* Error codes. */
enum { CB_OK = 0, CB_EINVAL = 1, CB_ECUDA = 2, CB_ENOMEM = 3, CB_ESTATE = 4 };

/* A deck state (driver/definitions.h:79-95); geometry 1 rectangle, 2 circle, 3 point.
 * Pass the extents already nudged as driver/read_input.cpp:268-276 does. */
typedef struct {
  double density, energy, xvel, yvel;
  int geometry;
  double xmin, ymin, xmax, ymax, radius;
} cb_state;

/* Safety factors of calc_dt (driver/definitions.h:240-247). */
typedef struct {
  double dtmin, dtc_safe, dtu_safe, dtv_safe, dtdiv_safe;
} cb_dt_params;

/* Library version and last error of the calling thread. */
int cb_version(void);
const char *cb_last_error(void);

/* Device discovery for the model's create_context / report_context
 * (driver/initialise.h:160-162; the CUDA model's src/cuda/initialise.cpp:25-45). */
int cb_device_count(int *count);
int cb_device_name(int device, char *name, size_t len);

/* Lifecycle.  Replaces the allocation in field_type's constructor
 * (driver/definitions.cpp:4-41) and src/cuda/finalise.cpp:22-58's release.
 * precision is CB_FP64 or CB_FP32; device is a CUDA device ordinal. */
int cb_create(int nx, int ny, int precision, int device, cb_chunk **out);
int cb_destroy(cb_chunk *c);
/* gamma of the ideal-gas law; the reference hard-codes 1.4 (src/serial/ideal_gas.cpp:41-42). */
int cb_set_gamma(cb_chunk *c, double gamma);
int cb_set_option(cb_chunk *c, int option, int value);
int cb_get_extent(const cb_chunk *c, int field, int *size_x, int *size_y);

/* Host <-> device copies of whole fields (the model's Buffer2D::mirrored(),
 * src/serial/context.h:82-86).  n must equal size_x * size_y of the field. */
int cb_read_field(cb_chunk *c, int field, double *host, size_t n, int layout);
int cb_write_field(cb_chunk *c, int field, const double *host, size_t n, int layout);
/* 1-D geometry arrays; n = its reference length (nx+4/ny+4 cell, nx+5/ny+5 vertex). */
int cb_read_geom(cb_chunk *c, int geom, double *host, size_t n);
int cb_write_geom(cb_chunk *c, int geom, const double *host, size_t n);

/* Setup: driver/build_field.h:24, driver/initialise_chunk.h:24, driver/generate_chunk.h:24. */
int cb_build_field(cb_chunk *c);
int cb_initialise_chunk(cb_chunk *c, double xmin, double ymin, double xmax, double ymax);
/* src/serial/initialise_chunk.cpp:30-85 for one chunk of a decomposed grid:
 * the chunk's first cell is cell (left, bottom) (1-based) of the x_cells x
 * y_cells grid over [xmin, xmax] x [ymin, ymax]; dx, dy from the whole grid,
 * the chunk's origin xmin + dx * (left - 1) as the reference forms it
 * (driver/comms.cpp:64-156 gives left and bottom). */
int cb_initialise_chunk_in(cb_chunk *c, double xmin, double ymin, double xmax, double ymax, int x_cells, int y_cells, int left, int bottom);
int cb_generate_chunk(cb_chunk *c, int nstates, const cb_state *states);

/* Hydro phases. */
/* driver/ideal_gas.h:24 -- pressure, soundspeed from level 0 (or level 1 if predict). */
int cb_ideal_gas(cb_chunk *c, int predict, int halo_depth);
/* driver/viscosity.h:24. */
int cb_viscosity(cb_chunk *c, int halo_depth);
/* driver/calc_dt.h:26-27 -- the minimum over cells, on the device; returns the
 * kernel's dt_min_val and control/jldt/kldt/small as src/serial/calc_dt.cpp:73-79 forms them. */
int cb_calc_dt(cb_chunk *c, const cb_dt_params *p, double *dt_min_val, int *control, int *jldt, int *kldt, int *small);
/* The Lagrangian pass run ahead (no counterpart in the reference; for the
 * driver's step under CB_OPT_FUSE_CALLS).  Arms the next cb_calc_dt -- when it
 * is the fused ideal_gas + viscosity + calc_dt pass on a folding chunk -- to
 * enqueue, behind the minimum's read-back, the Lagrangian pass with the dt
 * the driver will take, min(min(minimum, dtold * dtrise), dtmax)
 * (driver/timestep.cpp:93), formed on the device: the GPU keeps working while
 * the host reads the minimum back.  The four calls that follow --
 * cb_pdv(predictor, full), cb_accelerate, cb_pdv(corrector), cb_flux_calc
 * with halo depths 1, 2, 2, 2 -- find their work done when their dt is that
 * clamp's (host arithmetic, the same order); any other call, or a different
 * dt or depth, first enqueues the calls matched so far, and the results are
 * those of the calls made one by one (FP64 to the bit).  Until the four
 * calls are made, level-1 fields, soundspeed and the volume fluxes hold the
 * pass's outputs.  One-shot: arm before each cb_calc_dt. */
int cb_set_dt_ahead(cb_chunk *c, double dtold, double dtrise, double dtmax);
/* Passes run ahead, and those the four calls consumed, since cb_create. */
int cb_dt_ahead_stats(const cb_chunk *c, long long *launched, long long *used);
/* driver/PdV.h:24.  full = 0: the PdV kernel alone (src/serial/PdV.cpp:36-87);
 * full = 1 with predict = 1: the model's whole predictor step (:92-133:
 * kernel, ideal_gas on level 1, depth-1 pressure halo, revert) in one pass. */
int cb_pdv(cb_chunk *c, int predict, double dt, int full, int halo_depth);
/* driver/revert.h:24. */
int cb_revert(cb_chunk *c);
/* driver/accelerate.h:24. */
int cb_accelerate(cb_chunk *c, double dt, int halo_depth);
/* driver/flux_calc.h:24. */
int cb_flux_calc(cb_chunk *c, double dt, int halo_depth);
/* The Lagrangian step of driver/hydro.cpp:69-75 in one pass: the calls
 * cb_pdv(c, 1, dt, 1, 1), cb_accelerate(c, dt, halo_depth),
 * cb_pdv(c, 0, dt, 0, halo_depth) and cb_flux_calc(c, dt, halo_depth) (the
 * reference's PdV.cpp:36-133 predictor and corrector with ideal_gas,
 * update_halo(pressure) and revert, accelerate.cpp:28-56, flux_calc.cpp:27-43),
 * with the same results and halo state.  One kernel when the chunk folds
 * halos (each tile recomputes the predicted pressures and level-1 velocities
 * of a one-cell ring around it); otherwise the four phases, one pass each.
 * No counterpart in the reference, whose model interface has the four calls. */
int cb_lagrangian(cb_chunk *c, double dt, int halo_depth);
/* driver/advec_cell.h:24 -- dir 1 = x, 2 = y. */
int cb_advec_cell(cb_chunk *c, int sweep_number, int direction, int halo_depth);
/* driver/advec_mom.h:24 -- which_vel 1 (x velocity), 2 (y velocity) or 3
 * (both in one pass, as the pair of calls at driver/advection.cpp:56-57 does). */
int cb_advec_mom(cb_chunk *c, int which_vel, int sweep_number, int direction, int halo_depth);
/* driver/reset_field.h:24. */
int cb_reset_field(cb_chunk *c, int halo_depth);
/* driver/update_halo.h:24 -- fields[15] flags (field_parameter order), depth 1 or 2. */
int cb_update_halo(cb_chunk *c, const int fields[15], int depth);
/* driver/field_summary.h:25 -- ideal_gas then volume, mass, internal energy,
 * kinetic energy, pressure*volume sums, reduced on the device. */
int cb_field_summary(cb_chunk *c, double out[5]);

/* Tiles (tiles_per_chunk > 1): each tile of the reference's chunk is its own
 * cb_chunk.  cb_set_external_faces marks which faces of a chunk lie on the
 * physical boundary (CB_FACE_* bits, default all four): cb_update_halo's
 * reflective fill writes those faces only, as update_halo_kernel fills the
 * faces whose chunk and tile neighbours are both external
 * (src/serial/update_halo.cpp:41-71); with any face internal, producers do
 * not fold halos.  cb_copy_tile_halo fills dst's halo on `side` (one
 * CB_FACE_* value) from src, the neighbouring tile on that side, for the
 * listed fields (fields[f] == 1) to `depth` -- one of the four
 * update_tile_halo_{l,r,b,t}_kernel calls of driver/update_tile_halo.cpp:27-91
 * (driver/update_tile_halo_kernel.h:25-86; index rules of
 * src/serial/update_tile_halo_kernel.cpp).  The copy is ordered after the
 * work already enqueued for both chunks and before any work enqueued later. */
int cb_set_external_faces(cb_chunk *c, int faces);
int cb_copy_tile_halo(cb_chunk *dst, cb_chunk *src, int side, const int fields[15], int depth);

/* Chunks of a decomposed run in different processes (one per GPU): the face
 * strips of driver/comms.cpp:clover_exchange (the pack / unpack index rules
 * of src/serial/pack_kernel.cpp:27-300) between a chunk and a linear device
 * buffer, for the caller to move between ranks (NCCL send/recv of device
 * buffers, or any other transport).  cb_pack_face writes the strip the
 * neighbour on `side` (one CB_FACE_* value) needs, `depth` deep, of the listed
 * fields (fields[f] == 1) to dev_buf; cb_unpack_face fills the chunk's own
 * halo on `side` from the strip that neighbour packed for it.  The strip is
 * cb_face_strip_size elements of the chunk's precision: per listed field in
 * field order, depth rows across the face of the field's extent along it
 * (interior + 2 * depth, + 1 for the arrays one longer that way), the row
 * nearest the face first.  Both enqueue on the chunk's stream (cb_get_stream)
 * after its earlier work; neighbours along a face share its extent.  A
 * caller's update_halo is then: left/right strips, then bottom/top (so the
 * corners arrive), then cb_update_halo for the physical faces
 * (cb_set_external_faces). */
int cb_face_strip_size(cb_chunk *c, int side, const int fields[15], int depth, size_t *elements);
int cb_pack_face(cb_chunk *c, int side, const int fields[15], int depth, void *dev_buf, size_t capacity);
int cb_unpack_face(cb_chunk *c, int side, const int fields[15], int depth, const void *dev_buf, size_t capacity);
/* Waits for everything enqueued on the chunk. */
int cb_synchronize(cb_chunk *c);
/* The CUDA stream (a cudaStream_t) the chunk's work is enqueued on, for
 * callers that time it with their own events or order their own work after it. */
int cb_get_stream(cb_chunk *c, void **stream);
/* Number of kernels the library has launched for this chunk so far. */
int cb_launch_count(const cb_chunk *c, long long *count);

/* ------------------------------------------------------------------------
 * Whole-run residency: the hydro loop of driver/hydro.cpp:53-111 (the
 * while loop over hydro steps) run on the device as one CUDA graph, its
 * host-side logic -- the dt clamp of driver/timestep.cpp:75-96, time, the
 * end test and the summary schedule of driver/hydro.cpp:87-111 -- moved
 * into small kernels, so the host waits once for the whole run.  Each step
 * launches exactly the phases the calls above make for the driver's
 * sequence (driver/timestep.cpp:37-109, driver/advection.cpp:29-105,
 * src/serial/PdV.cpp:92-133), with the same halo bookkeeping, and the
 * fields end bit-identical to that sequence's.  Call it after the start-up
 * sequence of driver/start.cpp:43-138 (or after any number of steps made
 * through the phase calls).
 * ------------------------------------------------------------------------ */
typedef struct {
  double dtmin, dtmax, dtrise;                       /* driver/definitions.h:246-249 */
  double dtc_safe, dtu_safe, dtv_safe, dtdiv_safe;   /* calc_dt's safety factors */
  double end_time;
  int end_step;
  int summary_frequency;                             /* 0: a summary at the end only */
  int fold;                                          /* 1: producers write the halos the next update_halo
                                                        needs (halo_depth > 0 in the phase calls); 0: none do */
  int fuse;                                          /* 1 (with fold = 1, meshes of 8 cells and more): phases that
                                                        share inputs run as one pass -- ideal_gas, viscosity and
                                                        calc_dt; the PdV predictor, accelerate, the PdV corrector
                                                        and flux_calc (as cb_lagrangian); reset_field inside the
                                                        second sweeps -- six kernels a step; FP64 results unchanged
                                                        to the bit, FP32 within its rounding (the fused kernels may
                                                        contract differently) */
} cb_run_params;

/* The driver's loop state (driver/definitions.h:258-280). */
typedef struct {
  int step;         /* in: steps made so far; out: after the call */
  int advect_x;     /* in/out: 1 when the next step sweeps x first */
  double time;      /* in/out: simulated time */
  double dtold;     /* in/out: dt of the last step (dtinit before the first) */
  double dt;        /* out: dt of the last step */
  int done;         /* out: 1 once time reached end_time or step reached end_step */
} cb_run_state;

/* Runs hydro steps until the run is complete or max_steps (>= 1) steps were
 * made.  dt_trace (NULL, or max_steps doubles) receives each step's dt;
 * summaries (NULL when max_summaries is 0; else 7 doubles per record: step,
 * time, volume, mass, internal energy, kinetic energy, pressure*volume)
 * receives the summaries of driver/hydro.cpp:95-111 in order, the first
 * max_summaries of them; *nsummaries (may be NULL) counts all of them.  A dt
 * below dtmin returns CB_ESTATE (the state then includes that step, as the
 * driver's report does).  The chunk keeps the run's instantiated graph (and
 * a few device buffers) until it is destroyed: the next cb_run on it
 * launches that graph again, without capturing, when the chunk is as the
 * graph was captured for -- the same buffers and buffer map, halo state,
 * physical faces, gamma, fold / fuse and safety factors -- and max_steps and max_summaries
 * fit the kept buffers; otherwise it captures anew. */
int cb_run(cb_chunk *c, const cb_run_params *p, cb_run_state *state, int max_steps, double *dt_trace, double *summaries,
           int max_summaries, int *nsummaries);

/* ------------------------------------------------------------------------
 * Batched ensemble: many independent decks advanced by one persistent
 * kernel launch.  No counterpart in the reference, whose driver runs one
 * deck per process; each deck here follows exactly the per-chunk sequence
 * of the calls above (the reference driver's, driver/start.cpp:43-138 and
 * driver/hydro.cpp:46-223) with its own gamma, states, dt controls and end
 * time, and its fields end bit-identical to that sequence's.
 * ------------------------------------------------------------------------ */
typedef struct cb_batch cb_batch;

#define CB_DECK_MAX_STATES 8

/* One deck: mesh, domain, gamma, states (index 0 the background; extents
 * already nudged as driver/read_input.cpp:268-276 does) and the controls of
 * driver/definitions.h:227-256.  nx and ny must be at least 8. */
typedef struct {
  int nx, ny;
  double xmin, ymin, xmax, ymax;
  double gamma;
  int nstates;
  cb_state states[CB_DECK_MAX_STATES];
  double dtinit, dtmin, dtmax, dtrise;
  double dtc_safe, dtu_safe, dtv_safe, dtdiv_safe;
  double end_time;
  int end_step;
  int summary_frequency;
} cb_deck;

/* Deck status after a run. */
enum { CB_DECK_PENDING = 0, CB_DECK_DONE = 1, CB_DECK_SMALL_DT = 2, CB_DECK_STAGE_FAIL = 3, CB_DECK_SYNC_FAIL = 4 };

/* How the persistent launch is laid out.  A deck of c cells runs on a lane of
 * w CTAs, w the power of two >= c / cells_per_cta (at most max_lane_width,
 * the deck's tile count and the grid).  The decks wait in one queue per
 * width, largest estimated run (cells x steps) first, and the queues are
 * worked widest first: at width W the grid forms lanes of W consecutive CTAs,
 * each lane takes the queue's next deck until the queue is empty, then splits
 * into the lanes of the next width.  ctas_per_sm (0 = as many as fit) sets
 * the grid; variant picks the tile shapes (0: 64 x 16 tiles for accelerate
 * and flux_calc, 1: 64 x 8 tiles and more CTAs per SM).  The lanes count
 * that cb_batch_get_schedule and the trials report is the sum over the widths
 * of grid / width. */
typedef struct {
  int cells_per_cta;
  int max_lane_width;
  int ctas_per_sm;
  int variant;
} cb_batch_schedule;

typedef struct {
  cb_batch_schedule schedule;
  int lanes, ctas;
  float ms; /* mean time of one whole-ensemble run */
} cb_batch_trial;

/* Allocates every deck's fields (one pool on `device`), its geometry
 * (src/serial/initialise_chunk.cpp:30-85) and tensor maps, and a default
 * schedule. */
int cb_batch_create(int ndecks, const cb_deck *decks, int precision, int device, cb_batch **out);
int cb_batch_destroy(cb_batch *b);
/* Lays the launch out (see cb_batch_schedule) and captures it in a CUDA graph. */
int cb_batch_set_schedule(cb_batch *b, const cb_batch_schedule *s);
int cb_batch_get_schedule(const cb_batch *b, cb_batch_schedule *s, int *lanes, int *ctas);
/* Runs the ensemble once per candidate schedule (plus a warm-up) and keeps the
 * fastest; trials[0..*ntrials) receives every candidate's timing. */
int cb_batch_autotune(cb_batch *b, int repeats, cb_batch_trial *trials, int max_trials, int *ntrials, cb_batch_schedule *best);
/* Enqueues one run of the whole ensemble from t = 0 (one graph launch: the
 * descriptors are reset and the persistent kernel advances every deck to its
 * end) and returns without waiting. */
int cb_batch_run(cb_batch *b);
/* Waits for the run and checks the launch; *ms receives its device time. */
int cb_batch_synchronize(cb_batch *b, float *ms);
/* Results of deck `deck` of the last run: status (CB_DECK_*), steps, time reached, summary records. */
int cb_batch_deck_result(cb_batch *b, int deck, int *status, int *steps, double *time, int *nsummaries);
/* Summary records (step, time, volume, mass, internal energy, kinetic energy,
 * pressure*volume: 7 doubles each) of deck `deck`; *count = records written. */
int cb_batch_read_summaries(cb_batch *b, int deck, double *out, int max_records, int *count);
/* dt of every step of deck `deck`. */
int cb_batch_read_dt(cb_batch *b, int deck, double *out, int max_steps, int *count);
/* Final field of deck `deck`, as cb_read_field. */
int cb_batch_read_field(cb_batch *b, int deck, int field, double *host, size_t n, int layout);
int cb_batch_get_stream(cb_batch *b, void **stream);
/* Kernels the batch has launched so far. */
int cb_batch_launch_count(const cb_batch *b, long long *count);

/* ------------------------------------------------------------------------
 * Adjoint: the gradient of the final kinetic energy (field_summary's ke
 * after the last step) with respect to the initial interior density0 and
 * energy0 of every cell and to gamma, with the dt sequence of the forward
 * run held fixed.  No counterpart in the reference.  FP64 only.  The
 * forward run is the plain path above (the driver's call order); the
 * reverse sweep runs hand-written adjoint kernels of every phase over
 * checkpoints of the level-0 state every K steps (K = ceil(sqrt(steps))
 * unless set), re-running each segment and each step forward as it goes.
 * ------------------------------------------------------------------------ */
typedef struct cb_adjoint cb_adjoint;

/* A problem from a deck (mesh, domain, states, dt controls; nx, ny >= 8).
 * The initial state is the deck's until cb_adjoint_set_initial replaces it. */
int cb_adjoint_create(const cb_deck *deck, int device, cb_adjoint **out);
int cb_adjoint_destroy(cb_adjoint *a);
/* Initial interior density0 and energy0 (nx * ny values each, x fastest)
 * and gamma; the halos follow from the interior as the driver's start
 * (driver/start.cpp:103-118) makes them. */
int cb_adjoint_set_initial(cb_adjoint *a, const double *density0, const double *energy0, double gamma);
/* Steps between checkpoints (0: ceil(sqrt(steps))). */
int cb_adjoint_set_checkpoint_interval(cb_adjoint *a, int k);
/* Forward run of `steps` steps from the initial state.  dt NULL: each step's
 * dt comes from calc_dt and the driver's clamp (driver/timestep.cpp:75-96)
 * and is recorded; else the given sequence is used.  *ke receives the final
 * kinetic energy. */
int cb_adjoint_forward(cb_adjoint *a, int steps, const double *dt, double *ke);
/* The last forward run's dt sequence. */
int cb_adjoint_dt(const cb_adjoint *a, double *out, int max_steps, int *count);
/* Reverse sweep of the last forward run: dKE/d density0, dKE/d energy0
 * (nx * ny each, x fastest; either may be NULL) and dKE/d gamma. */
int cb_adjoint_gradient(cb_adjoint *a, double *g_density0, double *g_energy0, double *g_gamma);
/* Tangent-linear run of the last forward run's map in the direction
 * (d_density0, d_energy0, d_gamma): *ke the final kinetic energy, *dke its
 * directional derivative. */
int cb_adjoint_tangent(cb_adjoint *a, const double *d_density0, const double *d_energy0, double d_gamma, double *ke, double *dke);
/* Final field of the last tangent run: which 0 its values (the plain
 * path's), 1 its tangents; n = the field's extent as cb_get_extent. */
int cb_adjoint_read_tangent(cb_adjoint *a, int field, int which, double *host, size_t n);
/* A field of the primal chunk as it stands (cb_read_field, x fastest). */
int cb_adjoint_read_field(cb_adjoint *a, int field, double *host, size_t n);
/* Checkpoint interval and count of the last forward run, steps re-run by
 * the last reverse sweep, and the device memory the adjoint holds. */
int cb_adjoint_stats(const cb_adjoint *a, int *checkpoint_interval, int *checkpoints, long long *recomputed_steps, size_t *device_bytes);

/* DIAGNOSTIC, not part of the hydro interface: a self-test of the FP64
 * kernels' quotient of two mesh widths (formed with a precomputed reciprocal)
 * against the device's division operator on `samples` pseudo-random pairs of
 * positive operands; *mismatches counts the quotients that differ in any bit.
 * The test suite calls it; a solver never needs to.  No counterpart in the
 * reference. */
int cb_selftest_width_ratio(long long samples, unsigned long long seed, long long *mismatches);

/* DIAGNOSTIC, not part of the hydro interface: runs the kernels' two bounded
 * waits to their limit on purpose, with limit_ms (0 < limit_ms <= 1000) in
 * place of the kernels' own limits (1 s for a tile's staging wait, 2 s for
 * the ensemble's lane barrier): a staging wait on an mbarrier that nothing
 * completes (no copy in flight) and a lane barrier whose second CTA never
 * arrives.  Reports each wait's error flag (*stage_flag, *lane_abort: 1 when
 * it gave up), what it returned (0: gave up) and how long it waited.  The
 * device stays usable afterwards.  The test suite calls it; a solver never
 * needs to.  No counterpart in the reference. */
int cb_selftest_wait_limits(double limit_ms, int *stage_flag, int *stage_returned, double *stage_ms, int *lane_abort, int *lane_returned,
                            double *lane_ms);

/* The field summary of cb_field_summary (ideal_gas, then the five sums) over
 * FP64 device arrays the caller owns, allocating no memory: for callers that
 * must not allocate device memory where they need the summary (their device
 * memory comes from their own pool, or the call sits inside a loop that must
 * stay allocation-free).  No counterpart in the reference.  Arrays are device
 * pointers to element (0, 0) of each field, rows `pitch` elements apart, in
 * the reference's index convention; celldx/celldy hold nx+4 / ny+4 widths.
 * pressure and soundspeed receive the interior ideal-gas values; sums (device,
 * 5 doubles) receives volume, mass, internal energy, kinetic energy and
 * pressure*volume.  The work is enqueued on `stream` (a cudaStream_t; NULL for
 * the default stream) and the call returns without waiting.  The reduction
 * scratch is one fixed device array inside the library, with room for 16384
 * blocks of 32 x 8 cells: a mesh is accepted when
 * ceil(nx / 32) * ceil(ny / 8) <= 16384 (4,194,304 cells when nx is a
 * multiple of 32 and ny of 8; a 2050 x 2040 mesh, 4,182,000 cells, needs
 * 16575 blocks and is rejected with CB_EINVAL).  The array is shared by all
 * calls on a device: the first call on each device looks up its address in
 * the device's primary context and keeps it, so make that call before any
 * stream capture, do not call the function from another context on the same
 * device (cuCtxCreate) or across cudaDeviceReset, and do not let calls
 * overlap on the GPU. */
int cb_field_summary_noalloc(int nx, int ny, long long pitch, const double *density0, const double *energy0, const double *xvel0,
                             const double *yvel0, const double *celldx, const double *celldy, double *pressure, double *soundspeed,
                             double gamma, double *sums, void *stream);

#ifdef __cplusplus
}
#endif
#endif
