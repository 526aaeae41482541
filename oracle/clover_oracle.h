/*
 * clover_oracle.h -- CPU restatement of the CloverLeaf hydro path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker for the CUDA
 * implementation in cloverleaf_b200/.  Only tests/, __graft_entry__.smoke()
 * and bench.py's CPU-baseline leg may load it.  The product path never calls
 * it and never falls back to it.
 *
 * Every function restates one routine of the reference's serial model
 * (src/serial/NAME.cpp) or driver (driver/NAME.cpp) operation for operation, with
 * the same index ranges, the same expression order (so results are
 * bit-identical when compiled without FMA contraction) and the same quirks.
 * The only extension is gamma as a parameter (the reference hard-codes 1.4,
 * src/serial/ideal_gas.cpp:41-42); at gamma = 1.4 the arithmetic is the same.
 *
 * Indexing follows the reference: interior cell (j, k) of the Fortran
 * original is C index (j + 1, k + 1); x_min = y_min = 1, x_max = nx,
 * y_max = ny; every 2-D array carries a 2-deep halo.  All 2-D arrays here are
 * allocated with the vertex extent (nx + 5) x (ny + 5) and an x-fast row
 * stride of nx + 5; the reference's smaller extents are a subset of it.
 */
#ifndef CLOVER_ORACLE_H
#define CLOVER_ORACLE_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Field ids: 0..14 follow driver/definitions.h:61-77 (field_parameter). */
enum {
  OC_DENSITY0 = 0, OC_DENSITY1 = 1, OC_ENERGY0 = 2, OC_ENERGY1 = 3,
  OC_PRESSURE = 4, OC_VISCOSITY = 5, OC_SOUNDSPEED = 6,
  OC_XVEL0 = 7, OC_XVEL1 = 8, OC_YVEL0 = 9, OC_YVEL1 = 10,
  OC_VOL_FLUX_X = 11, OC_VOL_FLUX_Y = 12, OC_MASS_FLUX_X = 13, OC_MASS_FLUX_Y = 14,
  OC_WORK1 = 15, OC_WORK2, OC_WORK3, OC_WORK4, OC_WORK5, OC_WORK6, OC_WORK7,
  OC_VOLUME = 22, OC_XAREA = 23, OC_YAREA = 24,
  OC_NUM_2D = 25
};
enum { OC_CELLX = 0, OC_CELLY, OC_CELLDX, OC_CELLDY, OC_VERTEXX, OC_VERTEXY,
       OC_VERTEXDX, OC_VERTEXDY, OC_NUM_1D };

typedef struct {
  int nx, ny;       /* interior cells */
  int sx, sy;       /* allocated 2-D extent: nx + 5, ny + 5 */
  double gamma;
  double *f[OC_NUM_2D];
  double *g[OC_NUM_1D]; /* 1-D geometry, length max(nx, ny) + 6 */
} oc_chunk;

/* A deck state (driver/definitions.h:79-95); geometry 1 rect, 2 circle, 3 point. */
typedef struct {
  double density, energy, xvel, yvel;
  int geometry;
  double xmin, ymin, xmax, ymax, radius;
} oc_state;

/* Deck-level configuration (driver/definitions.h:227-256 subset). */
typedef struct {
  int x_cells, y_cells;
  double xmin, ymin, xmax, ymax;
  double dtinit, dtmin, dtmax, dtrise, dtu_safe, dtv_safe, dtc_safe, dtdiv_safe;
  double end_time;
  int end_step;
  int summary_frequency;
  int number_of_states;
  const oc_state *states; /* already nudged by dx/100 as driver/read_input.cpp:268-276 does */
  double gamma;
} oc_config;

/* One field_summary record: step, time, vol, mass, ie, ke, press. */
typedef struct {
  int step;
  double time, vol, mass, ie, ke, press;
} oc_summary;

oc_chunk *oc_create(int nx, int ny, double gamma);
void oc_destroy(oc_chunk *c);
size_t oc_index(const oc_chunk *c, int i, int j);
double *oc_field(oc_chunk *c, int id);
double *oc_geom(oc_chunk *c, int id);

/* Setup (src/serial/build_field.cpp, initialise_chunk.cpp, generate_chunk.cpp). */
void oc_build_field(oc_chunk *c);
void oc_initialise_chunk(oc_chunk *c, double xmin, double ymin, double xmax, double ymax);
void oc_generate_chunk(oc_chunk *c, int nstates, const oc_state *states);

/* Per-phase kernels. */
void oc_ideal_gas(oc_chunk *c, int predict);
void oc_viscosity(oc_chunk *c);
double oc_calc_dt(oc_chunk *c, double dtmin, double dtc_safe, double dtu_safe, double dtv_safe,
                  double dtdiv_safe, int *control, int *jldt, int *kldt, int *small);
void oc_pdv_kernel(oc_chunk *c, int predict, double dt);
void oc_revert(oc_chunk *c);
void oc_accelerate(oc_chunk *c, double dt);
void oc_flux_calc(oc_chunk *c, double dt);
void oc_advec_cell(oc_chunk *c, int sweep_number, int dir);
void oc_advec_mom(oc_chunk *c, int which_vel, int sweep_number, int direction);
void oc_reset_field(oc_chunk *c);
void oc_update_halo(oc_chunk *c, const int fields[15], int depth);
void oc_update_halo_faces(oc_chunk *c, const int fields[15], int depth, int faces); /* :41-71, faces masked */
void oc_tile_halo(oc_chunk *dst, const oc_chunk *src, int side, const int fields[15], int depth); /* update_tile_halo_kernel.cpp */
void oc_field_summary(oc_chunk *c, double out[5]);
/* The same sums in exactly rounded form (per-cell terms identical, sum with
 * a double-double accumulator): the order-free value of the five sums. */
void oc_field_summary_exact(oc_chunk *c, double out[5]);

/* Driver-level composites. */
void oc_pdv(oc_chunk *c, int predict, double dt);   /* src/serial/PdV.cpp:92-133 */
void oc_advection(oc_chunk *c, int advect_x);       /* driver/advection.cpp:29-105 */

/* Whole run: driver/start.cpp:43-138 + driver/hydro.cpp:46-223.  Fills up to
 * max_summaries records (step 0 first, then every summary_frequency steps,
 * then the final one) and returns how many were written, or -1 on error.
 * The chunk is left in its final state. */
int oc_run(oc_chunk *c, const oc_config *cfg, oc_summary *summaries, int max_summaries,
           int *steps_done, double *dt_trace, int dt_trace_len);

#ifdef __cplusplus
}
#endif
#endif
