// advec_mom.cpp -- driver/advec_mom.h:24 (src/serial/advec_mom.cpp:230-244).
// The driver calls x velocity then y velocity for each sweep
// (driver/advection.cpp:56-57, :85-86); the reference's which_vel 1 call
// builds the node fluxes and masses the which_vel 2 call reuses (:81-103).
// Here the which_vel 1 call advances both components in one pass and the
// matching which_vel 2 call does nothing.  After sweep 1 the velocities'
// depth-2 halo (asked for after the next advec_cell) is folded in.
#include "advec_mom.h"
#include "b200_runtime.h"

void advec_mom_driver(global_variables &globals, int tile, int which_vel, int direction, int sweep_number) {
  clover::Runtime &rt = *globals.context.rt;
  cb_chunk *c = clover::b200_chunk(globals, tile);
  const int fold = sweep_number == 1 ? clover::b200_fold(globals, 2) : 0;
  if (which_vel == 1) {
    clover::b200_check(cb_advec_mom(c, 3, sweep_number, direction, fold), "advec_mom");
    rt.mom_pending_dir = direction;
    rt.mom_pending_sweep = sweep_number;
    return;
  }
  if (rt.mom_pending_dir == direction && rt.mom_pending_sweep == sweep_number) {
    rt.mom_pending_dir = rt.mom_pending_sweep = 0;
    return;
  }
  clover::b200_check(cb_advec_mom(c, which_vel, sweep_number, direction, fold), "advec_mom");
}
