// reset_field.cpp -- driver/reset_field.h:24 (src/serial/reset_field.cpp:56-71).
// Folds the depth-1 level-0 halo of the next step's
// update_halo(pressure, energy0, density0, xvel0, yvel0; 1) (driver/timestep.cpp:53-60).
#include "reset_field.h"
#include "b200_runtime.h"
#include "timer.h"

void reset_field(global_variables &globals) {
  double kernel_time = 0;
  if (globals.profiler_on) kernel_time = timer();
  clover::Runtime &rt = *globals.context.rt;
  rt.mom_pending_dir = rt.mom_pending_sweep = 0;
  for (int tile = 0; tile < globals.config.tiles_per_chunk; ++tile)
    clover::b200_check(cb_reset_field(clover::b200_chunk(globals, tile), clover::b200_fold(globals, 1)), "reset_field");
  clover::b200_profile_sync(globals);
  if (globals.profiler_on) globals.profiler.reset += timer() - kernel_time;
}
