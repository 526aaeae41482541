// flux_calc.cpp -- driver/flux_calc.h:24 (src/serial/flux_calc.cpp:48-61).
// Folds the depth-2 volume-flux halo of driver/advection.cpp:40-46.
#include "flux_calc.h"
#include "b200_runtime.h"
#include "timer.h"

void flux_calc(global_variables &globals) {
  double kernel_time = 0;
  if (globals.profiler_on) kernel_time = timer();
  for (int tile = 0; tile < globals.config.tiles_per_chunk; ++tile)
    clover::b200_check(cb_flux_calc(clover::b200_chunk(globals, tile), globals.dt, clover::b200_fold(globals, 2)), "flux_calc");
  clover::b200_profile_sync(globals);
  if (globals.profiler_on) globals.profiler.flux += timer() - kernel_time;
}
