// accelerate.cpp -- driver/accelerate.h:24 (src/serial/accelerate.cpp:61-74).
// Folds the depth-2 xvel1/yvel1 halo that the advection's second update_halo
// asks for (driver/advection.cpp:49-55); nothing in between changes them.
#include "accelerate.h"
#include "b200_runtime.h"
#include "timer.h"

void accelerate(global_variables &globals) {
  double kernel_time = 0;
  if (globals.profiler_on) kernel_time = timer();
  for (int tile = 0; tile < globals.config.tiles_per_chunk; ++tile)
    clover::b200_check(cb_accelerate(clover::b200_chunk(globals, tile), globals.dt, clover::b200_fold(globals, 2)), "accelerate");
  clover::b200_profile_sync(globals);
  if (globals.profiler_on) globals.profiler.acceleration += timer() - kernel_time;
}
