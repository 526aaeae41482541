// ideal_gas.cpp -- driver/ideal_gas.h:24.  Pressure and sound speed from
// level 0, or level 1 when predict (src/serial/ideal_gas.cpp:55-66).
// During the time loop the driver follows this call with
// update_halo(pressure, ..., depth 1) (driver/timestep.cpp:53-60); the kernel
// folds that pressure halo in.  At start-up (step 0) nothing is folded.
#include "ideal_gas.h"
#include "b200_runtime.h"

void ideal_gas(global_variables &globals, const int tile, bool predict) {
  const int fold = (!predict && globals.step > 0) ? clover::b200_fold(globals, 1) : 0;
  clover::b200_check(cb_ideal_gas(clover::b200_chunk(globals, tile), predict ? 1 : 0, fold), "ideal_gas");
}
