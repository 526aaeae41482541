// viscosity.cpp -- driver/viscosity.h:24 (src/serial/viscosity.cpp:74-81).
// Folds the depth-1 viscosity halo the driver asks for next
// (driver/timestep.cpp:66-69).
#include "viscosity.h"
#include "b200_runtime.h"

void viscosity(global_variables &globals) {
  for (int tile = 0; tile < globals.config.tiles_per_chunk; ++tile)
    clover::b200_check(cb_viscosity(clover::b200_chunk(globals, tile), clover::b200_fold(globals, 1)), "viscosity");
}
