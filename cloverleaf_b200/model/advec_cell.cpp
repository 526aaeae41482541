// advec_cell.cpp -- driver/advec_cell.h:24 (src/serial/advec_cell.cpp:225-232).
// Both sweeps are followed by update_halo(density1, energy1, ..., mass
// fluxes; depth 2) (driver/advection.cpp:49-55, :77-83); the kernel folds it.
#include "advec_cell.h"
#include "b200_runtime.h"

void advec_cell_driver(global_variables &globals, int tile, int sweep_number, int direction) {
  clover::b200_check(cb_advec_cell(clover::b200_chunk(globals, tile), sweep_number, direction, clover::b200_fold(globals, 2)), "advec_cell");
}
