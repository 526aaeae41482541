// revert.cpp -- driver/revert.h:24 (src/serial/revert.cpp:29-53).  The
// driver's PdV predictor reverts inside cb_pdv; this entry serves any other caller.
#include "revert.h"
#include "b200_runtime.h"

void revert(global_variables &globals) {
  for (int tile = 0; tile < globals.config.tiles_per_chunk; ++tile)
    clover::b200_check(cb_revert(clover::b200_chunk(globals, tile)), "revert");
}
