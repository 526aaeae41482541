// b200_runtime.h -- per-run state of the b200 model and the helpers every
// model file uses to reach the chunk on the device.
#pragma once

#include <string>

#include "cloverb200.h"
#include "context.h"
#include "definitions.h"

namespace clover {

struct Runtime {
  cb_chunk *chunk = nullptr; // the one tile's chunk (tiles_per_chunk 1)
  bool fold = true;          // fold update_halo into the producing kernels
  bool fuse = true;          // run the driver's phase calls as the library's fused passes (CB_OPT_FUSE_CALLS)
  bool ahead = true;         // with fuse: calc_dt also runs the Lagrangian pass ahead (cb_set_dt_ahead)
  // advec_mom pairing (driver/advection.cpp:56-57, :85-86): the which_vel 1
  // call advances both velocity components; the matching which_vel 2 call
  // of the same sweep is then a no-op.
  int mom_pending_dir = 0, mom_pending_sweep = 0;
};

// Aborts through the driver's report_error (driver/report.cpp:31-46) with the
// library's message when a C-ABI call fails.
void b200_check(int rc, const char *where);

// The chunk backing a tile (the model supports one tile per chunk).
cb_chunk *b200_chunk(global_variables &globals, int tile);

// The halo depth a producer folds in, or 0 when folding is off.
inline int b200_fold(global_variables &globals, int depth) { return globals.context.rt && globals.context.rt->fold ? depth : 0; }

// The reference CUDA model synchronises inside profiled regions
// (src/cuda/PdV.cpp:101-104); so does this one, only when profiling.
void b200_profile_sync(global_variables &globals, int tile = 0);

} // namespace clover
