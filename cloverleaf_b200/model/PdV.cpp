// PdV.cpp -- driver/PdV.h:24, the model's PdV driver (src/serial/PdV.cpp:92-133).
// The predictor's kernel, ideal_gas on level 1, the depth-1 pressure halo and
// revert are one device pass (cb_pdv full = 1); the corrector folds the
// depth-2 density1/energy1 halo the advection asks for next
// (driver/advection.cpp:40-46).
#include "PdV.h"
#include "b200_runtime.h"
#include "comms.h"
#include "report.h"
#include "timer.h"

void PdV(global_variables &globals, bool predict) {
  double kernel_time = 0;
  if (globals.profiler_on) kernel_time = timer();
  globals.error_condition = 0;
  for (int tile = 0; tile < globals.config.tiles_per_chunk; ++tile) {
    cb_chunk *c = clover::b200_chunk(globals, tile);
    if (predict) clover::b200_check(cb_pdv(c, 1, globals.dt, 1, 1), "PdV");
    else clover::b200_check(cb_pdv(c, 0, globals.dt, 0, clover::b200_fold(globals, 2)), "PdV");
  }
  clover_check_error(globals.error_condition);
  clover::b200_profile_sync(globals);
  if (globals.profiler_on) globals.profiler.PdV += timer() - kernel_time;
  if (globals.error_condition == 1) report_error((char *)"PdV", (char *)"error in PdV");
}
