// field_summary.cpp -- driver/field_summary.h:25 (src/serial/field_summary.cpp:44-104).
// ideal_gas and the five sums are one device pass with an on-device
// reduction; five doubles come back to the host.  When CLOVER_CAPTURE_SUMMARY
// names a file the sums are also appended there at full precision (the
// driver's report prints 7 digits), in the same format as the oracle's
// capture hook, so runs can be compared value for value.
#include "field_summary.h"
#include "b200_runtime.h"
#include "report.h"
#include "timer.h"

#include <cstdio>
#include <cstdlib>

void field_summary(global_variables &globals, parallel_ &parallel) {
  clover_report_step_header(globals, parallel);
  double kernel_time = 0;
  if (globals.profiler_on) kernel_time = timer();
  double vol = 0.0, mass = 0.0, ie = 0.0, ke = 0.0, press = 0.0;
  for (int tile = 0; tile < globals.config.tiles_per_chunk; ++tile) {
    double s[5];
    clover::b200_check(cb_field_summary(clover::b200_chunk(globals, tile), s), "field_summary");
    vol += s[0];
    mass += s[1];
    ie += s[2];
    ke += s[3];
    press += s[4];
  }
  clover_sum(vol);
  clover_sum(mass);
  clover_sum(ie);
  clover_sum(ke);
  clover_sum(press);
  if (globals.profiler_on) globals.profiler.summary += timer() - kernel_time;
  if (const char *path = std::getenv("CLOVER_CAPTURE_SUMMARY")) {
    if (FILE *out = std::fopen(path, "a")) {
      std::fprintf(out, "%d %.17e %.17e %.17e %.17e %.17e %.17e\n", globals.step, globals.time, vol, mass, ie, ke, press);
      std::fclose(out);
    }
  }
  clover_report_step(globals, parallel, vol, mass, ie, ke, press);
}
