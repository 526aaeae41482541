// b200_runtime.cpp -- shared helpers of the b200 model files.
#include "b200_runtime.h"

#include <cstdlib>
#include <iostream>

#include "report.h"

namespace clover {

[[noreturn]] void b200_fatal(const std::string &where) {
  std::string msg = "libcloverb200: " + std::string(cb_last_error());
  report_error((char *)where.c_str(), (char *)msg.c_str());
  std::abort(); // report_error does not return; keep the compiler informed
}

void b200_check(int rc, const char *where) {
  if (rc != 0) b200_fatal(where);
}

cb_chunk *b200_chunk(global_variables &globals, int tile) {
  if (tile != 0 || !globals.context.rt || !globals.context.rt->chunk)
    b200_fatal("b200 model: tile " + std::to_string(tile) + " has no device chunk (tiles_per_chunk must be 1)");
  return globals.context.rt->chunk;
}

void b200_profile_sync(global_variables &globals, int tile) {
  if (globals.profiler_on) b200_check(cb_synchronize(b200_chunk(globals, tile)), "profile");
}

} // namespace clover
