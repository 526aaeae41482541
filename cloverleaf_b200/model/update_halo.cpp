// update_halo.cpp -- driver/update_halo.h:24, with the structure of
// src/serial/update_halo.cpp:690-718: tile halos (driver code), the MPI
// exchange (comms_kernel.cpp; nothing to do on one chunk), then the
// reflective external-face fill on the device.  Fields whose halo a folded
// producer has already written are skipped by the library.
#include "update_halo.h"
#include "b200_runtime.h"
#include "comms.h"
#include "comms_kernel.h"
#include "timer.h"
#include "update_tile_halo.h"

void update_halo(global_variables &globals, int fields[NUM_FIELDS], const int depth) {
  double kernel_time = 0;
  if (globals.profiler_on) kernel_time = timer();
  update_tile_halo(globals, fields, depth);
  if (globals.profiler_on) {
    globals.profiler.tile_halo_exchange += timer() - kernel_time;
    kernel_time = timer();
  }
  clover_exchange(globals, fields, depth);
  if (globals.profiler_on) {
    globals.profiler.mpi_halo_exchange += timer() - kernel_time;
    kernel_time = timer();
  }
  const auto &nb = globals.chunk.chunk_neighbours;
  if (nb[chunk_left] == external_face || nb[chunk_right] == external_face || nb[chunk_bottom] == external_face ||
      nb[chunk_top] == external_face) {
    for (int tile = 0; tile < globals.config.tiles_per_chunk; ++tile)
      clover::b200_check(cb_update_halo(clover::b200_chunk(globals, tile), fields, depth), "update_halo");
  }
  clover::b200_profile_sync(globals);
  if (globals.profiler_on) globals.profiler.self_halo_exchange += timer() - kernel_time;
}
