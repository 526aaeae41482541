// comms_kernel.cpp -- driver/comms_kernel.h:26-41.  The b200 model runs the
// whole mesh as one chunk on one GPU (no MPI decomposition), so a chunk never
// has a neighbour to exchange with; the entries stay for the driver to link
// against and fail loudly if a decomposed run ever reaches them.
#include "comms_kernel.h"
#include "b200_runtime.h"

void clover_allocate_buffers(global_variables &, parallel_ &) {}

void clover_exchange(global_variables &globals, const int *, int) {
  for (int face = 0; face < 4; ++face)
    if (globals.chunk.chunk_neighbours[face] != external_face)
      clover::b200_fatal("clover_exchange: the b200 model does not run MPI-decomposed meshes");
}

#define B200_NO_MPI(name)                                                                                                        \
  void name(global_variables &, clover::StagingBuffer1D<double>, clover::StagingBuffer1D<double>, int, int, int, MPI_Request &, \
            MPI_Request &) {                                                                                                     \
    clover::b200_fatal(#name ": the b200 model does not run MPI-decomposed meshes");                                             \
  }
B200_NO_MPI(clover_send_recv_message_left)
B200_NO_MPI(clover_send_recv_message_right)
B200_NO_MPI(clover_send_recv_message_top)
B200_NO_MPI(clover_send_recv_message_bottom)
