// pack_kernel.cpp -- driver/pack_kernel.h:25-48.  MPI halo packing; only a
// decomposed run calls these, which the b200 model does not support.
#include "pack_kernel.h"
#include "b200_runtime.h"

#define B200_NO_PACK(name)                                                                                                       \
  void name(global_variables &, int, int, int, int, clover::Buffer2D<double> &, clover::Buffer1D<double> &, int, int, int, int, \
            int, int, int) {                                                                                                     \
    clover::b200_fatal(#name ": the b200 model does not run MPI-decomposed meshes");                                             \
  }
B200_NO_PACK(clover_pack_message_left)
B200_NO_PACK(clover_unpack_message_left)
B200_NO_PACK(clover_pack_message_right)
B200_NO_PACK(clover_unpack_message_right)
B200_NO_PACK(clover_pack_message_top)
B200_NO_PACK(clover_unpack_message_top)
B200_NO_PACK(clover_pack_message_bottom)
B200_NO_PACK(clover_unpack_message_bottom)
