// update_tile_halo_kernel.cpp -- driver/update_tile_halo_kernel.h:25-86.
// Tile-to-tile halo copies happen only with tiles_per_chunk > 1, which the
// b200 model rejects in build_field; the entries exist for the driver to link.
#include "update_tile_halo_kernel.h"
#include "b200_runtime.h"

#define B2 clover::Buffer2D<double> &
#define B200_NO_TILES(name)                                                                                                      \
  void name(global_variables &, int, int, int, int, B2, B2, B2, B2, B2, B2, B2, B2, B2, B2, B2, B2, B2, B2, B2, int, int, int, \
            int, B2, B2, B2, B2, B2, B2, B2, B2, B2, B2, B2, B2, B2, B2, B2, const int *, int) {                                 \
    clover::b200_fatal(#name ": the b200 model runs one tile per chunk");                                                       \
  }
B200_NO_TILES(update_tile_halo_l_kernel)
B200_NO_TILES(update_tile_halo_r_kernel)
B200_NO_TILES(update_tile_halo_t_kernel)
B200_NO_TILES(update_tile_halo_b_kernel)
