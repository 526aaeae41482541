// initialise_chunk.cpp -- driver/initialise_chunk.h:24: the mesh geometry
// (src/serial/initialise_chunk.cpp:30-85) of the one tile covering the chunk.
#include "initialise_chunk.h"
#include "b200_runtime.h"

void initialise_chunk(const int tile, global_variables &globals) {
  const tile_info &ti = globals.chunk.tiles[tile].info;
  if (ti.t_left != 1 || ti.t_bottom != 1 || ti.t_right != globals.config.grid.x_cells || ti.t_top != globals.config.grid.y_cells)
    clover::b200_fatal("initialise_chunk: the b200 model runs the whole mesh as one chunk and tile");
  const grid_type &g = globals.config.grid;
  clover::b200_check(cb_initialise_chunk(clover::b200_chunk(globals, tile), g.xmin, g.ymin, g.xmax, g.ymax), "initialise_chunk");
}
