/*
 Crown Copyright 2012 AWE.

 This file is part of CloverLeaf.

 CloverLeaf is free software: you can redistribute it and/or modify it under
 the terms of the GNU General Public License as published by the
 Free Software Foundation, either version 3 of the License, or (at your option)
 any later version.

 CloverLeaf is distributed in the hope that it will be useful, but
 WITHOUT ANY WARRANTY; without even the implied warranty of MERCHANTABILITY or
 FITNESS FOR A PARTICULAR PURPOSE. See the GNU General Public License for more
 details.

 You should have received a copy of the GNU General Public License along with
 CloverLeaf. If not, see http://www.gnu.org/licenses/.
 */

// Derived from the reference's model file of the same name (the notice above
// is the reference's); modified as described below.
// Oracle capture hook -- a model file compiled INTO the reference build under
// oracle/_ref/ in place of src/serial/finalise.cpp (which does nothing).  When
// CLOVER_CAPTURE_FIELDS names a file, it writes the interior of the final
// fields as raw little-endian doubles so per-cell parity can be checked:
//   char[4] "CLVF", int32 nx, int32 ny, int32 nfields, then per field
//   int32 id, int32 w, int32 h, w*h doubles (x fastest).
// Cell fields cover [2, nx+2) x [2, ny+2); node fields [2, nx+3) x [2, ny+3).
// Field ids follow driver/definitions.h:61-77.
#include "finalise.h"
#include "context.h"

#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <vector>

static void put(FILE *out, int id, clover::Buffer2D<double> &b, int w, int h) {
  int32_t hdr[3] = {id, w, h};
  std::fwrite(hdr, sizeof(int32_t), 3, out);
  std::vector<double> row(w);
  for (int k = 0; k < h; ++k) {
    for (int j = 0; j < w; ++j) row[j] = b(2 + j, 2 + k);
    std::fwrite(row.data(), sizeof(double), w, out);
  }
}

void finalise(global_variables &globals) {
  const char *path = std::getenv("CLOVER_CAPTURE_FIELDS");
  if (!path) return;
  FILE *out = std::fopen(path, "wb");
  if (!out) return;
  tile_type &t = globals.chunk.tiles[0];
  const int nx = t.info.t_xmax - t.info.t_xmin + 1, ny = t.info.t_ymax - t.info.t_ymin + 1;
  int32_t hdr[3] = {nx, ny, 9};
  std::fwrite("CLVF", 1, 4, out);
  std::fwrite(hdr, sizeof(int32_t), 3, out);
  field_type &f = t.field;
  put(out, 0, f.density0, nx, ny);
  put(out, 2, f.energy0, nx, ny);
  put(out, 4, f.pressure, nx, ny);
  put(out, 5, f.viscosity, nx, ny);
  put(out, 6, f.soundspeed, nx, ny);
  put(out, 7, f.xvel0, nx + 1, ny + 1);
  put(out, 9, f.yvel0, nx + 1, ny + 1);
  put(out, 11, f.vol_flux_x, nx + 1, ny);
  put(out, 12, f.vol_flux_y, nx, ny + 1);
  std::fclose(out);
}
