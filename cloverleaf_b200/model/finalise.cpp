// finalise.cpp -- driver/finalise.h:24.  Releases the device chunk (the
// reference CUDA model frees its buffers here, src/cuda/finalise.cpp:22-58).
// When CLOVER_CAPTURE_FIELDS names a file it first writes the interior of the
// final fields in the CLVF format the oracle's capture hook uses:
//   "CLVF", int32 nx, ny, nfields, then per field int32 id, w, h and w*h doubles.
#include "finalise.h"
#include "b200_runtime.h"

#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <vector>

static void put(FILE *out, cb_chunk *c, int id, int nx, int ny, int w, int h) {
  int sx = 0, sy = 0;
  cb_get_extent(c, id, &sx, &sy);
  std::vector<double> buf((size_t)sx * sy);
  clover::b200_check(cb_read_field(c, id, buf.data(), buf.size(), CB_LAYOUT_XFAST), "finalise");
  int32_t hdr[3] = {id, w, h};
  std::fwrite(hdr, sizeof(int32_t), 3, out);
  for (int k = 0; k < h; ++k) std::fwrite(&buf[(size_t)(2 + k) * sx + 2], sizeof(double), w, out);
  (void)nx;
  (void)ny;
}

void finalise(global_variables &globals) {
  if (!globals.context.rt || !globals.context.rt->chunk) return;
  cb_chunk *c = globals.context.rt->chunk;
  if (const char *path = std::getenv("CLOVER_CAPTURE_FIELDS")) {
    if (FILE *out = std::fopen(path, "wb")) {
      const tile_info &ti = globals.chunk.tiles[0].info;
      const int nx = ti.t_xmax - ti.t_xmin + 1, ny = ti.t_ymax - ti.t_ymin + 1;
      int32_t hdr[3] = {nx, ny, 9};
      std::fwrite("CLVF", 1, 4, out);
      std::fwrite(hdr, sizeof(int32_t), 3, out);
      put(out, c, CB_DENSITY0, nx, ny, nx, ny);
      put(out, c, CB_ENERGY0, nx, ny, nx, ny);
      put(out, c, CB_PRESSURE, nx, ny, nx, ny);
      put(out, c, CB_VISCOSITY, nx, ny, nx, ny);
      put(out, c, CB_SOUNDSPEED, nx, ny, nx, ny);
      put(out, c, CB_XVEL0, nx, ny, nx + 1, ny + 1);
      put(out, c, CB_YVEL0, nx, ny, nx + 1, ny + 1);
      put(out, c, CB_VOL_FLUX_X, nx, ny, nx + 1, ny);
      put(out, c, CB_VOL_FLUX_Y, nx, ny, nx, ny + 1);
      std::fclose(out);
    }
  }
  cb_destroy(c);
  globals.context.rt->chunk = nullptr;
}
