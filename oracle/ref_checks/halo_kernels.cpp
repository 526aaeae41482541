// Test infrastructure: runs the reference's own halo kernels --
// update_tile_halo_{l,r,b,t}_kernel (src/serial/update_tile_halo_kernel.cpp)
// and update_halo_kernel (src/serial/update_halo.cpp:33-684) -- on seeded
// fields and writes the result, so that the C oracle's restatements
// (oc_tile_halo, oc_update_halo_faces) can be checked against the reference
// code itself.  The reference driver cannot reach these with
// tiles_per_chunk > 1 (it crashes in its tile decomposition), so they are
// called directly.  Built by oracle/Makefile (target refchecks) from the
// reference sources where they lie.
//
//   halo_kernels tile <side 1|2|4|8> <depth> <nx> <ny> <nx2> <ny2> <out>
//     dst tile nx x ny, src tile nx2 x ny2 (the src on dst's `side`); writes dst
//   halo_kernels halo <faces 0..15> <depth> <nx> <ny> <out>
//     the reflective fill of one tile whose external faces are `faces`
// Every element of field f (0..14, driver/definitions.h:61-77) of tile t starts
// as f * 1e6 + t * 1e5 + j * 300 + i + 0.25 (exact in double); the output is
// the 15 fields of dst, each x-fastest over its whole extent, as raw doubles.
#include <array>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "definitions.h"
#include "update_tile_halo_kernel.h"

void update_halo_kernel(int x_min, int x_max, int y_min, int y_max, const std::array<int, 4> &chunk_neighbours,
                        const std::array<int, 4> &tile_neighbours, field_type &field, const int fields[NUM_FIELDS], int depth);

static clover::Buffer2D<double> *field_of(field_type &f, int id) {
  clover::Buffer2D<double> *all[15] = {&f.density0, &f.density1, &f.energy0, &f.energy1, &f.pressure, &f.viscosity, &f.soundspeed,
                                       &f.xvel0, &f.xvel1, &f.yvel0, &f.yvel1, &f.vol_flux_x, &f.vol_flux_y, &f.mass_flux_x, &f.mass_flux_y};
  return all[id];
}

static void seed(field_type &f, int tile) {
  for (int id = 0; id < 15; ++id) {
    clover::Buffer2D<double> &b = *field_of(f, id);
    for (size_t i = 0; i < b.sizeX; ++i)
      for (size_t j = 0; j < b.sizeY; ++j) b(i, j) = id * 1e6 + tile * 1e5 + (double)j * 300 + (double)i + 0.25;
  }
}

static void write(field_type &f, const char *path) {
  FILE *out = std::fopen(path, "wb");
  if (!out) std::exit(2);
  for (int id = 0; id < 15; ++id) {
    clover::Buffer2D<double> &b = *field_of(f, id);
    for (size_t j = 0; j < b.sizeY; ++j)
      for (size_t i = 0; i < b.sizeX; ++i) std::fwrite(&b(i, j), sizeof(double), 1, out);
  }
  std::fclose(out);
}

int main(int argc, char **argv) {
  if (argc < 2) return 1;
  clover::context ctx;
  int fields[NUM_FIELDS];
  for (int &x : fields) x = 0;
  for (int id = 0; id < 15; ++id) fields[id] = 1;
  if (std::strcmp(argv[1], "tile") == 0 && argc == 9) {
    const int side = std::atoi(argv[2]), depth = std::atoi(argv[3]);
    const int nx = std::atoi(argv[4]), ny = std::atoi(argv[5]), nx2 = std::atoi(argv[6]), ny2 = std::atoi(argv[7]);
    field_type d(nx + 4, ny + 4, ctx), s(nx2 + 4, ny2 + 4, ctx);
    seed(d, 0);
    seed(s, 1);
    // the kernels do not read their global_variables argument
    global_variables &g = *reinterpret_cast<global_variables *>(&ctx);
    auto call = [&](auto kernel) {
      kernel(g, 1, nx, 1, ny, d.density0, d.energy0, d.pressure, d.viscosity, d.soundspeed, d.density1, d.energy1, d.xvel0, d.yvel0,
             d.xvel1, d.yvel1, d.vol_flux_x, d.vol_flux_y, d.mass_flux_x, d.mass_flux_y, 1, nx2, 1, ny2, s.density0, s.energy0,
             s.pressure, s.viscosity, s.soundspeed, s.density1, s.energy1, s.xvel0, s.yvel0, s.xvel1, s.yvel1, s.vol_flux_x,
             s.vol_flux_y, s.mass_flux_x, s.mass_flux_y, fields, depth);
    };
    if (side == 1) call(update_tile_halo_l_kernel);
    else if (side == 2) call(update_tile_halo_r_kernel);
    else if (side == 4) call(update_tile_halo_b_kernel);
    else if (side == 8) call(update_tile_halo_t_kernel);
    else return 1;
    write(d, argv[8]);
    return 0;
  }
  if (std::strcmp(argv[1], "halo") == 0 && argc == 7) {
    const int faces = std::atoi(argv[2]), depth = std::atoi(argv[3]);
    const int nx = std::atoi(argv[4]), ny = std::atoi(argv[5]);
    field_type d(nx + 4, ny + 4, ctx);
    seed(d, 0);
    const std::array<int, 4> chunk = {external_face, external_face, external_face, external_face};
    std::array<int, 4> tile = {0, 0, 0, 0};
    // tile_neighbours is indexed with tile_left, tile_right, tile_bottom, tile_top
    if (faces & 1) tile[tile_left] = external_tile;
    if (faces & 2) tile[tile_right] = external_tile;
    if (faces & 4) tile[tile_bottom] = external_tile;
    if (faces & 8) tile[tile_top] = external_tile;
    update_halo_kernel(1, nx, 1, ny, chunk, tile, d, fields, depth);
    write(d, argv[6]);
    return 0;
  }
  return 1;
}
