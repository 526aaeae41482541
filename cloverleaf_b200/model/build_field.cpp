// build_field.cpp -- driver/build_field.h:24.  Creates the tile's chunk on
// the device (all fields zeroed, src/serial/build_field.cpp:29-180) and binds
// every buffer of the tile's field_type to its slot.
#include "build_field.h"
#include "b200_runtime.h"

void build_field(global_variables &globals) {
  if (globals.config.tiles_per_chunk != 1 || globals.chunk.tiles.size() != 1)
    clover::b200_fatal("build_field: the b200 model runs one tile per chunk (tiles_per_chunk 1)");
  tile_type &t = globals.chunk.tiles[0];
  const int nx = t.info.t_xmax - t.info.t_xmin + 1, ny = t.info.t_ymax - t.info.t_ymin + 1;
  clover::Runtime &rt = *globals.context.rt;
  if (!rt.chunk) clover::b200_check(cb_create(nx, ny, globals.context.precision, globals.context.device, &rt.chunk), "build_field");
  clover::b200_check(cb_set_option(rt.chunk, CB_OPT_FUSE_CALLS, rt.fold && rt.fuse ? 1 : 0), "build_field");
  clover::b200_check(cb_build_field(rt.chunk), "build_field");
  field_type &f = t.field;
  cb_chunk *c = rt.chunk;
  f.density0.bind(c, CB_DENSITY0);
  f.density1.bind(c, CB_DENSITY1);
  f.energy0.bind(c, CB_ENERGY0);
  f.energy1.bind(c, CB_ENERGY1);
  f.pressure.bind(c, CB_PRESSURE);
  f.viscosity.bind(c, CB_VISCOSITY);
  f.soundspeed.bind(c, CB_SOUNDSPEED);
  f.xvel0.bind(c, CB_XVEL0);
  f.xvel1.bind(c, CB_XVEL1);
  f.yvel0.bind(c, CB_YVEL0);
  f.yvel1.bind(c, CB_YVEL1);
  f.vol_flux_x.bind(c, CB_VOL_FLUX_X);
  f.vol_flux_y.bind(c, CB_VOL_FLUX_Y);
  f.mass_flux_x.bind(c, CB_MASS_FLUX_X);
  f.mass_flux_y.bind(c, CB_MASS_FLUX_Y);
  clover::Buffer2D<double> *work[7] = {&f.work_array1, &f.work_array2, &f.work_array3, &f.work_array4,
                                       &f.work_array5, &f.work_array6, &f.work_array7};
  for (int w = 0; w < 7; ++w) work[w]->bind(c, CB_WORK_ARRAY1 + w);
  f.volume.bind(c, CB_VOLUME);
  f.xarea.bind(c, CB_XAREA);
  f.yarea.bind(c, CB_YAREA);
  f.cellx.bind(c, CB_CELLX);
  f.celly.bind(c, CB_CELLY);
  f.celldx.bind(c, CB_CELLDX);
  f.celldy.bind(c, CB_CELLDY);
  f.vertexx.bind(c, CB_VERTEXX);
  f.vertexy.bind(c, CB_VERTEXY);
  f.vertexdx.bind(c, CB_VERTEXDX);
  f.vertexdy.bind(c, CB_VERTEXDY);
}
