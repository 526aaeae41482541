// calc_dt.cpp -- driver/calc_dt.h:26-27.  The minimum over the mesh is taken
// on the device; the host receives dt_min_val and forms control / jldt /
// kldt as src/serial/calc_dt.cpp:73-79 does.  The small-timestep diagnostic
// of :85-110 is printed from device data when it triggers.  With fused calls
// the library is first given the driver's dt clamp (driver/timestep.cpp:93:
// dtold, dtrise, dtmax), so the Lagrangian pass runs on the GPU while the
// host reads the minimum back and prints the step line (not with --dump,
// whose files between the phases would show the pass's outputs early).
#include "calc_dt.h"
#include "b200_runtime.h"

#include <iostream>
#include <vector>

static double at(cb_chunk *c, int field, int i, int j) {
  int sx = 0, sy = 0;
  cb_get_extent(c, field, &sx, &sy);
  std::vector<double> buf((size_t)sx * sy);
  clover::b200_check(cb_read_field(c, field, buf.data(), buf.size(), CB_LAYOUT_XFAST), "calc_dt");
  return buf[(size_t)j * sx + i];
}

void calc_dt(global_variables &globals, int tile, double &local_dt, std::string &local_control, double &xl_pos, double &yl_pos,
             int &jldt, int &kldt) {
  local_dt = g_big;
  cb_chunk *c = clover::b200_chunk(globals, tile);
  const global_config &cfg = globals.config;
  cb_dt_params p{cfg.dtmin, cfg.dtc_safe, cfg.dtu_safe, cfg.dtv_safe, cfg.dtdiv_safe};
  int l_control = 0, small = 0;
  const clover::Runtime *rt = globals.context.rt.get();
  if (rt && rt->fold && rt->fuse && rt->ahead && cfg.dumpDir.empty())
    clover::b200_check(cb_set_dt_ahead(c, globals.dtold, cfg.dtrise, cfg.dtmax), "calc_dt");
  clover::b200_check(cb_calc_dt(c, &p, &local_dt, &l_control, &jldt, &kldt, &small), "calc_dt");
  if (small != 0) {
    const int nx = globals.chunk.tiles[tile].info.t_xmax - globals.chunk.tiles[tile].info.t_xmin + 1;
    const int ny = globals.chunk.tiles[tile].info.t_ymax - globals.chunk.tiles[tile].info.t_ymin + 1;
    std::vector<double> cellx(nx + 4), celly(ny + 4);
    cb_read_geom(c, CB_CELLX, cellx.data(), cellx.size());
    cb_read_geom(c, CB_CELLY, celly.data(), celly.size());
    std::cout << "Timestep information:" << std::endl
              << "j, k                 : " << jldt << " " << kldt << std::endl
              << "x, y                 : " << cellx[jldt] << " " << celly[kldt] << std::endl
              << "timestep : " << local_dt << std::endl
              << "Cell velocities;" << std::endl
              << at(c, CB_XVEL0, jldt, kldt) << " " << at(c, CB_YVEL0, jldt, kldt) << std::endl
              << at(c, CB_XVEL0, jldt + 1, kldt) << " " << at(c, CB_YVEL0, jldt + 1, kldt) << std::endl
              << at(c, CB_XVEL0, jldt + 1, kldt + 1) << " " << at(c, CB_YVEL0, jldt + 1, kldt + 1) << std::endl
              << at(c, CB_XVEL0, jldt, kldt + 1) << " " << at(c, CB_YVEL0, jldt, kldt + 1) << std::endl
              << "density, energy, pressure, soundspeed " << std::endl
              << at(c, CB_DENSITY0, jldt, kldt) << " " << at(c, CB_ENERGY0, jldt, kldt) << " " << at(c, CB_PRESSURE, jldt, kldt) << " "
              << at(c, CB_SOUNDSPEED, jldt, kldt) << std::endl;
  }
  if (l_control == 1) local_control = "sound";
  if (l_control == 2) local_control = "xvel";
  if (l_control == 3) local_control = "yvel";
  if (l_control == 4) local_control = "div";
  (void)xl_pos;
  (void)yl_pos;
}
