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
// oracle/_ref/ in place of src/serial/field_summary.cpp.  It is test
// infrastructure: it performs the serial model's field summary (ideal gas,
// then the five sums in the same sequential order as
// src/serial/field_summary.cpp:44-104) and additionally appends the sums at
// full precision to the file named by CLOVER_CAPTURE_SUMMARY, because the
// driver's own report prints only 7 significant digits.
#include "field_summary.h"
#include "context.h"
#include "ideal_gas.h"
#include "report.h"
#include "timer.h"

#include <cstdio>
#include <cstdlib>

void field_summary(global_variables &globals, parallel_ &parallel) {
  clover_report_step_header(globals, parallel);

  double kernel_time = 0;
  if (globals.profiler_on) kernel_time = timer();
  for (int tile = 0; tile < globals.config.tiles_per_chunk; ++tile)
    ideal_gas(globals, tile, false);
  if (globals.profiler_on) {
    globals.profiler.ideal_gas += timer() - kernel_time;
    kernel_time = timer();
  }

  double vol = 0.0, mass = 0.0, ie = 0.0, ke = 0.0, press = 0.0;
  for (int tile = 0; tile < globals.config.tiles_per_chunk; ++tile) {
    tile_type &t = globals.chunk.tiles[tile];
    const int nx = t.info.t_xmax - t.info.t_xmin + 1;
    const int ny = t.info.t_ymax - t.info.t_ymin + 1;
    field_type &f = t.field;
    for (int idx = 0; idx < nx * ny; idx++) {
      const int j = t.info.t_xmin + 1 + idx % nx;
      const int k = t.info.t_ymin + 1 + idx / nx;
      double vsqrd = 0.0;
      for (int kv = k; kv <= k + 1; ++kv)
        for (int jv = j; jv <= j + 1; ++jv)
          vsqrd += 0.25 * (f.xvel0(jv, kv) * f.xvel0(jv, kv) + f.yvel0(jv, kv) * f.yvel0(jv, kv));
      double cell_vol = f.volume(j, k);
      double cell_mass = cell_vol * f.density0(j, k);
      vol += cell_vol;
      mass += cell_mass;
      ie += cell_mass * f.energy0(j, k);
      ke += cell_mass * 0.5 * vsqrd;
      press += cell_vol * f.pressure(j, k);
    }
  }
  clover_sum(vol);
  clover_sum(mass);
  clover_sum(ie);
  clover_sum(ke);
  clover_sum(press);
  if (globals.profiler_on) globals.profiler.summary += timer() - kernel_time;

  if (const char *path = std::getenv("CLOVER_CAPTURE_SUMMARY")) {
    if (FILE *out = std::fopen(path, "a")) {
      std::fprintf(out, "%d %.17e %.17e %.17e %.17e %.17e %.17e\n", globals.step, globals.time, vol, mass, ie, ke, press);
      std::fclose(out);
    }
  }
  clover_report_step(globals, parallel, vol, mass, ie, ke, press);
}
