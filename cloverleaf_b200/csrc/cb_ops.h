// cb_ops.h -- declarations of the phase-kernel launchers.  The definitions
// (cb_ops_impl.cuh) are compiled only in cb_fp64.cu (with -fmad=false, for
// bit parity with the reference) and cb_fp32.cu; the C-ABI translation unit
// sees these declarations alone, so no kernel is ever compiled with the
// wrong contraction setting.
#pragma once

#include <cuda_runtime.h>

#include "cb_chunk.h"

namespace cb {

struct DevState {
  double density, energy, xvel, yvel;
  int geometry;
  double xmin, ymin, xmax, ymax, radius;
};

struct DtConsts {
  double dtc_safe, dtu_safe, dtv_safe, dtdiv_safe;
};

struct HaloJob {
  int nfields;
  int field[15];
};

// The fields of one face strip (cb_pack_face / cb_unpack_face) and where
// each starts in the strip buffer (elements).
struct StripJob {
  int nfields;
  int field[15];
  long long off[15];
};

template <typename T> struct Ops {
  static cudaError_t generate_chunk(Chunk &c, const DevState *d_states, int nstates);
  static cudaError_t ideal_gas(Chunk &c, int predict, int fold);
  static cudaError_t viscosity(Chunk &c, int fold);
  static cudaError_t calc_dt(Chunk &c, const DtConsts &k);
  static cudaError_t pdv(Chunk &c, int predict, double dt, int mode, int fold);
  static cudaError_t revert(Chunk &c);
  static cudaError_t accelerate(Chunk &c, double dt, int fold);
  static cudaError_t flux_calc(Chunk &c, double dt, int fold);
  // reset_fold >= 0: the sweep also does reset_field's copy of what it writes (fold depth reset_fold)
  static cudaError_t advec_cell(Chunk &c, int sweep, int dir, int fold, void *dd, void *de, int reset_fold = -1);
  // du / dv null (with reset_fold >= 0): the velocities to level 0 only (de null in advec_cell, with
  // reset_fold >= 0 and fold 2: the energy to level 0 only)
  static cudaError_t advec_mom(Chunk &c, int vel_mask, int sweep, int dir, int fold, void *du, void *dv, int reset_fold = -1);
  // one x sweep, advec_cell then advec_mom of both velocities, as one pass over
  // the tiles away from the mesh edge and the one-phase kernels over the edge
  // strip; outputs to the spares 0..3 like advec_cell / advec_mom (the caller
  // swaps).  reset_fold >= 0: reset_field's copy too, and with level0_only the
  // new energy and velocities go to level 0 alone.  sweep_x_fusable: whether
  // the mesh has such tiles (otherwise the call is refused).
  static bool sweep_x_fusable(const Chunk &c);
  static cudaError_t advec_sweep_x(Chunk &c, int sweep, int cell_fold, int mom_fold, int reset_fold, bool level0_only,
                                   const int *store_mf = nullptr);
  static cudaError_t reset_field(Chunk &c, int fold);
  // level 1 as the phase-by-phase step leaves it, after steps whose second
  // sweeps wrote energy and velocities to level 0 only: energy1 from level 0
  // with its depth-2 halo, xvel1 / yvel1 from level 0 inside and from
  // (u_ring, v_ring), the first sweep's momentum output, on their halo ring
  static cudaError_t restore_level1(Chunk &c, const void *u_ring, const void *v_ring);
  // the reflective fill on the chunk's external faces (c.external_faces)
  static cudaError_t update_halo(Chunk &c, const HaloJob &job, int depth);
  // one strip of driver/update_tile_halo.cpp: dst's halo on `side` (CB_FACE_*) from the
  // interior of src, the neighbouring tile on that side; enqueued on dst's stream
  static cudaError_t tile_halo(Chunk &dst, const Chunk &src, int side, const HaloJob &job, int depth);
  // one face strip of driver/comms.cpp:clover_exchange between the chunk and
  // a linear device buffer: pack = the strip the neighbour on `side` needs,
  // unpack = the chunk's own halo on `side` from that neighbour's strip
  static cudaError_t face_strip(Chunk &c, int side, const StripJob &job, int depth, void *buf, bool pack);
  static cudaError_t field_summary(Chunk &c, const int *store_ps = nullptr);
  // fused passes of the resident loop: ideal_gas + viscosity + calc_dt, and the Lagrangian step
  static cudaError_t ig_visc_dt(Chunk &c, const DtConsts &k, int ig_fold, int fold, bool write_ss = true, bool write_p = true);
  // the PdV predictor, accelerate, the PdV corrector and flux_calc in one
  // pass, every output folded (depths above zero); the predicted pressure
  // goes to p_out, with the pressure's outer halo ring (which the pass does
  // not write) copied there first when keep_ring is set
  static cudaError_t lagrange(Chunk &c, void *p_out, double dt, int p_fold, int acc_fold, int pdv_fold, int flux_fold, bool keep_ring,
                              const int *store_ps = nullptr, bool p_from_de = false);
};

extern template struct Ops<double>;
extern template struct Ops<float>;

} // namespace cb
