// cb_adj.cu -- the adjoint part of the C ABI (cb_adjoint_* in
// include/cloverb200.h): the gradient of the final kinetic energy with
// respect to the initial density, energy and gamma, with the dt sequence of
// the forward run held fixed, by reverse sweeps of hand-written adjoint
// kernels (cb_adj.cuh) over sqrt(N)-step checkpoints; and the tangent-linear
// run that checks it.
//
// The primal run is the FP64 plain path itself: a cb_chunk advanced through
// the C ABI in the driver's call order.  Checkpoints hold the level-0 state
// (the only state a step carries: every other field is recomputed inside
// the step).  The reverse sweep restores a checkpoint, re-runs its segment
// keeping each step's start state, and for each step from the last re-runs
// it once more while copying the inputs of every phase (the step's tape),
// then runs the phases' adjoint kernels in reverse order.
//
// Compiled with -fmad=false: the tangent-linear kernels reproduce the plain
// path's values bit for bit.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "../../include/cloverb200.h"
#include "cb_adj.cuh"
#include "cb_chunk.h"

namespace cb {
int set_last_error(int code, const std::string &msg);
} // namespace cb

using namespace cb;
using namespace cb::adj;

namespace {

// Slots of the step tape (primal values) and of the adjoint slabs.
enum Tape { S_R0, S_E0, S_U0, S_V0, S_P1, S_Q, S_P3, S_U4, S_V4, S_R5, S_E5, S_FX, S_FY, S_R7, S_E7, S_M7, S_U8, S_V8, S_R9, S_E9, S_M9, NTAPE };
enum Bar {
  B_R0, B_E0, B_U0, B_V0, B_P1, B_Q, B_P3, B_U4, B_V4, B_R5, B_E5, B_FX, B_FY, B_R7, B_E7, B_M7, B_U8, B_V8, B_R9, B_E9, B_M9, B_U10,
  B_V10, W_PV, W_EF, W_NF, W_CM, W_NMPRE, W_NMPOST, W_MFU, W_MFV, NBAR
};
// Primal work arrays of the adjoint sweeps.
enum Work { P_PV, P_MF, P_EF, P_NF, P_CM, P_NMPOST, P_NMPRE, P_MFU, P_MFV, NWORK };
// Tangent-linear slots: the 15 fields, the advection outputs, work arrays.
enum Tl { T_FIELDS = 15, T_R1N = 15, T_E1N, T_U1N, T_V1N, T_PV, T_EF, T_NF, T_CM, T_NMPOST, T_NMPRE, T_FU, T_FV, NTL };

int fail(int code, const std::string &m) { return set_last_error(code, m); }
int cuda_fail(cudaError_t e, const char *where) {
  return fail(CB_ECUDA, std::string(where) + ": " + cudaGetErrorName(e) + ": " + cudaGetErrorString(e));
}

#define ACUDA(expr)                                                                                                                          \
  do {                                                                                                                                       \
    cudaError_t _e = (expr);                                                                                                                 \
    if (_e != cudaSuccess) return cuda_fail(_e, __func__);                                                                                   \
  } while (0)
#define ACALL(expr)                                                                                                                          \
  do {                                                                                                                                       \
    int _r = (expr);                                                                                                                         \
    if (_r != CB_OK) return _r;                                                                                                              \
  } while (0)

} // namespace

struct cb_adjoint {
  cb_deck deck{};
  int nx = 0, ny = 0;
  double gamma = 1.4;
  cb_chunk *prim = nullptr;
  std::vector<double> rho_init, e_init; // interior initial values (x fastest)
  bool have_initial = false;
  // last forward run
  int nsteps = 0;
  std::vector<double> dts;
  int K = 0, K_req = 0;                 // checkpoint interval (0 requested = ceil(sqrt(N)))
  std::vector<double *> ck;             // 4 slabs per checkpoint: density0, energy0, xvel0, yvel0
  std::vector<double *> seg;            // 4 slabs per step of a segment
  double *fin[4] = {};                  // the last forward run's final level-0 state
  double *tape[NTAPE] = {};
  double *bar[NBAR] = {};
  double *work[NWORK] = {};
  double *tl_v[NTL] = {}, *tl_d[NTL] = {};
  double *d_scal = nullptr;             // [0] gamma adjoint, [1] ke, [2] dke
  double *d_terms = nullptr;            // per-cell ke terms (value, tangent)
  size_t slab_bytes = 0;
  size_t device_bytes = 0;
  long long recomputed = 0;             // steps re-run by the last reverse sweep
  bool forward_ok = false;

  double *slab(double *p) const { return p + prim->off; } // element (0, 0)
  Grid grid() const {
    Grid g;
    g.nx = nx;
    g.ny = ny;
    g.pitch = (int)prim->pitch;
    g.cdx = prim->geom_d[CELLDX];
    g.cdy = prim->geom_d[CELLDY];
    g.vdx = prim->geom_d[VERTEXDX];
    g.vdy = prim->geom_d[VERTEXDY];
    return g;
  }
};

namespace {

cudaError_t new_slab(cb_adjoint *a, double **p) {
  cudaError_t e = cudaMalloc(p, a->slab_bytes);
  if (e == cudaSuccess) {
    a->device_bytes += a->slab_bytes;
    e = cudaMemsetAsync(*p, 0, a->slab_bytes, a->prim->stream);
  }
  return e;
}

void free_slabs(cb_adjoint *a, std::vector<double *> &v) {
  for (double *p : v)
    if (p) cudaFree(p), a->device_bytes -= a->slab_bytes;
  v.clear();
}

cudaError_t zero(cb_adjoint *a, double *p) { return cudaMemsetAsync(p, 0, a->slab_bytes, a->prim->stream); }

// Copies field f of the primal chunk (whole allocation, halos included) to/from a slab.
cudaError_t save_field(cb_adjoint *a, int f, double *dst) {
  return cudaMemcpyAsync(dst, a->prim->buf[a->prim->fbuf[f]], a->slab_bytes, cudaMemcpyDeviceToDevice, a->prim->stream);
}
cudaError_t load_field(cb_adjoint *a, int f, const double *src) {
  return cudaMemcpyAsync(a->prim->buf[a->prim->fbuf[f]], src, a->slab_bytes, cudaMemcpyDeviceToDevice, a->prim->stream);
}

const int LEVEL0[4] = {CB_DENSITY0, CB_ENERGY0, CB_XVEL0, CB_YVEL0};

int save_state(cb_adjoint *a, double *const *dst) {
  for (int k = 0; k < 4; ++k) ACUDA(save_field(a, LEVEL0[k], dst[k]));
  return CB_OK;
}
int load_state(cb_adjoint *a, double *const *src) {
  for (int k = 0; k < 4; ++k) ACUDA(load_field(a, LEVEL0[k], src[k]));
  return CB_OK;
}

int update_halo(cb_chunk *c, std::initializer_list<int> fl, int depth) {
  int f[15] = {};
  for (int x : fl) f[x] = 1;
  return cb_update_halo(c, f, depth);
}

// driver/start.cpp:43-138 with the interior density0 / energy0 replaced by
// the initial values, before the halo update.
int start(cb_adjoint *a) {
  cb_chunk *c = a->prim;
  const cb_deck &d = a->deck;
  ACALL(cb_build_field(c));
  ACALL(cb_initialise_chunk(c, d.xmin, d.ymin, d.xmax, d.ymax));
  ACALL(cb_generate_chunk(c, d.nstates, d.states));
  ACALL(cb_set_gamma(c, a->gamma));
  const size_t row = sizeof(double) * a->nx;
  for (int k = 0; k < 2; ++k) {
    const std::vector<double> &h = k == 0 ? a->rho_init : a->e_init;
    double *dst = (double *)c->base(k == 0 ? CB_DENSITY0 : CB_ENERGY0) + 2 * c->pitch + 2;
    ACUDA(cudaMemcpy2DAsync(dst, sizeof(double) * c->pitch, h.data(), row, row, a->ny, cudaMemcpyHostToDevice, c->stream));
  }
  ACUDA(cudaStreamSynchronize(c->stream));
  ACALL(cb_ideal_gas(c, 0, 0));
  ACALL(update_halo(c, {CB_DENSITY0, CB_ENERGY0, CB_PRESSURE, CB_VISCOSITY, CB_DENSITY1, CB_ENERGY1, CB_XVEL0, CB_YVEL0, CB_XVEL1, CB_YVEL1}, 2));
  return CB_OK;
}

// One step of the plain path (HydroRun.hydro_step / driver/hydro.cpp:53-89)
// with dt given.  tape != null: the inputs each phase's adjoint needs are
// copied into the tape as the step runs.
int step(cb_adjoint *a, int n, double dt, double *const *tape) {
  cb_chunk *c = a->prim;
  const int d1 = (n % 2 == 1) ? 1 : 2, d2 = 3 - d1;
  auto save = [&](int f, int slot) -> cudaError_t { return tape ? save_field(a, f, tape[slot]) : cudaSuccess; };
  if (tape)
    for (int k = 0; k < 4; ++k) ACUDA(save(LEVEL0[k], S_R0 + k));
  ACALL(cb_ideal_gas(c, 0, 1));
  ACUDA(save(CB_PRESSURE, S_P1));
  ACALL(update_halo(c, {CB_PRESSURE, CB_ENERGY0, CB_DENSITY0, CB_XVEL0, CB_YVEL0}, 1));
  ACALL(cb_viscosity(c, 1));
  ACUDA(save(CB_VISCOSITY, S_Q));
  ACALL(update_halo(c, {CB_VISCOSITY}, 1));
  ACALL(cb_pdv(c, 1, dt, 1, 1));
  ACUDA(save(CB_PRESSURE, S_P3));
  ACALL(cb_accelerate(c, dt, 2));
  ACUDA(save(CB_XVEL1, S_U4));
  ACUDA(save(CB_YVEL1, S_V4));
  ACALL(cb_pdv(c, 0, dt, 0, 2));
  ACUDA(save(CB_DENSITY1, S_R5));
  ACUDA(save(CB_ENERGY1, S_E5));
  ACALL(cb_flux_calc(c, dt, 2));
  ACUDA(save(CB_VOL_FLUX_X, S_FX));
  ACUDA(save(CB_VOL_FLUX_Y, S_FY));
  ACALL(update_halo(c, {CB_ENERGY1, CB_DENSITY1, CB_VOL_FLUX_X, CB_VOL_FLUX_Y}, 2));
  ACALL(cb_advec_cell(c, 1, d1, 2));
  ACUDA(save(CB_DENSITY1, S_R7));
  ACUDA(save(CB_ENERGY1, S_E7));
  ACUDA(save(d1 == 1 ? CB_MASS_FLUX_X : CB_MASS_FLUX_Y, S_M7));
  ACALL(update_halo(c, {CB_DENSITY1, CB_ENERGY1, CB_XVEL1, CB_YVEL1, CB_MASS_FLUX_X, CB_MASS_FLUX_Y}, 2));
  ACALL(cb_advec_mom(c, 3, 1, d1, 2));
  ACUDA(save(CB_XVEL1, S_U8));
  ACUDA(save(CB_YVEL1, S_V8));
  ACALL(cb_advec_cell(c, 2, d2, 2));
  ACUDA(save(CB_DENSITY1, S_R9));
  ACUDA(save(CB_ENERGY1, S_E9));
  ACUDA(save(d2 == 1 ? CB_MASS_FLUX_X : CB_MASS_FLUX_Y, S_M9));
  ACALL(update_halo(c, {CB_DENSITY1, CB_ENERGY1, CB_XVEL1, CB_YVEL1, CB_MASS_FLUX_X, CB_MASS_FLUX_Y}, 2));
  ACALL(cb_advec_mom(c, 3, 2, d2, 0));
  ACALL(cb_reset_field(c, 1));
  return CB_OK;
}

// driver/timestep.cpp:75-96: dt from calc_dt, clamped by dtold * dtrise and dtmax.
int record_dt(cb_adjoint *a, double dtold, double *dt) {
  const cb_deck &d = a->deck;
  ACALL(cb_ideal_gas(a->prim, 0, 1));
  ACALL(cb_viscosity(a->prim, 1));
  cb_dt_params p{d.dtmin, d.dtc_safe, d.dtu_safe, d.dtv_safe, d.dtdiv_safe};
  double dtlp = 0.0;
  int control, jl, kl, small;
  ACALL(cb_calc_dt(a->prim, &p, &dtlp, &control, &jl, &kl, &small));
  double v = 1.0e21;
  if (dtlp <= v) v = dtlp;
  double m = dtold * d.dtrise;
  m = m < v ? m : v;
  v = d.dtmax < m ? d.dtmax : m;
  if (v < d.dtmin) return fail(CB_ESTATE, "cb_adjoint_forward: small timestep " + std::to_string(v));
  *dt = v;
  return CB_OK;
}

dim3 grid_of(int w, int h) { return dim3((unsigned)((w + 31) / 32), (unsigned)((h + 7) / 8)); }
const dim3 BLK(32, 8);

// --------------------------------------------------------------------------
// Tangent-linear run
// --------------------------------------------------------------------------

struct TlState {
  int map[NTL]; // slot -> slab index (the advection outputs swap with their inputs)
};

int tl_halo(cb_adjoint *a, double *v, double *d, int field, int depth) {
  const Grid g = a->grid();
  const int len = std::max(a->nx, a->ny) + 5 + 2 * depth;
  for (int pass = 0; pass < 2; ++pass) {
    k_tl_halo<<<(len + 127) / 128, 128, 0, a->prim->stream>>>(g, VD{v, d}, field, depth, pass);
    ACUDA(cudaGetLastError());
  }
  return CB_OK;
}

int adj_unfold(cb_adjoint *a, double *b, int field, int depth) {
  const Grid g = a->grid();
  const int len = std::max(a->nx, a->ny) + 5 + 2 * depth;
  for (int pass = 1; pass >= 0; --pass) {
    k_adj_unfold<<<(len + 127) / 128, 128, 0, a->prim->stream>>>(g, a->slab(b), field, depth, pass);
    ACUDA(cudaGetLastError());
  }
  return CB_OK;
}

} // namespace

extern "C" {

int cb_adjoint_create(const cb_deck *deck, int device, cb_adjoint **out) {
  if (!out || !deck) return fail(CB_EINVAL, "cb_adjoint_create: null argument");
  *out = nullptr;
  if (deck->nx < 8 || deck->ny < 8) return fail(CB_EINVAL, "cb_adjoint_create: mesh must have at least 8 cells per direction");
  if (deck->nstates < 1 || deck->nstates > CB_DECK_MAX_STATES) return fail(CB_EINVAL, "cb_adjoint_create: needs 1 to 8 states");
  if (!(deck->gamma > 1.0)) return fail(CB_EINVAL, "cb_adjoint_create: gamma must be above 1");
  cb_adjoint *a = new (std::nothrow) cb_adjoint();
  if (!a) return fail(CB_ENOMEM, "cb_adjoint_create: out of host memory");
  a->deck = *deck;
  a->nx = deck->nx;
  a->ny = deck->ny;
  a->gamma = deck->gamma;
  int r = cb_create(deck->nx, deck->ny, CB_FP64, device, &a->prim);
  if (r != CB_OK) {
    delete a;
    return r;
  }
  a->slab_bytes = a->prim->alloc_elems * sizeof(double);
  auto bail = [&](cudaError_t e) {
    cb_adjoint_destroy(a);
    return cuda_fail(e, "cb_adjoint_create");
  };
  cudaError_t e = cudaSuccess;
  for (auto &p : a->tape)
    if ((e = new_slab(a, &p)) != cudaSuccess) return bail(e);
  for (auto &p : a->fin)
    if ((e = new_slab(a, &p)) != cudaSuccess) return bail(e);
  for (auto &p : a->bar)
    if ((e = new_slab(a, &p)) != cudaSuccess) return bail(e);
  for (auto &p : a->work)
    if ((e = new_slab(a, &p)) != cudaSuccess) return bail(e);
  for (int k = 0; k < NTL; ++k) {
    if ((e = new_slab(a, &a->tl_v[k])) != cudaSuccess) return bail(e);
    if ((e = new_slab(a, &a->tl_d[k])) != cudaSuccess) return bail(e);
  }
  if ((e = cudaMalloc(&a->d_scal, sizeof(double) * 4)) != cudaSuccess) return bail(e);
  if ((e = cudaMalloc(&a->d_terms, sizeof(double) * 2 * (size_t)a->nx * a->ny)) != cudaSuccess) return bail(e);
  a->device_bytes += sizeof(double) * (4 + 2 * (size_t)a->nx * a->ny);
  // default initial state: the deck's own
  a->rho_init.assign((size_t)a->nx * a->ny, 0.0);
  a->e_init.assign((size_t)a->nx * a->ny, 0.0);
  r = cb_build_field(a->prim);
  if (r == CB_OK) r = cb_initialise_chunk(a->prim, deck->xmin, deck->ymin, deck->xmax, deck->ymax);
  if (r == CB_OK) r = cb_generate_chunk(a->prim, deck->nstates, deck->states);
  if (r == CB_OK) {
    const size_t row = sizeof(double) * a->nx;
    for (int k = 0; k < 2 && e == cudaSuccess; ++k) {
      const double *src = (const double *)a->prim->base(k == 0 ? CB_DENSITY0 : CB_ENERGY0) + 2 * a->prim->pitch + 2;
      e = cudaMemcpy2D((k == 0 ? a->rho_init : a->e_init).data(), row, src, sizeof(double) * a->prim->pitch, row, a->ny,
                       cudaMemcpyDeviceToHost);
    }
  }
  if (r != CB_OK || e != cudaSuccess) {
    cb_adjoint_destroy(a);
    return r != CB_OK ? r : cuda_fail(e, "cb_adjoint_create");
  }
  a->have_initial = true;
  *out = a;
  return CB_OK;
}

int cb_adjoint_destroy(cb_adjoint *a) {
  if (!a) return CB_OK;
  if (a->prim) cudaStreamSynchronize(a->prim->stream);
  free_slabs(a, a->ck);
  free_slabs(a, a->seg);
  for (auto &p : a->tape) cudaFree(p);
  for (auto &p : a->fin) cudaFree(p);
  for (auto &p : a->bar) cudaFree(p);
  for (auto &p : a->work) cudaFree(p);
  for (int k = 0; k < NTL; ++k) cudaFree(a->tl_v[k]), cudaFree(a->tl_d[k]);
  cudaFree(a->d_scal);
  cudaFree(a->d_terms);
  if (a->prim) cb_destroy(a->prim);
  delete a;
  return CB_OK;
}

int cb_adjoint_set_initial(cb_adjoint *a, const double *density0, const double *energy0, double gamma) {
  if (!a || !density0 || !energy0) return fail(CB_EINVAL, "cb_adjoint_set_initial: null argument");
  if (!(gamma > 1.0) || !std::isfinite(gamma)) return fail(CB_EINVAL, "cb_adjoint_set_initial: gamma must be a finite value above 1");
  const size_t n = (size_t)a->nx * a->ny;
  a->rho_init.assign(density0, density0 + n);
  a->e_init.assign(energy0, energy0 + n);
  a->gamma = gamma;
  a->forward_ok = false;
  return CB_OK;
}

int cb_adjoint_set_checkpoint_interval(cb_adjoint *a, int k) {
  if (!a || k < 0) return fail(CB_EINVAL, "cb_adjoint_set_checkpoint_interval: bad argument");
  a->K_req = k;
  return CB_OK;
}

int cb_adjoint_forward(cb_adjoint *a, int steps, const double *dt, double *ke) {
  if (!a || steps < 1) return fail(CB_EINVAL, "cb_adjoint_forward: need at least one step");
  ACUDA(cudaSetDevice(a->prim->device));
  a->forward_ok = false;
  a->K = a->K_req > 0 ? std::min(a->K_req, steps) : std::max(1, (int)std::ceil(std::sqrt((double)steps)));
  const int nck = (steps + a->K - 1) / a->K; // checkpoints at steps 0, K, 2K, ... below steps
  free_slabs(a, a->seg);
  if ((int)a->ck.size() != 4 * nck) {
    free_slabs(a, a->ck);
    a->ck.assign(4 * nck, nullptr);
    for (auto &p : a->ck) ACUDA(new_slab(a, &p));
  }
  a->seg.assign(4 * a->K, nullptr);
  for (auto &p : a->seg) ACUDA(new_slab(a, &p));
  ACALL(start(a));
  std::vector<double> rec;
  double dtold = a->deck.dtinit;
  for (int n = 1; n <= steps; ++n) {
    if ((n - 1) % a->K == 0) ACALL(save_state(a, &a->ck[4 * ((n - 1) / a->K)]));
    double h;
    if (dt) {
      h = dt[n - 1];
    } else {
      ACALL(record_dt(a, dtold, &h));
      dtold = h;
    }
    rec.push_back(h);
    ACALL(step(a, n, h, nullptr));
  }
  ACALL(save_state(a, a->fin));
  double s[5];
  ACALL(cb_field_summary(a->prim, s));
  if (ke) *ke = s[3];
  a->dts = rec;
  a->nsteps = steps;
  a->forward_ok = true;
  return CB_OK;
}

int cb_adjoint_dt(const cb_adjoint *a, double *out, int max_steps, int *count) {
  if (!a || !out) return fail(CB_EINVAL, "cb_adjoint_dt: null argument");
  const int n = std::min((int)a->dts.size(), max_steps);
  std::copy(a->dts.begin(), a->dts.begin() + n, out);
  if (count) *count = n;
  return CB_OK;
}

int cb_adjoint_gradient(cb_adjoint *a, double *g_density0, double *g_energy0, double *g_gamma) {
  if (!a) return fail(CB_EINVAL, "cb_adjoint_gradient: null adjoint");
  if (!a->forward_ok) return fail(CB_ESTATE, "cb_adjoint_gradient: run cb_adjoint_forward first");
  ACUDA(cudaSetDevice(a->prim->device));
  cudaStream_t st = a->prim->stream;
  const Grid g = a->grid();
  const int nx = a->nx, ny = a->ny;
  const double gm1 = a->gamma - 1.0;
  auto T = [&](int k) { return a->slab(a->tape[k]); };
  auto B = [&](int k) { return a->slab(a->bar[k]); };
  auto W = [&](int k) { return a->slab(a->work[k]); };
  auto VDp = [&](double *p) { return VD{p, nullptr}; };
  double *gbar = a->d_scal;
  ACUDA(cudaMemsetAsync(gbar, 0, sizeof(double), st));
  for (auto &p : a->bar) ACUDA(zero(a, p));
  // seed: the final kinetic energy (the level-0 state after the last step)
  k_adj_ke<<<grid_of(nx, ny), BLK, 0, st>>>(g, a->slab(a->fin[0]), a->slab(a->fin[2]), a->slab(a->fin[3]), B(B_R0), B(B_U0), B(B_V0));
  ACUDA(cudaGetLastError());
  a->recomputed = 0;
  const int N = a->nsteps, K = a->K;
  for (int s = (N - 1) / K; s >= 0; --s) {
    const int first = s * K + 1, last = std::min(N, (s + 1) * K);
    // restore the checkpoint and re-run the segment, keeping each step's start state
    ACALL(load_state(a, &a->ck[4 * s]));
    for (int n = first; n <= last; ++n) {
      ACALL(save_state(a, &a->seg[4 * (n - first)]));
      if (n < last) {
        ACALL(step(a, n, a->dts[n - 1], nullptr));
        ++a->recomputed;
      }
    }
    for (int n = last; n >= first; --n) {
      // the step's tape
      ACALL(load_state(a, &a->seg[4 * (n - first)]));
      ACALL(step(a, n, a->dts[n - 1], a->tape));
      ++a->recomputed;
      const double dt = a->dts[n - 1];
      const int d1 = (n % 2 == 1) ? 1 : 2, d2 = 3 - d1;
      // reset_field: the level-0 adjoint (its depth-1 halo folded back) moves to level 1
      ACALL(adj_unfold(a, a->bar[B_R0], DENSITY0, 1));
      ACALL(adj_unfold(a, a->bar[B_E0], ENERGY0, 1));
      ACALL(adj_unfold(a, a->bar[B_U0], XVEL0, 1));
      ACALL(adj_unfold(a, a->bar[B_V0], YVEL0, 1));
      for (int k = B_P1; k < NBAR; ++k) ACUDA(zero(a, a->bar[k]));
      k_adj_add<<<grid_of(nx, ny), BLK, 0, st>>>(g, B(B_R0), B(B_R9), 2, 2, nx, ny);
      k_adj_add<<<grid_of(nx, ny), BLK, 0, st>>>(g, B(B_E0), B(B_E9), 2, 2, nx, ny);
      k_adj_add<<<grid_of(nx + 1, ny + 1), BLK, 0, st>>>(g, B(B_U0), B(B_U10), 2, 2, nx + 1, ny + 1);
      k_adj_add<<<grid_of(nx + 1, ny + 1), BLK, 0, st>>>(g, B(B_V0), B(B_V10), 2, 2, nx + 1, ny + 1);
      ACUDA(cudaGetLastError());
      for (int k = B_R0; k <= B_V0; ++k) ACUDA(zero(a, a->bar[k]));

      // advec_mom of sweep dir (mom_sweep = dir + 2 (sweep - 1)); vel: its input
      // velocities; rho, mf: its density1 and mass flux; b_un/b_vn the adjoint
      // of its output, b_u/b_v of its input, b_rho, b_mf likewise.
      auto mom = [&](int dir, int sweep, int vu, int vv, int rho, int mf, int b_un, int b_vn, int b_u, int b_v, int b_rho, int b_mf) -> int {
        const int ms = dir + 2 * (sweep - 1);
        const int na = dir == 1 ? nx : ny, nl = dir == 1 ? ny : nx;
        k_tl_mom_nf<double><<<grid_of(na + 4, nl + 1), BLK, 0, st>>>(g, dir, VDp(T(mf)), VDp(W(P_NF)));
        k_tl_mom_cm<double><<<grid_of(na + 4, nl + 2), BLK, 0, st>>>(g, dir, ms, VDp(T(rho)), VDp(T(S_FX)), VDp(T(S_FY)), VDp(W(P_CM)));
        k_tl_mom_nm<double><<<grid_of(na + 3, nl + 1), BLK, 0, st>>>(g, dir, VDp(W(P_CM)), VDp(W(P_NF)), VDp(W(P_NMPOST)), VDp(W(P_NMPRE)));
        k_tl_mom_flux<double><<<grid_of(na + 2, nl + 1), BLK, 0, st>>>(g, dir, VDp(W(P_NF)), VDp(W(P_NMPRE)), VDp(T(vu)), VDp(T(vv)),
                                                                       VDp(W(P_MFU)), VDp(W(P_MFV)));
        ACUDA(cudaGetLastError());
        for (int k = W_NF; k <= W_MFV; ++k) ACUDA(zero(a, a->bar[k]));
        k_adj_mom_update<<<grid_of(na + 1, nl + 1), BLK, 0, st>>>(g, dir, W(P_NMPRE), W(P_NMPOST), W(P_MFU), W(P_MFV), T(vu), T(vv), B(b_un),
                                                                   B(b_vn), B(b_u), B(b_v), B(W_NMPRE), B(W_NMPOST), B(W_MFU), B(W_MFV));
        k_adj_mom_flux<<<grid_of(na + 2, nl + 1), BLK, 0, st>>>(g, dir, W(P_NF), W(P_NMPRE), T(vu), T(vv), B(W_MFU), B(W_MFV), B(W_NF),
                                                                 B(W_NMPRE), B(b_u), B(b_v));
        k_adj_mom_nm<<<grid_of(na + 3, nl + 1), BLK, 0, st>>>(g, dir, B(W_NMPRE), B(W_NMPOST), B(W_NF), B(W_CM));
        k_adj_mom_cm<<<grid_of(na + 4, nl + 2), BLK, 0, st>>>(g, dir, ms, T(rho), T(S_FX), T(S_FY), B(W_CM), B(b_rho), B(B_FX), B(B_FY));
        k_adj_mom_nf<<<grid_of(na + 4, nl + 1), BLK, 0, st>>>(g, dir, B(W_NF), B(b_mf));
        ACUDA(cudaGetLastError());
        return CB_OK;
      };
      // advec_cell of sweep dir; rho/e its inputs, b_rn/b_en/b_mf the adjoints
      // of its outputs, b_r/b_e of its inputs.
      auto cell = [&](int dir, int sweep, int rho, int e, int b_rn, int b_en, int b_mf, int b_r, int b_e) -> int {
        const int na = dir == 1 ? nx : ny, nl = dir == 1 ? ny : nx;
        const int vf = dir == 1 ? S_FX : S_FY, bvf = dir == 1 ? B_FX : B_FY;
        ACALL(adj_unfold(a, a->bar[b_rn], DENSITY1, 2));
        ACALL(adj_unfold(a, a->bar[b_en], ENERGY1, 2));
        ACALL(adj_unfold(a, a->bar[b_mf], dir == 1 ? MASS_FLUX_X : MASS_FLUX_Y, 2));
        k_tl_cell_pv<double><<<grid_of(na + 2, nl), BLK, 0, st>>>(g, dir, sweep, VDp(T(S_FX)), VDp(T(S_FY)), VDp(W(P_PV)));
        k_tl_cell_face<double><<<grid_of(na + 1, nl), BLK, 0, st>>>(g, dir, VDp(T(vf)), VDp(W(P_PV)), VDp(T(rho)), VDp(T(e)), VDp(W(P_MF)),
                                                                    VDp(W(P_EF)));
        ACUDA(cudaGetLastError());
        ACUDA(zero(a, a->bar[W_PV]));
        ACUDA(zero(a, a->bar[W_EF]));
        k_adj_cell_update<<<grid_of(na, nl), BLK, 0, st>>>(g, dir, T(vf), W(P_PV), T(rho), T(e), W(P_MF), W(P_EF), B(b_rn), B(b_en), B(bvf),
                                                            B(W_PV), B(b_r), B(b_e), B(b_mf), B(W_EF));
        k_adj_cell_face<<<grid_of(na + 1, nl), BLK, 0, st>>>(g, dir, T(vf), W(P_PV), T(rho), T(e), B(b_mf), B(W_EF), B(bvf), B(W_PV), B(b_r),
                                                              B(b_e));
        k_adj_cell_pv<<<grid_of(na + 2, nl), BLK, 0, st>>>(g, dir, sweep, B(W_PV), B(B_FX), B(B_FY));
        ACUDA(cudaGetLastError());
        return CB_OK;
      };
      // advec_mom sweep 2 (no fold: its halo ring is the input's)
      k_adj_add_ring<<<grid_of(nx + 5, ny + 5), BLK, 0, st>>>(g, B(B_U10), B(B_U8), nx + 5, ny + 5, 2, nx + 2, ny + 2);
      k_adj_add_ring<<<grid_of(nx + 5, ny + 5), BLK, 0, st>>>(g, B(B_V10), B(B_V8), nx + 5, ny + 5, 2, nx + 2, ny + 2);
      ACUDA(cudaGetLastError());
      ACALL(mom(d2, 2, S_U8, S_V8, S_R9, S_M9, B_U10, B_V10, B_U8, B_V8, B_R9, B_M9));
      ACALL(cell(d2, 2, S_R7, S_E7, B_R9, B_E9, B_M9, B_R7, B_E7));
      ACALL(adj_unfold(a, a->bar[B_U8], XVEL1, 2));
      ACALL(adj_unfold(a, a->bar[B_V8], YVEL1, 2));
      ACALL(mom(d1, 1, S_U4, S_V4, S_R7, S_M7, B_U8, B_V8, B_U4, B_V4, B_R7, B_M7));
      ACALL(cell(d1, 1, S_R5, S_E5, B_R7, B_E7, B_M7, B_R5, B_E5));
      // flux_calc
      ACALL(adj_unfold(a, a->bar[B_FX], VOL_FLUX_X, 2));
      ACALL(adj_unfold(a, a->bar[B_FY], VOL_FLUX_Y, 2));
      k_adj_flux<<<grid_of(nx + 1, ny + 1), BLK, 0, st>>>(g, dt, B(B_FX), B(B_FY), B(B_U0), B(B_V0), B(B_U4), B(B_V4));
      ACUDA(cudaGetLastError());
      // PdV corrector
      ACALL(adj_unfold(a, a->bar[B_R5], DENSITY1, 2));
      ACALL(adj_unfold(a, a->bar[B_E5], ENERGY1, 2));
      k_adj_pdv<0><<<grid_of(nx, ny), BLK, 0, st>>>(g, dt, T(S_U0), T(S_V0), T(S_U4), T(S_V4), T(S_R0), T(S_E0), T(S_P3), T(S_Q), B(B_R5),
                                                    B(B_E5), nullptr, B(B_U0), B(B_V0), B(B_U4), B(B_V4), B(B_R0), B(B_E0), B(B_P3), B(B_Q), gm1,
                                                    gbar);
      ACUDA(cudaGetLastError());
      // accelerate
      ACALL(adj_unfold(a, a->bar[B_U4], XVEL1, 2));
      ACALL(adj_unfold(a, a->bar[B_V4], YVEL1, 2));
      k_adj_accelerate<<<grid_of(nx + 1, ny + 1), BLK, 0, st>>>(g, dt, T(S_R0), T(S_P3), T(S_Q), T(S_U0), T(S_V0), B(B_U4), B(B_V4), B(B_R0),
                                                                 B(B_P3), B(B_Q), B(B_U0), B(B_V0));
      ACUDA(cudaGetLastError());
      // PdV predictor (its ideal_gas pressure is the output that lives on)
      ACALL(adj_unfold(a, a->bar[B_P3], PRESSURE, 1));
      k_adj_pdv<1><<<grid_of(nx, ny), BLK, 0, st>>>(g, dt, T(S_U0), T(S_V0), nullptr, nullptr, T(S_R0), T(S_E0), T(S_P1), T(S_Q), nullptr,
                                                    nullptr, B(B_P3), B(B_U0), B(B_V0), nullptr, nullptr, B(B_R0), B(B_E0), B(B_P1), B(B_Q), gm1,
                                                    gbar);
      ACUDA(cudaGetLastError());
      // viscosity
      ACALL(adj_unfold(a, a->bar[B_Q], VISCOSITY, 1));
      k_adj_viscosity<<<grid_of(nx, ny), BLK, 0, st>>>(g, T(S_U0), T(S_V0), T(S_P1), T(S_R0), B(B_Q), B(B_U0), B(B_V0), B(B_P1), B(B_R0));
      ACUDA(cudaGetLastError());
      // ideal_gas
      ACALL(adj_unfold(a, a->bar[B_P1], PRESSURE, 1));
      k_adj_ideal_gas<<<grid_of(nx, ny), BLK, 0, st>>>(g, T(S_R0), T(S_E0), B(B_P1), B(B_R0), B(B_E0), gm1, gbar);
      ACUDA(cudaGetLastError());
    }
  }
  // the start's update_halo (depth 2) of the initial density and energy
  ACALL(adj_unfold(a, a->bar[B_R0], DENSITY0, 2));
  ACALL(adj_unfold(a, a->bar[B_E0], ENERGY0, 2));
  const size_t row = sizeof(double) * nx;
  const int pitch = (int)a->prim->pitch;
  if (g_density0)
    ACUDA(cudaMemcpy2DAsync(g_density0, row, B(B_R0) + 2 * pitch + 2, sizeof(double) * pitch, row, ny, cudaMemcpyDeviceToHost, st));
  if (g_energy0)
    ACUDA(cudaMemcpy2DAsync(g_energy0, row, B(B_E0) + 2 * pitch + 2, sizeof(double) * pitch, row, ny, cudaMemcpyDeviceToHost, st));
  double gg = 0.0;
  ACUDA(cudaMemcpyAsync(&gg, gbar, sizeof(double), cudaMemcpyDeviceToHost, st));
  ACUDA(cudaStreamSynchronize(st));
  if (g_gamma) *g_gamma = gg;
  return CB_OK;
}

int cb_adjoint_tangent(cb_adjoint *a, const double *d_density0, const double *d_energy0, double d_gamma, double *ke, double *dke) {
  if (!a || !d_density0 || !d_energy0) return fail(CB_EINVAL, "cb_adjoint_tangent: null argument");
  if (!a->forward_ok) return fail(CB_ESTATE, "cb_adjoint_tangent: run cb_adjoint_forward first (it fixes the dt sequence)");
  ACUDA(cudaSetDevice(a->prim->device));
  cudaStream_t st = a->prim->stream;
  const Grid g = a->grid();
  const int nx = a->nx, ny = a->ny;
  const double gm1 = a->gamma - 1.0;
  // the initial state: values as the plain path's start, tangents of density0 / energy0
  ACALL(start(a));
  int map[NTL];
  for (int k = 0; k < NTL; ++k) map[k] = k;
  for (int k = 0; k < NTL; ++k) {
    ACUDA(zero(a, a->tl_v[k]));
    ACUDA(zero(a, a->tl_d[k]));
  }
  for (int f = 0; f < 15; ++f) ACUDA(cudaMemcpyAsync(a->tl_v[f], a->prim->buf[a->prim->fbuf[f]], a->slab_bytes, cudaMemcpyDeviceToDevice, st));
  const size_t row = sizeof(double) * nx;
  const int pitch = (int)a->prim->pitch;
  ACUDA(cudaMemcpy2DAsync(a->slab(a->tl_d[DENSITY0]) + 2 * pitch + 2, sizeof(double) * pitch, d_density0, row, row, ny, cudaMemcpyHostToDevice,
                          st));
  ACUDA(cudaMemcpy2DAsync(a->slab(a->tl_d[ENERGY0]) + 2 * pitch + 2, sizeof(double) * pitch, d_energy0, row, row, ny, cudaMemcpyHostToDevice,
                          st));
  ACUDA(cudaStreamSynchronize(st));
  auto V = [&](int k) { return VD{a->slab(a->tl_v[map[k]]), a->slab(a->tl_d[map[k]])}; };
  auto halo = [&](int k, int field, int depth) { return tl_halo(a, V(k).v, V(k).d, field, depth); };
  ACALL(halo(DENSITY0, DENSITY0, 2));
  ACALL(halo(ENERGY0, ENERGY0, 2));
  for (int n = 1; n <= a->nsteps; ++n) {
    const double dt = a->dts[n - 1];
    const int d1 = (n % 2 == 1) ? 1 : 2, d2 = 3 - d1;
    k_tl_ideal_gas<D1><<<grid_of(nx, ny), BLK, 0, st>>>(g, V(DENSITY0), V(ENERGY0), V(PRESSURE), gm1, d_gamma);
    ACUDA(cudaGetLastError());
    ACALL(halo(PRESSURE, PRESSURE, 1));
    k_tl_viscosity<D1><<<grid_of(nx, ny), BLK, 0, st>>>(g, V(XVEL0), V(YVEL0), V(PRESSURE), V(DENSITY0), V(VISCOSITY));
    ACUDA(cudaGetLastError());
    ACALL(halo(VISCOSITY, VISCOSITY, 1));
    k_tl_pdv<D1><<<grid_of(nx, ny), BLK, 0, st>>>(g, 1, dt, V(XVEL0), V(YVEL0), V(XVEL1), V(YVEL1), V(DENSITY0), V(ENERGY0), V(PRESSURE),
                                                  V(VISCOSITY), V(DENSITY1), V(ENERGY1), V(PRESSURE), gm1, d_gamma);
    ACUDA(cudaGetLastError());
    ACALL(halo(PRESSURE, PRESSURE, 1));
    k_tl_accelerate<D1><<<grid_of(nx + 1, ny + 1), BLK, 0, st>>>(g, dt, V(DENSITY0), V(PRESSURE), V(VISCOSITY), V(XVEL0), V(YVEL0), V(XVEL1),
                                                                 V(YVEL1));
    ACUDA(cudaGetLastError());
    ACALL(halo(XVEL1, XVEL1, 2));
    ACALL(halo(YVEL1, YVEL1, 2));
    k_tl_pdv<D1><<<grid_of(nx, ny), BLK, 0, st>>>(g, 0, dt, V(XVEL0), V(YVEL0), V(XVEL1), V(YVEL1), V(DENSITY0), V(ENERGY0), V(PRESSURE),
                                                  V(VISCOSITY), V(DENSITY1), V(ENERGY1), V(PRESSURE), gm1, d_gamma);
    ACUDA(cudaGetLastError());
    ACALL(halo(DENSITY1, DENSITY1, 2));
    ACALL(halo(ENERGY1, ENERGY1, 2));
    k_tl_flux<D1><<<grid_of(nx + 1, ny + 1), BLK, 0, st>>>(g, dt, V(XVEL0), V(YVEL0), V(XVEL1), V(YVEL1), V(VOL_FLUX_X), V(VOL_FLUX_Y));
    ACUDA(cudaGetLastError());
    ACALL(halo(VOL_FLUX_X, VOL_FLUX_X, 2));
    ACALL(halo(VOL_FLUX_Y, VOL_FLUX_Y, 2));
    auto cell = [&](int dir, int sweep) -> int {
      const int na = dir == 1 ? nx : ny, nl = dir == 1 ? ny : nx;
      const int vf = dir == 1 ? VOL_FLUX_X : VOL_FLUX_Y, mf = dir == 1 ? MASS_FLUX_X : MASS_FLUX_Y;
      k_tl_cell_pv<D1><<<grid_of(na + 2, nl), BLK, 0, st>>>(g, dir, sweep, V(VOL_FLUX_X), V(VOL_FLUX_Y), V(T_PV));
      k_tl_cell_face<D1><<<grid_of(na + 1, nl), BLK, 0, st>>>(g, dir, V(vf), V(T_PV), V(DENSITY1), V(ENERGY1), V(mf), V(T_EF));
      k_tl_cell_update<D1><<<grid_of(na, nl), BLK, 0, st>>>(g, dir, V(vf), V(T_PV), V(DENSITY1), V(ENERGY1), V(mf), V(T_EF), V(T_R1N),
                                                            V(T_E1N));
      ACUDA(cudaGetLastError());
      std::swap(map[DENSITY1], map[T_R1N]);
      std::swap(map[ENERGY1], map[T_E1N]);
      ACALL(halo(DENSITY1, DENSITY1, 2));
      ACALL(halo(ENERGY1, ENERGY1, 2));
      ACALL(halo(mf, mf, 2));
      return CB_OK;
    };
    auto mom = [&](int dir, int sweep) -> int {
      const int ms = dir + 2 * (sweep - 1);
      const int na = dir == 1 ? nx : ny, nl = dir == 1 ? ny : nx;
      const int mf = dir == 1 ? MASS_FLUX_X : MASS_FLUX_Y;
      k_tl_mom_nf<D1><<<grid_of(na + 4, nl + 1), BLK, 0, st>>>(g, dir, V(mf), V(T_NF));
      k_tl_mom_cm<D1><<<grid_of(na + 4, nl + 2), BLK, 0, st>>>(g, dir, ms, V(DENSITY1), V(VOL_FLUX_X), V(VOL_FLUX_Y), V(T_CM));
      k_tl_mom_nm<D1><<<grid_of(na + 3, nl + 1), BLK, 0, st>>>(g, dir, V(T_CM), V(T_NF), V(T_NMPOST), V(T_NMPRE));
      k_tl_mom_flux<D1><<<grid_of(na + 2, nl + 1), BLK, 0, st>>>(g, dir, V(T_NF), V(T_NMPRE), V(XVEL1), V(YVEL1), V(T_FU), V(T_FV));
      k_tl_mom_update<D1><<<grid_of(na + 1, nl + 1), BLK, 0, st>>>(g, dir, V(T_NMPRE), V(T_NMPOST), V(T_FU), V(T_FV), V(XVEL1), V(YVEL1),
                                                                   V(T_U1N), V(T_V1N));
      ACUDA(cudaGetLastError());
      if (sweep == 2) { // no fold: the halo ring is the input's
        k_tl_ring<D1><<<grid_of(nx + 5, ny + 5), BLK, 0, st>>>(g, V(XVEL1), V(T_U1N), nx + 5, ny + 5, 2, nx + 2, ny + 2);
        k_tl_ring<D1><<<grid_of(nx + 5, ny + 5), BLK, 0, st>>>(g, V(YVEL1), V(T_V1N), nx + 5, ny + 5, 2, nx + 2, ny + 2);
        ACUDA(cudaGetLastError());
      }
      std::swap(map[XVEL1], map[T_U1N]);
      std::swap(map[YVEL1], map[T_V1N]);
      if (sweep == 1) {
        ACALL(halo(XVEL1, XVEL1, 2));
        ACALL(halo(YVEL1, YVEL1, 2));
      }
      return CB_OK;
    };
    ACALL(cell(d1, 1));
    ACALL(mom(d1, 1));
    ACALL(cell(d2, 2));
    ACALL(mom(d2, 2));
    // reset_field
    k_tl_copy<D1><<<grid_of(nx, ny), BLK, 0, st>>>(g, V(DENSITY1), V(DENSITY0), 2, 2, nx, ny);
    k_tl_copy<D1><<<grid_of(nx, ny), BLK, 0, st>>>(g, V(ENERGY1), V(ENERGY0), 2, 2, nx, ny);
    k_tl_copy<D1><<<grid_of(nx + 1, ny + 1), BLK, 0, st>>>(g, V(XVEL1), V(XVEL0), 2, 2, nx + 1, ny + 1);
    k_tl_copy<D1><<<grid_of(nx + 1, ny + 1), BLK, 0, st>>>(g, V(YVEL1), V(YVEL0), 2, 2, nx + 1, ny + 1);
    ACUDA(cudaGetLastError());
    ACALL(halo(DENSITY0, DENSITY0, 1));
    ACALL(halo(ENERGY0, ENERGY0, 1));
    ACALL(halo(XVEL0, XVEL0, 1));
    ACALL(halo(YVEL0, YVEL0, 1));
  }
  const int nc = nx * ny;
  k_tl_ke<<<grid_of(nx, ny), BLK, 0, st>>>(g, V(DENSITY0), V(XVEL0), V(YVEL0), a->d_terms, a->d_terms + nc);
  k_sum_fixed<<<1, 256, 0, st>>>(a->d_terms, nc, a->d_scal + 1);
  k_sum_fixed<<<1, 256, 0, st>>>(a->d_terms + nc, nc, a->d_scal + 2);
  ACUDA(cudaGetLastError());
  double s[2];
  ACUDA(cudaMemcpyAsync(s, a->d_scal + 1, sizeof(s), cudaMemcpyDeviceToHost, st));
  ACUDA(cudaStreamSynchronize(st));
  // leave the tangent run's final slabs in field order for cb_adjoint_read_tangent
  std::vector<double *> v(NTL), d(NTL);
  for (int k = 0; k < NTL; ++k) v[k] = a->tl_v[map[k]], d[k] = a->tl_d[map[k]];
  for (int k = 0; k < NTL; ++k) a->tl_v[k] = v[k], a->tl_d[k] = d[k];
  if (ke) *ke = s[0];
  if (dke) *dke = s[1];
  return CB_OK;
}

int cb_adjoint_read_tangent(cb_adjoint *a, int field, int which, double *host, size_t n) {
  if (!a || !host) return fail(CB_EINVAL, "cb_adjoint_read_tangent: null argument");
  if (field < 0 || field >= 15 || which < 0 || which > 1) return fail(CB_EINVAL, "cb_adjoint_read_tangent: bad field or selector");
  int sx, sy;
  ACALL(cb_get_extent(a->prim, field, &sx, &sy));
  if (n != (size_t)sx * sy) return fail(CB_EINVAL, "cb_adjoint_read_tangent: buffer size does not match the field");
  const double *src = a->slab(which == 0 ? a->tl_v[field] : a->tl_d[field]);
  ACUDA(cudaMemcpy2D(host, sizeof(double) * sx, src, sizeof(double) * a->prim->pitch, sizeof(double) * sx, sy, cudaMemcpyDeviceToHost));
  return CB_OK;
}

int cb_adjoint_read_field(cb_adjoint *a, int field, double *host, size_t n) {
  if (!a) return fail(CB_EINVAL, "cb_adjoint_read_field: null adjoint");
  return cb_read_field(a->prim, field, host, n, CB_LAYOUT_XFAST);
}

int cb_adjoint_stats(const cb_adjoint *a, int *checkpoint_interval, int *checkpoints, long long *recomputed_steps, size_t *device_bytes) {
  if (!a) return fail(CB_EINVAL, "cb_adjoint_stats: null adjoint");
  if (checkpoint_interval) *checkpoint_interval = a->K;
  if (checkpoints) *checkpoints = (int)a->ck.size() / 4;
  if (recomputed_steps) *recomputed_steps = a->recomputed;
  if (device_bytes) *device_bytes = a->device_bytes;
  return CB_OK;
}

} // extern "C"
