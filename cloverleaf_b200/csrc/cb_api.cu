// cb_api.cu -- the C ABI of libcloverb200 (declared in include/cloverb200.h).
//
// Host-side orchestration only: argument checks, allocation, the halo
// freshness bookkeeping that turns update_halo into a no-op after a folded
// producer, buffer swaps of the double-buffered phases, and the dispatch to
// the FP64 / FP32 kernel instantiations.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "../../include/cloverb200.h"
#include "cb_chunk.h"
#include "cb_ops.h"
#include "cb_tma.cuh"

using namespace cb;

namespace {

thread_local std::string g_err;

int fail(int code, const std::string &msg) {
  g_err = msg;
  return code;
}

int cuda_fail(cudaError_t e, const char *where) {
  return fail(CB_ECUDA, std::string(where) + ": " + cudaGetErrorName(e) + ": " + cudaGetErrorString(e));
}

// Every entry point on a chunk first runs the calls call fusion holds back
// (run_pending); the phase calls that may extend a held-back group check the
// chunk without it (CB_CHECK_CHUNK_HOLD) and decide themselves.  A Lagrangian
// pass run ahead (cb_set_dt_ahead) is settled by every entry point but the
// four calls it stands for (CB_CHECK_CHUNK_AHEAD), which match themselves
// against it.
#define CB_CHECK_CHUNK_AHEAD(c)                                                                                                              \
  do {                                                                                                                                       \
    if (!(c)) return fail(CB_EINVAL, std::string(__func__) + ": null chunk");                                                               \
    cudaError_t _e = select_device(c);                                                                                                       \
    if (_e != cudaSuccess) return cuda_fail(_e, __func__);                                                                                   \
  } while (0)

#define CB_CHECK_CHUNK_HOLD(c)                                                                                                               \
  do {                                                                                                                                       \
    CB_CHECK_CHUNK_AHEAD(c);                                                                                                                 \
    cudaError_t _e1 = settle_ahead(c);                                                                                                       \
    if (_e1 != cudaSuccess) return cuda_fail(_e1, __func__);                                                                                 \
  } while (0)

#define CB_CHECK_CHUNK(c)                                                                                                                    \
  do {                                                                                                                                       \
    CB_CHECK_CHUNK_HOLD(c);                                                                                                                  \
    cudaError_t _e2 = run_pending(c);                                                                                                        \
    if (_e2 != cudaSuccess) return cuda_fail(_e2, __func__);                                                                                 \
  } while (0)

#define CB_CUDA(expr)                                                                                                                        \
  do {                                                                                                                                       \
    cudaError_t _e = (expr);                                                                                                                 \
    if (_e != cudaSuccess) return cuda_fail(_e, __func__);                                                                                   \
  } while (0)

cudaError_t select_device(const cb_chunk *c) {
  int cur = -1;
  cudaError_t e = cudaGetDevice(&cur);
  if (e != cudaSuccess) return e;
  if (cur != c->device) return cudaSetDevice(c->device);
  return cudaSuccess;
}

// Dispatch to the instantiation of the chunk's precision.
template <typename F> cudaError_t dispatch(cb_chunk *c, F &&f) {
  if (c->precision == CB_FP64) return f(Ops<double>());
  return f(Ops<float>());
}

void field_extent(const cb_chunk *c, int f, int &sx, int &sy) {
  switch (kind_of(f)) {
    case VERTEX: sx = c->nx + 5; sy = c->ny + 5; break;
    case XFACE: sx = c->nx + 5; sy = c->ny + 4; break;
    case YFACE: sx = c->nx + 4; sy = c->ny + 5; break;
    default: sx = c->nx + 4; sy = c->ny + 4; break;
  }
}

int geom_len(const cb_chunk *c, int g) {
  switch (g) {
    case CELLX: case CELLDX: return c->nx + 4;
    case CELLY: case CELLDY: return c->ny + 4;
    case VERTEXX: case VERTEXDX: return c->nx + 5;
    default: return c->ny + 5;
  }
}

bool is_state_field(int f) { return f >= 0 && f < 15; }

// cb_advec_cell's launch and buffer swap; reset_fold >= 0: the sweep also does
// reset_field's copy of what it writes (the second sweep under call fusion).
cudaError_t launch_cell(cb_chunk *c, int sweep, int dir, int fold, int reset_fold) {
  void *dd = c->spare_base(0), *de = c->spare_base(1);
  cudaError_t e = dispatch(c, [&](auto ops) { return ops.advec_cell(*c, sweep, dir, fold, dd, de, reset_fold); });
  if (e != cudaSuccess) return e;
  std::swap(c->fbuf[DENSITY1], c->sbuf[0]);
  std::swap(c->fbuf[ENERGY1], c->sbuf[1]);
  return cudaSuccess;
}

// cb_advec_mom's launch and buffer swaps (the same reset_fold).
cudaError_t launch_mom(cb_chunk *c, int which_vel, int sweep, int dir, int fold, int reset_fold) {
  void *du = c->spare_base(2), *dv = c->spare_base(3);
  cudaError_t e = dispatch(c, [&](auto ops) { return ops.advec_mom(*c, which_vel, sweep, dir, fold, du, dv, reset_fold); });
  if (e != cudaSuccess) return e;
  if (which_vel & 1) std::swap(c->fbuf[XVEL1], c->sbuf[2]);
  if (which_vel & 2) std::swap(c->fbuf[YVEL1], c->sbuf[3]);
  return cudaSuccess;
}

bool x_fusable(const cb_chunk *c) { return c->precision == CB_FP64 ? Ops<double>::sweep_x_fusable(*c) : Ops<float>::sweep_x_fusable(*c); }

// An x sweep, cell and momentum parts, as one pass (with reset_field's copy
// when reset_fold >= 0), and the buffer swaps of both parts.
cudaError_t launch_sweep_x(cb_chunk *c, int sweep, int cell_fold, int mom_fold, int reset_fold) {
  cudaError_t e = dispatch(c, [&](auto ops) { return ops.advec_sweep_x(*c, sweep, cell_fold, mom_fold, reset_fold, false); });
  if (e != cudaSuccess) return e;
  std::swap(c->fbuf[DENSITY1], c->sbuf[0]);
  std::swap(c->fbuf[ENERGY1], c->sbuf[1]);
  std::swap(c->fbuf[XVEL1], c->sbuf[2]);
  std::swap(c->fbuf[YVEL1], c->sbuf[3]);
  return cudaSuccess;
}

// A Lagrangian pass run ahead that its calls did not all consume: the calls
// that matched it so far (their work was skipped) run now, as they were made;
// the pass's outputs are overwritten by them and by the calls still to come.
cudaError_t settle_ahead(cb_chunk *c) {
  DtAhead &a = c->ahead;
  if (!a.launched) return cudaSuccess;
  a.launched = false;
  cudaError_t e = cudaSuccess;
  const double dt = a.dt;
  if (a.stage >= 1) e = dispatch(c, [&](auto ops) { return ops.pdv(*c, 1, dt, 1, a.folds[0]); });
  if (e == cudaSuccess && a.stage >= 2) e = dispatch(c, [&](auto ops) { return ops.accelerate(*c, dt, a.folds[1]); });
  if (e == cudaSuccess && a.stage >= 3) e = dispatch(c, [&](auto ops) { return ops.pdv(*c, 0, dt, 0, a.folds[2]); });
  a.stage = 0;
  return e;
}

// Runs the calls call fusion held back, one by one as they were made.
cudaError_t run_pending(cb_chunk *c) {
  if (cudaError_t e0 = settle_ahead(c)) return e0;
  const Pending p = c->pend;
  c->pend = Pending{};
  cudaError_t e = cudaSuccess;
  auto go = [&](auto &&f) {
    if (e == cudaSuccess) e = dispatch(c, f);
  };
  switch (p.kind) {
    case PEND_IG:
    case PEND_IG_VISC:
      go([&](auto ops) { return ops.ideal_gas(*c, 0, p.ig_fold); });
      if (p.kind == PEND_IG_VISC) go([&](auto ops) { return ops.viscosity(*c, p.visc_fold); });
      break;
    case PEND_PDV1:
    case PEND_PDV1_ACC:
    case PEND_PDV1_ACC_PDV0:
      go([&](auto ops) { return ops.pdv(*c, 1, p.dt, 1, p.pdv1_fold); });
      if (p.kind != PEND_PDV1) go([&](auto ops) { return ops.accelerate(*c, p.dt, p.acc_fold); });
      if (p.kind == PEND_PDV1_ACC_PDV0) go([&](auto ops) { return ops.pdv(*c, 0, p.dt, 0, p.pdv0_fold); });
      break;
    case PEND_CELL:
    case PEND_CELL_MOM:
      e = launch_cell(c, p.cell_sweep, p.cell_dir, p.cell_fold, -1);
      if (e == cudaSuccess && p.kind == PEND_CELL_MOM) e = launch_mom(c, p.mom_mask, p.cell_sweep, p.cell_dir, p.mom_fold, -1);
      break;
    default: break;
  }
  return e;
}

int effective_fold(const cb_chunk *c, int depth) { return c->can_fold() ? depth : 0; }

int check_depth(int d, bool allow0) {
  if (d == 1 || d == 2 || (allow0 && d == 0)) return CB_OK;
  return fail(CB_EINVAL, "halo depth must be " + std::string(allow0 ? "0, 1 or 2" : "1 or 2") + ", got " + std::to_string(d));
}

cudaError_t upload_geom(cb_chunk *c) {
  {
    // reciprocals of the widths, rounded to nearest (the divisors of width_ratio)
    std::vector<double> r(4 * (size_t)c->geom_len, 0.0);
    const int src[4] = {CELLDX, CELLDY, VERTEXDX, VERTEXDY};
    for (int q = 0; q < 4; ++q)
      for (int k = 0; k < c->geom_len; ++k) {
        const double w = c->geom_h[src[q]][k];
        r[(size_t)q * c->geom_len + k] = w != 0.0 ? 1.0 / w : 0.0;
      }
    cudaError_t e = cudaMemcpyAsync(c->rgeom_d, r.data(), sizeof(double) * r.size(), cudaMemcpyHostToDevice, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream); // r dies here
    if (e != cudaSuccess) return e;
  }
  for (int g = 0; g < NUM_GEOM; ++g) {
    cudaError_t e = cudaMemcpyAsync(c->geom_d[g], c->geom_h[g], sizeof(double) * c->geom_len, cudaMemcpyHostToDevice, c->stream);
    if (e != cudaSuccess) return e;
    if (c->precision == CB_FP32) {
      std::vector<float> tmp(c->geom_len);
      for (int k = 0; k < c->geom_len; ++k) tmp[k] = (float)c->geom_h[g][k];
      e = cudaMemcpyAsync(c->geom_t[g], tmp.data(), sizeof(float) * c->geom_len, cudaMemcpyHostToDevice, c->stream);
      if (e != cudaSuccess) return e;
      e = cudaStreamSynchronize(c->stream); // tmp dies here
      if (e != cudaSuccess) return e;
    }
  }
  return cudaSuccess;
}

void release(cb_chunk *c) {
  for (auto &p : c->buf)
    if (p) cudaFree(p), p = nullptr;
  for (int g = 0; g < NUM_GEOM; ++g) {
    if (c->geom_d[g]) cudaFree(c->geom_d[g]);
    if (c->precision == CB_FP32 && c->geom_t[g]) cudaFree(c->geom_t[g]);
    delete[] c->geom_h[g];
    c->geom_d[g] = nullptr;
    c->geom_t[g] = nullptr;
    c->geom_h[g] = nullptr;
  }
  if (c->rgeom_d) cudaFree(c->rgeom_d);
  c->rgeom_d = nullptr;
  if (c->d_dt_bits) cudaFree(c->d_dt_bits);
  if (c->d_partials) cudaFree(c->d_partials);
  if (c->d_counter) cudaFree(c->d_counter);
  if (c->d_sums) cudaFree(c->d_sums);
  if (c->d_err) cudaFree(c->d_err);
  if (c->h_scalars) cudaFreeHost(c->h_scalars);
  if (c->ev_order) cudaEventDestroy(c->ev_order);
  c->ev_order = nullptr;
  if (c->ev_dt) cudaEventDestroy(c->ev_dt);
  c->ev_dt = nullptr;
  if (c->d_dt_ahead) cudaFree(c->d_dt_ahead);
  c->d_dt_ahead = nullptr;
  if (c->stream) cudaStreamDestroy(c->stream);
  c->d_dt_bits = nullptr;
  c->d_partials = nullptr;
  c->d_counter = nullptr;
  c->d_sums = nullptr;
  c->d_err = nullptr;
  c->h_scalars = nullptr;
  c->stream = nullptr;
}

using EncodeTiled = CUresult (*)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *, const cuuint64_t *,
                                 const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave, CUtensorMapSwizzle,
                                 CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

} // namespace

namespace cb {

// One 2-D tensor map per buffer and staged box height: the whole allocation
// as a (pitch x ny+6) array, boxes of BOX_X x h elements (cb_tma.cuh).
bool encode_buffer_maps(void *const *bufs, int nbuf, long long pitch, int ny, int precision, CUtensorMap (*maps)[NUM_BOX_H],
                        std::string *err) {
  static EncodeTiled encode = nullptr;
  if (!encode) {
    void *fn = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) != cudaSuccess || !fn) {
      *err = "cuTensorMapEncodeTiled is not available from the driver";
      return false;
    }
    encode = (EncodeTiled)fn;
  }
  const size_t esize = precision == CB_FP64 ? 8 : 4;
  const cuuint64_t dims[2] = {(cuuint64_t)pitch, (cuuint64_t)(ny + 6)};
  const cuuint64_t strides[1] = {(cuuint64_t)(pitch * esize)};
  const cuuint32_t estr[2] = {1, 1};
  for (int b = 0; b < nbuf; ++b)
    for (int h = 0; h < NUM_BOX_H; ++h) {
      const cuuint32_t box[2] = {(cuuint32_t)BOX_X, (cuuint32_t)BOX_HEIGHTS[h]};
      CUresult r = encode(&maps[b][h], precision == CB_FP64 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, bufs[b],
                          dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                          CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
      if (r != CUDA_SUCCESS) {
        *err = "cuTensorMapEncodeTiled failed with code " + std::to_string((int)r);
        return false;
      }
    }
  return true;
}

// The 1-D geometry of src/serial/initialise_chunk.cpp:30-85, into
// g[NUM_GEOM] arrays of at least max(nx, ny) + 5 entries, for a chunk of
// nx x ny cells whose first cell is cell (left, bottom) of a grid of
// x_cells x y_cells over [gxmin, gxmax] x [gymin, gymax] (1-based global
// indices; the chunk's own indices start at 1, as the reference's tile's).
void chunk_geometry_at(int nx, int ny, double gxmin, double gymin, double gxmax, double gymax, int x_cells, int y_cells, int left, int bottom,
                       double *const *g) {
  const int x_min = 1, y_min = 1, x_max = nx, y_max = ny;
  double dx = (gxmax - gxmin) / (double)(x_cells);
  double dy = (gymax - gymin) / (double)(y_cells);
  double xmin = gxmin + dx * (double)(left - 1);
  double ymin = gymin + dy * (double)(bottom - 1);
  const int xrange = (x_max + 3) - (x_min - 2) + 1, yrange = (y_max + 3) - (y_min - 2) + 1;
  for (int j = 0; j < xrange; j++) {
    g[VERTEXX][j] = xmin + dx * (j - 1 - x_min);
    g[VERTEXDX][j] = dx;
  }
  for (int k = 0; k < yrange; k++) {
    g[VERTEXY][k] = ymin + dy * (k - 1 - y_min);
    g[VERTEXDY][k] = dy;
  }
  const int xrange1 = (x_max + 2) - (x_min - 2) + 1, yrange1 = (y_max + 2) - (y_min - 2) + 1;
  for (int j = 0; j < xrange1; j++) {
    g[CELLX][j] = 0.5 * (g[VERTEXX][j] + g[VERTEXX][j + 1]);
    g[CELLDX][j] = dx;
  }
  for (int k = 0; k < yrange1; k++) {
    g[CELLY][k] = 0.5 * (g[VERTEXY][k] + g[VERTEXY][k + 1]);
    g[CELLDY][k] = dy;
  }
}

void chunk_geometry(int nx, int ny, double gxmin, double gymin, double gxmax, double gymax, double *const *g) {
  chunk_geometry_at(nx, ny, gxmin, gymin, gxmax, gymax, nx, ny, 1, 1, g);
}

} // namespace cb

namespace {

bool encode_maps(cb_chunk *c) {
  if (!encode_buffer_maps(c->buf, NUM_BUF, c->pitch, c->ny, c->precision, c->tmap, &g_err)) return false;
  c->tmap_ok = true;
  return true;
}

// A staging wait that gave up in some kernel leaves a flag on the device;
// the host reports it at the next point that synchronises.
int check_device_error(cb_chunk *c, const char *where) {
  int err = 0;
  cudaError_t e = cudaMemcpy(&err, c->d_err, sizeof(int), cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return cuda_fail(e, where);
  if (err) return fail(CB_ECUDA, std::string(where) + ": a kernel's tile staging did not complete (TMA wait limit reached)");
  return CB_OK;
}

} // namespace

namespace cb {
int set_last_error(int code, const std::string &msg) { return fail(code, msg); }
cudaError_t run_pending_calls(cb_chunk *c) { return run_pending(c); }
} // namespace cb

namespace {

// The driver's dt from calc_dt's minimum (driver/timestep.cpp:93):
// min(min(dtlp, dtold * dtrise), dtmax), in the same order on the host and on
// the device (std::min(a, b) is b < a ? b : a).
__host__ __device__ inline double driver_dt_clamp(double dtlp, double dtold, double dtrise, double dtmax) {
  const double r = dtold * dtrise;
  const double m = r < dtlp ? r : dtlp;
  return dtmax < m ? dtmax : m;
}

__global__ void k_dt_ahead(const unsigned long long *dt_bits, double dtold, double dtrise, double dtmax, double *dt_out) {
  *dt_out = driver_dt_clamp(__longlong_as_double((long long)*dt_bits), dtold, dtrise, dtmax);
}

// Whether a call is the next of the four the pass run ahead stands for
// (stage: the calls matched before it), with the pass's dt and halo depth;
// if so it counts as matched.  A call that does not match settles the pass.
bool ahead_match(cb_chunk *c, int stage, double dt, int fold) {
  DtAhead &a = c->ahead;
  if (!a.launched || a.stage != stage || a.dt != dt || a.folds[stage] != fold) return false;
  a.stage = stage + 1;
  return true;
}

} // namespace

extern "C" {

int cb_version(void) { return 1; }

const char *cb_last_error(void) { return g_err.c_str(); }

int cb_device_count(int *count) {
  if (!count) return fail(CB_EINVAL, "cb_device_count: null count");
  *count = 0;
  cudaError_t e = cudaGetDeviceCount(count);
  if (e != cudaSuccess) {
    *count = 0;
    return cuda_fail(e, "cb_device_count");
  }
  return CB_OK;
}

int cb_device_name(int device, char *name, size_t len) {
  if (!name || len == 0) return fail(CB_EINVAL, "cb_device_name: null buffer");
  cudaDeviceProp prop;
  cudaError_t e = cudaGetDeviceProperties(&prop, device);
  if (e != cudaSuccess) return cuda_fail(e, "cb_device_name");
  std::snprintf(name, len, "%s (sm_%d%d, %d SMs, %.1f GB)", prop.name, prop.major, prop.minor, prop.multiProcessorCount,
                prop.totalGlobalMem / 1e9);
  return CB_OK;
}

int cb_create(int nx, int ny, int precision, int device, cb_chunk **out) {
  if (!out) return fail(CB_EINVAL, "cb_create: null out");
  *out = nullptr;
  if (nx < 1 || ny < 1) return fail(CB_EINVAL, "cb_create: mesh must have at least one cell in each direction");
  if (nx > (1 << 20) || ny > (1 << 20)) return fail(CB_EINVAL, "cb_create: mesh side above 1048576 cells");
  if (precision != CB_FP64 && precision != CB_FP32) return fail(CB_EINVAL, "cb_create: precision must be CB_FP64 or CB_FP32");
  int ndev = 0;
  cudaError_t e = cudaGetDeviceCount(&ndev);
  if (e != cudaSuccess) return cuda_fail(e, "cb_create");
  if (device < 0 || device >= ndev) return fail(CB_EINVAL, "cb_create: no CUDA device " + std::to_string(device));
  if ((e = cudaSetDevice(device)) != cudaSuccess) return cuda_fail(e, "cb_create");
  cb_chunk *c = new (std::nothrow) cb_chunk();
  if (!c) return fail(CB_ENOMEM, "cb_create: out of host memory");
  c->nx = nx;
  c->ny = ny;
  c->precision = precision;
  c->device = device;
  c->esize = precision == CB_FP64 ? 8 : 4;
  // Row layout: element (i, j) at allocation + off + j * pitch + i.  off puts
  // the first interior column (i = 2) on a 256-byte boundary and makes the
  // tiles' TMA boxes (starting at i = 2 + 64k - 4) 16-byte aligned; pitch
  // covers off + nx + 5 so the tensor-map rows hold whole mesh rows.
  const long long align = 256 / (long long)c->esize;
  c->off = (size_t)(align - 2);
  c->pitch = ((long long)c->off + nx + 5 + align - 1) / align * align;
  c->alloc_elems = c->off + (size_t)c->pitch * (size_t)(ny + 6) + (size_t)align;
  if (c->alloc_elems >= (size_t)1 << 31) {
    delete c;
    return fail(CB_EINVAL, "cb_create: mesh too large (a field must hold fewer than 2^31 elements)");
  }
  const size_t bytes = c->alloc_elems * c->esize;
  auto bail = [&](cudaError_t err, const char *what) {
    release(c);
    delete c;
    if (err == cudaErrorMemoryAllocation) return fail(CB_ENOMEM, std::string("cb_create: out of device memory allocating ") + what);
    return cuda_fail(err, "cb_create");
  };
  if ((e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking)) != cudaSuccess) return bail(e, "stream");
  if ((e = cudaEventCreateWithFlags(&c->ev_order, cudaEventDisableTiming)) != cudaSuccess) return bail(e, "event");
  if ((e = cudaEventCreateWithFlags(&c->ev_dt, cudaEventDisableTiming)) != cudaSuccess) return bail(e, "event");
  for (int b = 0; b < NUM_BUF; ++b)
    if ((e = cudaMalloc(&c->buf[b], bytes)) != cudaSuccess) return bail(e, "fields");
  for (int f = 0; f < 15; ++f) c->fbuf[f] = f;
  for (int s = 0; s < NUM_SPARE; ++s) c->sbuf[s] = 15 + s;
  if (!encode_maps(c)) {
    release(c);
    delete c;
    return fail(CB_ECUDA, "cb_create: " + g_err);
  }
  c->geom_len = std::max(nx, ny) + 6;
  for (int g = 0; g < NUM_GEOM; ++g) {
    c->geom_h[g] = new (std::nothrow) double[c->geom_len]();
    if (!c->geom_h[g]) return bail(cudaErrorMemoryAllocation, "geometry");
    if ((e = cudaMalloc(&c->geom_d[g], sizeof(double) * c->geom_len)) != cudaSuccess) return bail(e, "geometry");
    if (precision == CB_FP32) {
      if ((e = cudaMalloc(&c->geom_t[g], sizeof(float) * c->geom_len)) != cudaSuccess) return bail(e, "geometry");
    } else {
      c->geom_t[g] = c->geom_d[g];
    }
  }
  if ((e = cudaMalloc(&c->rgeom_d, sizeof(double) * 4 * c->geom_len)) != cudaSuccess) return bail(e, "geometry");
  cudaDeviceGetAttribute(&c->sms, cudaDevAttrMultiProcessorCount, device);
  c->summary_grid = c->sms * 8;
  if ((e = cudaMalloc(&c->d_dt_bits, sizeof(unsigned long long))) != cudaSuccess) return bail(e, "scratch");
  if ((e = cudaMalloc(&c->d_dt_ahead, sizeof(double))) != cudaSuccess) return bail(e, "scratch");
  if ((e = cudaMalloc(&c->d_partials, sizeof(double) * 5 * (size_t)c->summary_grid)) != cudaSuccess) return bail(e, "scratch");
  if ((e = cudaMalloc(&c->d_counter, sizeof(unsigned int))) != cudaSuccess) return bail(e, "scratch");
  if ((e = cudaMalloc(&c->d_sums, sizeof(double) * 5)) != cudaSuccess) return bail(e, "scratch");
  if ((e = cudaMalloc(&c->d_err, sizeof(int))) != cudaSuccess) return bail(e, "scratch");
  if ((e = cudaMemsetAsync(c->d_err, 0, sizeof(int), c->stream)) != cudaSuccess) return bail(e, "scratch");
  if ((e = cudaMallocHost(&c->h_scalars, sizeof(double) * 8)) != cudaSuccess) return bail(e, "pinned scratch");
  if ((e = cudaMemsetAsync(c->d_counter, 0, sizeof(unsigned int), c->stream)) != cudaSuccess) return bail(e, "scratch");
  for (int b = 0; b < NUM_BUF; ++b)
    if ((e = cudaMemsetAsync(c->buf[b], 0, bytes, c->stream)) != cudaSuccess) return bail(e, "fields");
  if ((e = upload_geom(c)) != cudaSuccess) return bail(e, "geometry");
  if ((e = cudaStreamSynchronize(c->stream)) != cudaSuccess) return bail(e, "setup");
  *out = c;
  return CB_OK;
}

int cb_destroy(cb_chunk *c) {
  if (!c) return CB_OK;
  select_device(c);
  if (c->stream) cudaStreamSynchronize(c->stream);
  run_cache_free(*c);
  release(c);
  delete c;
  return CB_OK;
}

int cb_set_gamma(cb_chunk *c, double gamma) {
  CB_CHECK_CHUNK(c);
  if (!(gamma > 1.0) || !std::isfinite(gamma)) return fail(CB_EINVAL, "cb_set_gamma: gamma must be a finite value above 1");
  c->gamma = gamma;
  return CB_OK;
}

int cb_set_option(cb_chunk *c, int option, int value) {
  CB_CHECK_CHUNK(c);
  if (option == CB_OPT_FOLD_HALO) {
    c->fold_enabled = value != 0;
    std::fill(std::begin(c->halo_fresh), std::end(c->halo_fresh), 0);
  } else if (option == CB_OPT_FUSE_CALLS) {
    c->fuse_calls = value != 0;
  } else {
    return fail(CB_EINVAL, "cb_set_option: unknown option " + std::to_string(option));
  }
  return CB_OK;
}

int cb_get_extent(const cb_chunk *c, int field, int *sx, int *sy) {
  if (!c || !sx || !sy) return fail(CB_EINVAL, "cb_get_extent: null argument");
  if (field < 0 || field >= NUM_FIELDS) return fail(CB_EINVAL, "cb_get_extent: bad field id " + std::to_string(field));
  field_extent(c, field, *sx, *sy);
  return CB_OK;
}

int cb_read_field(cb_chunk *c, int field, double *host, size_t n, int layout) {
  CB_CHECK_CHUNK(c);
  if (!host) return fail(CB_EINVAL, "cb_read_field: null host buffer");
  if (field < 0 || field >= NUM_FIELDS) return fail(CB_EINVAL, "cb_read_field: bad field id " + std::to_string(field));
  if (layout != CB_LAYOUT_XFAST && layout != CB_LAYOUT_YFAST) return fail(CB_EINVAL, "cb_read_field: bad layout");
  int sx, sy;
  field_extent(c, field, sx, sy);
  if (n != (size_t)sx * (size_t)sy)
    return fail(CB_EINVAL, "cb_read_field: buffer holds " + std::to_string(n) + " values, field has " + std::to_string((size_t)sx * sy));
  if (c->precision == CB_FP64 && layout == CB_LAYOUT_XFAST && is_state_field(field)) {
    // straight pitched copy into the caller's buffer (fast when it is pinned)
    CB_CUDA(cudaMemcpy2DAsync(host, sizeof(double) * sx, c->base(field), sizeof(double) * c->pitch, sizeof(double) * sx, sy,
                              cudaMemcpyDeviceToHost, c->stream));
    CB_CUDA(cudaStreamSynchronize(c->stream));
    return CB_OK;
  }
  std::vector<double> xf((size_t)sx * sy);
  if (field >= WORK1 && field <= WORK7) {
    // work arrays are intra-phase scratch the kernels keep on chip
    std::fill(xf.begin(), xf.end(), 0.0);
  } else if (field == VOLUME || field == XAREA || field == YAREA) {
    // derived from the 1-D widths exactly as src/serial/initialise_chunk.cpp:78-84 forms them
    const double dx = c->geom_h[CELLDX][0], dy = c->geom_h[CELLDY][0];
    for (int j = 0; j < sy; ++j)
      for (int i = 0; i < sx; ++i) {
        double v = 0.0;
        const bool in_cells = i < c->nx + 4 && j < c->ny + 4;
        if (field == VOLUME) v = in_cells ? dx * dy : 0.0;
        else if (field == XAREA) v = in_cells ? c->geom_h[CELLDY][j] : 0.0;
        else v = in_cells ? c->geom_h[CELLDX][i] : 0.0;
        xf[(size_t)j * sx + i] = v;
      }
  } else {
    CB_CUDA(cudaStreamSynchronize(c->stream));
    if (c->precision == CB_FP64) {
      CB_CUDA(cudaMemcpy2D(xf.data(), sizeof(double) * sx, c->base(field), sizeof(double) * c->pitch, sizeof(double) * sx, sy,
                           cudaMemcpyDeviceToHost));
    } else {
      std::vector<float> tmp((size_t)sx * sy);
      CB_CUDA(cudaMemcpy2D(tmp.data(), sizeof(float) * sx, c->base(field), sizeof(float) * c->pitch, sizeof(float) * sx, sy,
                           cudaMemcpyDeviceToHost));
      for (size_t k = 0; k < tmp.size(); ++k) xf[k] = tmp[k];
    }
  }
  if (layout == CB_LAYOUT_XFAST) {
    std::memcpy(host, xf.data(), sizeof(double) * xf.size());
  } else {
    for (int i = 0; i < sx; ++i)
      for (int j = 0; j < sy; ++j) host[(size_t)i * sy + j] = xf[(size_t)j * sx + i];
  }
  return CB_OK;
}

int cb_write_field(cb_chunk *c, int field, const double *host, size_t n, int layout) {
  CB_CHECK_CHUNK(c);
  if (!host) return fail(CB_EINVAL, "cb_write_field: null host buffer");
  if (!is_state_field(field))
    return fail(CB_EINVAL, "cb_write_field: field " + std::to_string(field) +
                               " is derived (geometry comes from the 1-D widths, work arrays are on-chip scratch)");
  if (layout != CB_LAYOUT_XFAST && layout != CB_LAYOUT_YFAST) return fail(CB_EINVAL, "cb_write_field: bad layout");
  int sx, sy;
  field_extent(c, field, sx, sy);
  if (n != (size_t)sx * (size_t)sy)
    return fail(CB_EINVAL, "cb_write_field: buffer holds " + std::to_string(n) + " values, field has " + std::to_string((size_t)sx * sy));
  if (c->precision == CB_FP64 && layout == CB_LAYOUT_XFAST) {
    CB_CUDA(cudaMemcpy2DAsync(c->base(field), sizeof(double) * c->pitch, host, sizeof(double) * sx, sizeof(double) * sx, sy,
                              cudaMemcpyHostToDevice, c->stream));
    CB_CUDA(cudaStreamSynchronize(c->stream));
    c->halo_fresh[field] = 0;
    return CB_OK;
  }
  std::vector<double> xf((size_t)sx * sy);
  if (layout == CB_LAYOUT_XFAST) {
    std::memcpy(xf.data(), host, sizeof(double) * xf.size());
  } else {
    for (int i = 0; i < sx; ++i)
      for (int j = 0; j < sy; ++j) xf[(size_t)j * sx + i] = host[(size_t)i * sy + j];
  }
  CB_CUDA(cudaStreamSynchronize(c->stream));
  if (c->precision == CB_FP64) {
    CB_CUDA(cudaMemcpy2D(c->base(field), sizeof(double) * c->pitch, xf.data(), sizeof(double) * sx, sizeof(double) * sx, sy,
                         cudaMemcpyHostToDevice));
  } else {
    std::vector<float> tmp(xf.size());
    for (size_t k = 0; k < tmp.size(); ++k) tmp[k] = (float)xf[k];
    CB_CUDA(cudaMemcpy2D(c->base(field), sizeof(float) * c->pitch, tmp.data(), sizeof(float) * sx, sizeof(float) * sx, sy,
                         cudaMemcpyHostToDevice));
  }
  c->halo_fresh[field] = 0;
  return CB_OK;
}

int cb_read_geom(cb_chunk *c, int geom, double *host, size_t n) {
  CB_CHECK_CHUNK(c);
  if (!host) return fail(CB_EINVAL, "cb_read_geom: null host buffer");
  if (geom < 0 || geom >= NUM_GEOM) return fail(CB_EINVAL, "cb_read_geom: bad geometry id");
  if (n != (size_t)geom_len(c, geom)) return fail(CB_EINVAL, "cb_read_geom: length mismatch");
  std::memcpy(host, c->geom_h[geom], sizeof(double) * n);
  return CB_OK;
}

int cb_write_geom(cb_chunk *c, int geom, const double *host, size_t n) {
  CB_CHECK_CHUNK(c);
  if (!host) return fail(CB_EINVAL, "cb_write_geom: null host buffer");
  if (geom < 0 || geom >= NUM_GEOM) return fail(CB_EINVAL, "cb_write_geom: bad geometry id");
  if (n != (size_t)geom_len(c, geom)) return fail(CB_EINVAL, "cb_write_geom: length mismatch");
  std::memcpy(c->geom_h[geom], host, sizeof(double) * n);
  CB_CUDA(upload_geom(c));
  return CB_OK;
}

// src/serial/build_field.cpp:29-180: every array to zero.
int cb_build_field(cb_chunk *c) {
  CB_CHECK_CHUNK(c);
  const size_t bytes = c->alloc_elems * c->esize;
  for (int b = 0; b < NUM_BUF; ++b) CB_CUDA(cudaMemsetAsync(c->buf[b], 0, bytes, c->stream));
  for (int g = 0; g < NUM_GEOM; ++g) std::fill(c->geom_h[g], c->geom_h[g] + c->geom_len, 0.0);
  CB_CUDA(upload_geom(c));
  std::fill(std::begin(c->halo_fresh), std::end(c->halo_fresh), 0);
  return CB_OK;
}

// src/serial/initialise_chunk.cpp:30-85 (single tile: t_left = t_bottom = 1).
int cb_initialise_chunk(cb_chunk *c, double gxmin, double gymin, double gxmax, double gymax) {
  CB_CHECK_CHUNK(c);
  if (!(gxmax > gxmin) || !(gymax > gymin)) return fail(CB_EINVAL, "cb_initialise_chunk: empty domain");
  chunk_geometry(c->nx, c->ny, gxmin, gymin, gxmax, gymax, c->geom_h);
  CB_CUDA(upload_geom(c));
  return CB_OK;
}

int cb_initialise_chunk_in(cb_chunk *c, double gxmin, double gymin, double gxmax, double gymax, int x_cells, int y_cells, int left,
                           int bottom) {
  CB_CHECK_CHUNK(c);
  if (!(gxmax > gxmin) || !(gymax > gymin)) return fail(CB_EINVAL, "cb_initialise_chunk_in: empty domain");
  if (x_cells < 1 || y_cells < 1 || left < 1 || bottom < 1 || left - 1 + c->nx > x_cells || bottom - 1 + c->ny > y_cells)
    return fail(CB_EINVAL, "cb_initialise_chunk_in: the chunk does not lie inside the grid");
  chunk_geometry_at(c->nx, c->ny, gxmin, gymin, gxmax, gymax, x_cells, y_cells, left, bottom, c->geom_h);
  CB_CUDA(upload_geom(c));
  return CB_OK;
}

int cb_generate_chunk(cb_chunk *c, int nstates, const cb_state *states) {
  CB_CHECK_CHUNK(c);
  if (nstates < 1 || !states) return fail(CB_EINVAL, "cb_generate_chunk: need at least the background state");
  static_assert(sizeof(cb_state) == sizeof(DevState), "cb_state layout");
  DevState *d = nullptr;
  CB_CUDA(cudaMalloc(&d, sizeof(DevState) * nstates));
  cudaError_t e = cudaMemcpyAsync(d, states, sizeof(DevState) * nstates, cudaMemcpyHostToDevice, c->stream);
  if (e == cudaSuccess) e = dispatch(c, [&](auto ops) { return ops.generate_chunk(*c, d, nstates); });
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  cudaFree(d);
  if (e != cudaSuccess) return cuda_fail(e, "cb_generate_chunk");
  c->halo_fresh[DENSITY0] = c->halo_fresh[ENERGY0] = c->halo_fresh[XVEL0] = c->halo_fresh[YVEL0] = 0;
  return CB_OK;
}

int cb_ideal_gas(cb_chunk *c, int predict, int halo_depth) {
  CB_CHECK_CHUNK(c);
  if (int r = check_depth(halo_depth, true)) return r;
  const int fold = effective_fold(c, halo_depth);
  if (c->fuse_calls && !predict && fold > 0) { // held back for calc_dt's pass
    c->pend.kind = PEND_IG;
    c->pend.ig_fold = fold;
  } else {
    CB_CUDA(dispatch(c, [&](auto ops) { return ops.ideal_gas(*c, predict ? 1 : 0, fold); }));
  }
  c->halo_fresh[PRESSURE] = fold;
  c->halo_fresh[SOUNDSPEED] = 0;
  return CB_OK;
}

int cb_viscosity(cb_chunk *c, int halo_depth) {
  CB_CHECK_CHUNK_HOLD(c);
  if (int r = check_depth(halo_depth, true)) return r;
  const int fold = effective_fold(c, halo_depth);
  if (c->pend.kind == PEND_IG && fold > 0) { // held back with ideal_gas for calc_dt's pass
    c->pend.kind = PEND_IG_VISC;
    c->pend.visc_fold = fold;
  } else {
    CB_CUDA(run_pending(c));
    CB_CUDA(dispatch(c, [&](auto ops) { return ops.viscosity(*c, fold); }));
  }
  c->halo_fresh[VISCOSITY] = fold;
  return CB_OK;
}

int cb_set_dt_ahead(cb_chunk *c, double dtold, double dtrise, double dtmax) {
  CB_CHECK_CHUNK_AHEAD(c);
  if (!(dtold > 0.0) || !(dtrise > 0.0) || !(dtmax > 0.0))
    return fail(CB_EINVAL, "cb_set_dt_ahead: dtold, dtrise and dtmax must be positive");
  c->ahead.armed = true;
  c->ahead.dtold = dtold;
  c->ahead.dtrise = dtrise;
  c->ahead.dtmax = dtmax;
  return CB_OK;
}

int cb_dt_ahead_stats(const cb_chunk *c, long long *launched, long long *used) {
  if (!c) return fail(CB_EINVAL, "cb_dt_ahead_stats: null chunk");
  if (launched) *launched = c->ahead.launched_count;
  if (used) *used = c->ahead.used_count;
  return CB_OK;
}

int cb_calc_dt(cb_chunk *c, const cb_dt_params *p, double *dt_min_val, int *control, int *jldt, int *kldt, int *small) {
  CB_CHECK_CHUNK_HOLD(c);
  if (!p || !dt_min_val) return fail(CB_EINVAL, "cb_calc_dt: null argument");
  const Pending held = c->pend;
  const bool fused = held.kind == PEND_IG_VISC;
  if (!fused) CB_CUDA(run_pending(c));
  c->pend = Pending{};
  DtAhead &ah = c->ahead;
  // the Lagrangian pass goes ahead when armed, with the fused pass, on a folding chunk outside cb_run
  const bool ahead = ah.armed && fused && c->fuse_calls && c->can_fold() && !c->dt_dev;
  ah.armed = false;
  DtConsts k{p->dtc_safe, p->dtu_safe, p->dtv_safe, p->dtdiv_safe};
  c->h_scalars[0] = g_big;
  CB_CUDA(cudaMemcpyAsync(c->d_dt_bits, &c->h_scalars[0], sizeof(double), cudaMemcpyHostToDevice, c->stream));
  if (fused) // ideal_gas, viscosity and calc_dt in one pass
    CB_CUDA(dispatch(c, [&](auto ops) { return ops.ig_visc_dt(*c, k, held.ig_fold, held.visc_fold); }));
  else
    CB_CUDA(dispatch(c, [&](auto ops) { return ops.calc_dt(*c, k); }));
  CB_CUDA(cudaMemcpyAsync(&c->h_scalars[1], c->d_dt_bits, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  if (ahead) {
    // the staging-error flag comes back with the minimum; then the pass is
    // enqueued behind the read-back, with the clamped dt read on the device
    int *h_err = reinterpret_cast<int *>(&c->h_scalars[7]);
    CB_CUDA(cudaMemcpyAsync(h_err, c->d_err, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    CB_CUDA(cudaEventRecord(c->ev_dt, c->stream));
    k_dt_ahead<<<1, 1, 0, c->stream>>>(c->d_dt_bits, ah.dtold, ah.dtrise, ah.dtmax, c->d_dt_ahead);
    c->launches += 1;
    CB_CUDA(cudaGetLastError());
    const int f1 = effective_fold(c, 1), f2 = effective_fold(c, 2);
    c->dt_dev = c->d_dt_ahead;
    // the pressure the fused pass just stored is eos_value's product of density0 and energy0,
    // so the Lagrangian pass forms it from them instead of staging it (the same bits)
    const cudaError_t le = dispatch(c, [&](auto ops) { return ops.lagrange(*c, c->spare_base(4), 0.0, f1, f2, f2, f2, true, nullptr, true); });
    c->dt_dev = nullptr;
    CB_CUDA(le);
    CB_CUDA(cudaEventSynchronize(c->ev_dt));
    if (*h_err) return fail(CB_ECUDA, "cb_calc_dt: a kernel's tile staging did not complete (TMA wait limit reached)");
    ah.launched = true;
    ah.stage = 0;
    ah.dt = driver_dt_clamp(c->h_scalars[1], ah.dtold, ah.dtrise, ah.dtmax);
    ah.folds[0] = f1;
    ah.folds[1] = ah.folds[2] = ah.folds[3] = f2;
    ah.launched_count += 1;
  } else {
    CB_CUDA(cudaStreamSynchronize(c->stream));
    if (int r = check_device_error(c, "cb_calc_dt")) return r;
  }
  const double dt = c->h_scalars[1];
  *dt_min_val = dt;
  // src/serial/calc_dt.cpp:73-79: control is always "sound" (jk_control = 1.1)
  double jk_control = 1.1;
  const int l_control = (int)(10.01 * (jk_control - (int)(jk_control)));
  jk_control = jk_control - (jk_control - (int)(jk_control));
  if (control) *control = l_control;
  if (jldt) *jldt = ((int)jk_control) % c->nx;
  if (kldt) *kldt = (int)(1.f + (jk_control / c->nx));
  if (small) *small = dt < p->dtmin ? 1 : 0;
  return CB_OK;
}

int cb_pdv(cb_chunk *c, int predict, double dt, int full, int halo_depth) {
  CB_CHECK_CHUNK_AHEAD(c);
  if (int r = check_depth(halo_depth, true)) return r;
  if (full && !predict) return fail(CB_EINVAL, "cb_pdv: full = 1 is the predictor step; use predict = 1");
  const int fold = effective_fold(c, halo_depth);
  if ((full && ahead_match(c, 0, dt, fold)) || (!predict && !full && ahead_match(c, 2, dt, fold))) {
    // done by the pass run ahead
  } else if (!predict && !full && c->pend.kind == PEND_PDV1_ACC && c->pend.dt == dt && fold > 0) {
    // the corrector, held back with the predictor and accelerate for flux_calc's pass
    c->pend.kind = PEND_PDV1_ACC_PDV0;
    c->pend.pdv0_fold = fold;
  } else {
    CB_CUDA(run_pending(c));
    if (full && c->fuse_calls && fold > 0) { // the predictor, held back for the Lagrangian pass
      c->pend.kind = PEND_PDV1;
      c->pend.dt = dt;
      c->pend.pdv1_fold = fold;
    } else {
      CB_CUDA(dispatch(c, [&](auto ops) { return ops.pdv(*c, predict ? 1 : 0, dt, full ? 1 : 0, fold); }));
    }
  }
  if (full && halo_depth > 0 && fold == 0) {
    // the predictor's own update_halo(pressure) (src/serial/PdV.cpp:118-124) on a mesh too small to fold
    HaloJob job{};
    job.nfields = 1;
    job.field[0] = PRESSURE;
    CB_CUDA(dispatch(c, [&](auto ops) { return ops.update_halo(*c, job, halo_depth); }));
  }
  if (full) {
    c->halo_fresh[PRESSURE] = fold;
    c->halo_fresh[SOUNDSPEED] = 0;
    c->halo_fresh[DENSITY1] = c->halo_fresh[ENERGY1] = 0;
  } else {
    c->halo_fresh[DENSITY1] = c->halo_fresh[ENERGY1] = fold;
  }
  return CB_OK;
}

int cb_revert(cb_chunk *c) {
  CB_CHECK_CHUNK(c);
  CB_CUDA(dispatch(c, [&](auto ops) { return ops.revert(*c); }));
  c->halo_fresh[DENSITY1] = c->halo_fresh[ENERGY1] = 0;
  return CB_OK;
}

int cb_accelerate(cb_chunk *c, double dt, int halo_depth) {
  CB_CHECK_CHUNK_AHEAD(c);
  if (int r = check_depth(halo_depth, true)) return r;
  const int fold = effective_fold(c, halo_depth);
  if (ahead_match(c, 1, dt, fold)) {
    // done by the pass run ahead
  } else if (c->pend.kind == PEND_PDV1 && c->pend.dt == dt && fold > 0) { // held back with the predictor
    c->pend.kind = PEND_PDV1_ACC;
    c->pend.acc_fold = fold;
  } else {
    CB_CUDA(run_pending(c));
    CB_CUDA(dispatch(c, [&](auto ops) { return ops.accelerate(*c, dt, fold); }));
  }
  c->halo_fresh[XVEL1] = c->halo_fresh[YVEL1] = fold;
  return CB_OK;
}

int cb_flux_calc(cb_chunk *c, double dt, int halo_depth) {
  CB_CHECK_CHUNK_AHEAD(c);
  if (int r = check_depth(halo_depth, true)) return r;
  const int fold = effective_fold(c, halo_depth);
  const Pending held = c->pend;
  if (ahead_match(c, 3, dt, fold)) { // the pass run ahead is complete: its predicted pressure went to the spare
    c->ahead.launched = false;
    c->ahead.stage = 0;
    c->ahead.used_count += 1;
    std::swap(c->fbuf[PRESSURE], c->sbuf[4]);
  } else if (held.kind == PEND_PDV1_ACC_PDV0 && held.dt == dt && fold > 0) {
    // the predictor, accelerate, the corrector and flux_calc as one pass (cb_lagrangian's)
    c->pend = Pending{};
    CB_CUDA(dispatch(c, [&](auto ops) {
      return ops.lagrange(*c, c->spare_base(4), dt, held.pdv1_fold, held.acc_fold, held.pdv0_fold, fold, true);
    }));
    std::swap(c->fbuf[PRESSURE], c->sbuf[4]); // the predicted pressure went to the spare
  } else {
    CB_CUDA(run_pending(c));
    CB_CUDA(dispatch(c, [&](auto ops) { return ops.flux_calc(*c, dt, fold); }));
  }
  c->halo_fresh[VOL_FLUX_X] = c->halo_fresh[VOL_FLUX_Y] = fold;
  return CB_OK;
}

int cb_lagrangian(cb_chunk *c, double dt, int halo_depth) {
  CB_CHECK_CHUNK(c);
  if (int r = check_depth(halo_depth, true)) return r;
  const int fold = effective_fold(c, halo_depth);
  if (fold == 0) { // nothing folds: the four phases as their own passes
    if (int r = cb_pdv(c, 1, dt, 1, 1)) return r;
    if (int r = cb_accelerate(c, dt, halo_depth)) return r;
    if (int r = cb_pdv(c, 0, dt, 0, halo_depth)) return r;
    return cb_flux_calc(c, dt, halo_depth);
  }
  CB_CUDA(dispatch(c, [&](auto ops) { return ops.lagrange(*c, c->spare_base(4), dt, 1, fold, fold, fold, true); }));
  std::swap(c->fbuf[PRESSURE], c->sbuf[4]); // the predicted pressure went to the spare
  c->halo_fresh[PRESSURE] = 1;
  c->halo_fresh[SOUNDSPEED] = 0;
  c->halo_fresh[XVEL1] = c->halo_fresh[YVEL1] = fold;
  c->halo_fresh[DENSITY1] = c->halo_fresh[ENERGY1] = fold;
  c->halo_fresh[VOL_FLUX_X] = c->halo_fresh[VOL_FLUX_Y] = fold;
  return CB_OK;
}

int cb_advec_cell(cb_chunk *c, int sweep_number, int direction, int halo_depth) {
  CB_CHECK_CHUNK(c);
  if (sweep_number != 1 && sweep_number != 2) return fail(CB_EINVAL, "cb_advec_cell: sweep_number must be 1 or 2");
  if (direction != 1 && direction != 2) return fail(CB_EINVAL, "cb_advec_cell: direction must be 1 (x) or 2 (y)");
  if (int r = check_depth(halo_depth, true)) return r;
  const int fold = effective_fold(c, halo_depth);
  if (c->fuse_calls && fold == 2 && (sweep_number == 2 || (direction == 1 && x_fusable(c)))) {
    // held back for its momentum sweep or reset_field (the buffers swap when it runs)
    c->pend.kind = PEND_CELL;
    c->pend.cell_sweep = sweep_number;
    c->pend.cell_dir = direction;
    c->pend.cell_fold = fold;
  } else {
    CB_CUDA(launch_cell(c, sweep_number, direction, fold, -1));
  }
  c->halo_fresh[DENSITY1] = c->halo_fresh[ENERGY1] = fold;
  c->halo_fresh[direction == 1 ? MASS_FLUX_X : MASS_FLUX_Y] = fold;
  return CB_OK;
}

int cb_advec_mom(cb_chunk *c, int which_vel, int sweep_number, int direction, int halo_depth) {
  CB_CHECK_CHUNK_HOLD(c);
  if (which_vel < 1 || which_vel > 3) return fail(CB_EINVAL, "cb_advec_mom: which_vel must be 1, 2 or 3");
  if (sweep_number != 1 && sweep_number != 2) return fail(CB_EINVAL, "cb_advec_mom: sweep_number must be 1 or 2");
  if (direction != 1 && direction != 2) return fail(CB_EINVAL, "cb_advec_mom: direction must be 1 (x) or 2 (y)");
  if (int r = check_depth(halo_depth, true)) return r;
  const int fold = effective_fold(c, halo_depth);
  const Pending held = c->pend;
  if (held.kind == PEND_CELL && held.cell_sweep == sweep_number && held.cell_dir == direction && which_vel == 3) {
    if (sweep_number == 2) { // held back with the cell sweep for reset_field
      c->pend.kind = PEND_CELL_MOM;
      c->pend.mom_fold = fold;
      c->pend.mom_mask = which_vel;
    } else { // a first x sweep: cell and momentum parts as one pass
      c->pend = Pending{};
      CB_CUDA(launch_sweep_x(c, 1, held.cell_fold, fold, -1));
    }
  } else {
    CB_CUDA(run_pending(c));
    CB_CUDA(launch_mom(c, which_vel, sweep_number, direction, fold, -1));
  }
  if (which_vel & 1) c->halo_fresh[XVEL1] = fold;
  if (which_vel & 2) c->halo_fresh[YVEL1] = fold;
  return CB_OK;
}

int cb_reset_field(cb_chunk *c, int halo_depth) {
  CB_CHECK_CHUNK_HOLD(c);
  if (int r = check_depth(halo_depth, true)) return r;
  const int fold = effective_fold(c, halo_depth);
  const Pending held = c->pend;
  if (held.kind == PEND_CELL_MOM) { // the second sweeps, each with reset_field's copy of what it writes
    c->pend = Pending{};
    if (held.cell_dir == 1 && x_fusable(c)) {
      CB_CUDA(launch_sweep_x(c, 2, held.cell_fold, held.mom_fold, fold));
    } else {
      CB_CUDA(launch_cell(c, 2, held.cell_dir, held.cell_fold, fold));
      CB_CUDA(launch_mom(c, held.mom_mask, 2, held.cell_dir, held.mom_fold, fold));
    }
  } else {
    CB_CUDA(run_pending(c));
    CB_CUDA(dispatch(c, [&](auto ops) { return ops.reset_field(*c, fold); }));
  }
  c->halo_fresh[DENSITY0] = c->halo_fresh[ENERGY0] = c->halo_fresh[XVEL0] = c->halo_fresh[YVEL0] = fold;
  return CB_OK;
}

int cb_update_halo(cb_chunk *c, const int fields[15], int depth) {
  CB_CHECK_CHUNK_HOLD(c); // a pass with nothing to do leaves held-back calls held back
  if (!fields) return fail(CB_EINVAL, "cb_update_halo: null field list");
  if (int r = check_depth(depth, false)) return r;
  HaloJob job{};
  for (int f = 0; f < 15; ++f) {
    if (fields[f] != 1) continue;
    if (c->can_fold() && c->halo_fresh[f] >= depth) continue; // a folded producer already wrote it
    job.field[job.nfields++] = f;
  }
  if (job.nfields) CB_CUDA(run_pending(c));
  CB_CUDA(dispatch(c, [&](auto ops) { return ops.update_halo(*c, job, depth); }));
  for (int k = 0; k < job.nfields; ++k) c->halo_fresh[job.field[k]] = std::max(c->halo_fresh[job.field[k]], depth);
  return CB_OK;
}

int cb_set_external_faces(cb_chunk *c, int faces) {
  CB_CHECK_CHUNK(c);
  if (faces < 0 || faces > 15) return fail(CB_EINVAL, "cb_set_external_faces: faces must be a mask of CB_FACE_* bits (0..15)");
  c->external_faces = faces;
  std::fill(std::begin(c->halo_fresh), std::end(c->halo_fresh), 0); // what the producers folded no longer applies
  return CB_OK;
}

int cb_copy_tile_halo(cb_chunk *dst, cb_chunk *src, int side, const int fields[15], int depth) {
  CB_CHECK_CHUNK(dst);
  if (!src || !fields) return fail(CB_EINVAL, "cb_copy_tile_halo: null argument");
  if (src == dst) return fail(CB_EINVAL, "cb_copy_tile_halo: a tile is not its own neighbour");
  if (src->device != dst->device || src->precision != dst->precision)
    return fail(CB_EINVAL, "cb_copy_tile_halo: the tiles must share a device and a precision");
  if (side != CB_FACE_LEFT && side != CB_FACE_RIGHT && side != CB_FACE_BOTTOM && side != CB_FACE_TOP)
    return fail(CB_EINVAL, "cb_copy_tile_halo: side must be one CB_FACE_* value");
  if (int r = check_depth(depth, false)) return r;
  const bool lr = side == CB_FACE_LEFT || side == CB_FACE_RIGHT;
  if (lr ? src->ny != dst->ny : src->nx != dst->nx)
    return fail(CB_EINVAL, "cb_copy_tile_halo: neighbouring tiles must share their extent along the common face");
  CB_CUDA(run_pending(src));
  HaloJob job{};
  for (int f = 0; f < 15; ++f)
    if (fields[f] == 1) job.field[job.nfields++] = f;
  if (job.nfields == 0) return CB_OK;
  // the copy comes after src's work so far and before its later work (each chunk has its own stream)
  CB_CUDA(cudaEventRecord(src->ev_order, src->stream));
  CB_CUDA(cudaStreamWaitEvent(dst->stream, src->ev_order, 0));
  CB_CUDA(dispatch(dst, [&](auto ops) { return ops.tile_halo(*dst, *src, side, job, depth); }));
  CB_CUDA(cudaEventRecord(dst->ev_order, dst->stream));
  CB_CUDA(cudaStreamWaitEvent(src->stream, dst->ev_order, 0));
  for (int k = 0; k < job.nfields; ++k) dst->halo_fresh[job.field[k]] = 0;
  return CB_OK;
}

namespace {

// The job of one face strip and its length in elements; CB_OK or an error.
int strip_job(const char *who, cb_chunk *c, int side, const int fields[15], int depth, StripJob &job, size_t &elements) {
  if (!fields) return fail(CB_EINVAL, std::string(who) + ": null fields");
  if (side != CB_FACE_LEFT && side != CB_FACE_RIGHT && side != CB_FACE_BOTTOM && side != CB_FACE_TOP)
    return fail(CB_EINVAL, std::string(who) + ": side must be one CB_FACE_* value");
  if (int r = check_depth(depth, false)) return r;
  const bool lr = side == CB_FACE_LEFT || side == CB_FACE_RIGHT;
  job = StripJob{};
  long long n = 0;
  for (int f = 0; f < 15; ++f) {
    if (fields[f] != 1) continue;
    // the arrays one longer in x (nodes, x faces) or in y (nodes, y faces): driver/definitions.cpp:4-41
    const bool node = f == XVEL0 || f == XVEL1 || f == YVEL0 || f == YVEL1;
    const int xe = node || f == VOL_FLUX_X || f == MASS_FLUX_X, ye = node || f == VOL_FLUX_Y || f == MASS_FLUX_Y;
    const int along_extra = lr ? ye : xe;
    job.field[job.nfields] = f;
    job.off[job.nfields] = n;
    ++job.nfields;
    n += (long long)((lr ? c->ny : c->nx) + 2 * depth + along_extra) * depth;
  }
  elements = (size_t)n;
  return CB_OK;
}

} // namespace

int cb_face_strip_size(cb_chunk *c, int side, const int fields[15], int depth, size_t *elements) {
  CB_CHECK_CHUNK(c);
  if (!elements) return fail(CB_EINVAL, "cb_face_strip_size: null elements");
  StripJob job;
  return strip_job("cb_face_strip_size", c, side, fields, depth, job, *elements);
}

int cb_pack_face(cb_chunk *c, int side, const int fields[15], int depth, void *dev_buf, size_t capacity) {
  CB_CHECK_CHUNK(c);
  StripJob job;
  size_t n = 0;
  if (int r = strip_job("cb_pack_face", c, side, fields, depth, job, n)) return r;
  if (n > 0 && !dev_buf) return fail(CB_EINVAL, "cb_pack_face: null buffer");
  if (capacity < n) return fail(CB_EINVAL, "cb_pack_face: buffer of " + std::to_string(capacity) + " elements, strip needs " + std::to_string(n));
  CB_CUDA(run_pending(c));
  CB_CUDA(dispatch(c, [&](auto ops) { return ops.face_strip(*c, side, job, depth, dev_buf, true); }));
  return CB_OK;
}

int cb_unpack_face(cb_chunk *c, int side, const int fields[15], int depth, const void *dev_buf, size_t capacity) {
  CB_CHECK_CHUNK(c);
  StripJob job;
  size_t n = 0;
  if (int r = strip_job("cb_unpack_face", c, side, fields, depth, job, n)) return r;
  if (n > 0 && !dev_buf) return fail(CB_EINVAL, "cb_unpack_face: null buffer");
  if (capacity < n) return fail(CB_EINVAL, "cb_unpack_face: buffer of " + std::to_string(capacity) + " elements, strip needs " + std::to_string(n));
  CB_CUDA(run_pending(c));
  CB_CUDA(dispatch(c, [&](auto ops) { return ops.face_strip(*c, side, job, depth, const_cast<void *>(dev_buf), false); }));
  for (int k = 0; k < job.nfields; ++k) c->halo_fresh[job.field[k]] = 0;
  return CB_OK;
}

int cb_field_summary(cb_chunk *c, double out[5]) {
  CB_CHECK_CHUNK(c);
  if (!out) return fail(CB_EINVAL, "cb_field_summary: null out");
  CB_CUDA(dispatch(c, [&](auto ops) { return ops.field_summary(*c); }));
  CB_CUDA(cudaMemcpyAsync(&c->h_scalars[2], c->d_sums, sizeof(double) * 5, cudaMemcpyDeviceToHost, c->stream));
  CB_CUDA(cudaStreamSynchronize(c->stream));
  if (int r = check_device_error(c, "cb_field_summary")) return r;
  for (int q = 0; q < 5; ++q) out[q] = c->h_scalars[2 + q];
  c->halo_fresh[PRESSURE] = 0;
  c->halo_fresh[SOUNDSPEED] = 0;
  return CB_OK;
}

int cb_synchronize(cb_chunk *c) {
  CB_CHECK_CHUNK(c);
  CB_CUDA(cudaStreamSynchronize(c->stream));
  return check_device_error(c, "cb_synchronize");
}

int cb_get_stream(cb_chunk *c, void **stream) {
  if (!c || !stream) return fail(CB_EINVAL, "cb_get_stream: null argument");
  *stream = (void *)c->stream;
  return CB_OK;
}

int cb_launch_count(const cb_chunk *c, long long *count) {
  if (!c || !count) return fail(CB_EINVAL, "cb_launch_count: null argument");
  *count = c->launches;
  return CB_OK;
}

} // extern "C"
