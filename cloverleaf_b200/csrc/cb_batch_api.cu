// cb_batch_api.cu -- the batched-ensemble part of the C ABI (cb_batch_* in
// include/cloverb200.h): allocation of many decks in one pool, their
// geometry and tensor maps, the lane schedule of the persistent launch, its
// CUDA graph, the autotuner, and read-back of each deck's results.
//
// Host code only; the kernel is kb_ensemble (cb_batch_impl.cuh), compiled
// into the FP64 and FP32 translation units.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <new>
#include <numeric>
#include <queue>
#include <string>
#include <vector>

#include "../../include/cloverb200.h"
#include "cb_batch.h"

namespace cb {
int set_last_error(int code, const std::string &msg);
bool encode_buffer_maps(void *const *bufs, int nbuf, long long pitch, int ny, int precision, CUtensorMap (*maps)[NUM_BOX_H],
                        std::string *err);
void chunk_geometry(int nx, int ny, double gxmin, double gymin, double gxmax, double gymax, double *const *g);
} // namespace cb

using namespace cb;

struct cb_batch {
  int n = 0;
  int precision = CB_FP64;
  int device = 0;
  int sms = 148;
  size_t esize = 8;
  std::vector<cb_deck> decks;
  std::vector<BatchDeck> desc;      // host copy of the descriptors (reset value of every run)
  std::vector<double> work;         // estimated cells x steps of each deck
  void *pool = nullptr;             // fields of every deck
  double *geom = nullptr;           // FP64 geometry of every deck
  double *rgeom = nullptr;          // reciprocal widths of every deck
  void *geom_t = nullptr;           // geometry in the storage type (FP32 form)
  CUtensorMap *maps = nullptr;      // [deck][BATCH_BUF][NUM_BOX_H]
  double *records = nullptr;        // summaries, dt traces, partials
  unsigned long long *slots = nullptr;
  BatchDeck *d_desc = nullptr;
  BatchDeck *h_desc = nullptr;      // pinned copy the graph uploads
  // launch layout
  cb_batch_schedule sched{};
  int grid = 0, nlanes = 0, nlevels = 0; // lanes over all widths
  size_t sync_words = 0;
  int *d_plan = nullptr;            // queue | level
  unsigned *d_sync = nullptr;       // lane_sync | lane_deck | next
  int *d_flags = nullptr;           // [0] abort, [1] staging error
  cudaStream_t stream = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  bool use_graph = true;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  bool ran = false, results_ok = false;
  long long launches = 0;
};

namespace {

int fail(int code, const std::string &m) { return set_last_error(code, m); }
int cuda_fail(cudaError_t e, const char *where) {
  return fail(CB_ECUDA, std::string(where) + ": " + cudaGetErrorName(e) + ": " + cudaGetErrorString(e));
}

#define BCUDA(expr)                                                                                                                          \
  do {                                                                                                                                       \
    cudaError_t _e = (expr);                                                                                                                 \
    if (_e != cudaSuccess) return cuda_fail(_e, __func__);                                                                                   \
  } while (0)

size_t round_up(size_t v, size_t a) { return (v + a - 1) / a * a; }

int next_pow2(long long v) {
  int p = 1;
  while (p < v && p < (1 << 20)) p <<= 1;
  return p;
}

// Steps a deck is expected to take: its end time over the dt the sound-speed
// (CFL) limit allows in its hottest state, capped by dtmax and end_step.
double estimate_steps(const cb_deck &d) {
  const double dx = (d.xmax - d.xmin) / d.nx, dy = (d.ymax - d.ymin) / d.ny;
  double cmax = 1e-12;
  for (int s = 0; s < d.nstates; ++s) {
    const double e = std::max(d.states[s].energy, 0.0);
    const double c = std::sqrt(d.gamma * (d.gamma - 1.0) * e) + std::fabs(d.states[s].xvel) + std::fabs(d.states[s].yvel);
    cmax = std::max(cmax, c);
  }
  const double dt = std::min(d.dtmax, d.dtc_safe * std::min(dx, dy) / cmax);
  double steps = d.end_time / std::max(dt, 1e-300) + 1.0;
  return std::min(steps, (double)d.end_step);
}

cudaError_t select_device(const cb_batch *b) {
  int cur = -1;
  cudaError_t e = cudaGetDevice(&cur);
  if (e != cudaSuccess) return e;
  return cur == b->device ? cudaSuccess : cudaSetDevice(b->device);
}

cudaError_t occupancy(const cb_batch *b, int variant, int *per_sm) {
  return b->precision == CB_FP64 ? BatchOps<double>::occupancy(variant, per_sm) : BatchOps<float>::occupancy(variant, per_sm);
}

// The deck queues of schedule s.  A deck of c cells gets w CTAs, w the power
// of two >= c / cells_per_cta (at most max_lane_width, its tile count and the
// grid, rounded down to a power of two); one queue per width, widest first,
// each largest estimated run (cells x steps) first.  The grid is every
// resident CTA; at width W it forms grid / W lanes, each with a lane slot
// (barrier counter, deck taken).
struct Plan {
  std::vector<int> queue, level; // level: width | first queue position | decks | first lane slot
  int ctas = 0, lanes = 0;
};

int tiles_of(const cb_deck &d) { return ((d.nx + 63) / 64) * ((d.ny + 15) / 16); }

int pow2_floor(int v) {
  int p = 1;
  while (p * 2 <= v) p *= 2;
  return p;
}

Plan make_plan(const cb_batch *b, const cb_batch_schedule &s, int grid_max) {
  const int maxw = std::max(1, std::min(s.max_lane_width > 0 ? s.max_lane_width : BATCH_MAX_LANE, BATCH_MAX_LANE));
  std::vector<int> w(b->n);
  for (int d = 0; d < b->n; ++d) {
    const long long cells = (long long)b->decks[d].nx * b->decks[d].ny;
    int wd = s.cells_per_cta > 0 ? next_pow2((cells + s.cells_per_cta - 1) / s.cells_per_cta) : 1;
    wd = std::min(wd, pow2_floor(maxw));
    while (wd > 1 && wd > tiles_of(b->decks[d])) wd >>= 1;
    w[d] = std::min(wd, pow2_floor(grid_max));
  }
  std::vector<int> widths(w);
  std::sort(widths.begin(), widths.end(), std::greater<int>());
  widths.erase(std::unique(widths.begin(), widths.end()), widths.end());
  Plan p;
  p.ctas = grid_max;
  for (int W : widths) {
    const int q0 = (int)p.queue.size();
    for (int d = 0; d < b->n; ++d)
      if (w[d] == W) p.queue.push_back(d);
    std::stable_sort(p.queue.begin() + q0, p.queue.end(), [&](int x, int y) { return b->work[x] > b->work[y]; });
    p.level.insert(p.level.end(), {W, q0, (int)p.queue.size() - q0, p.lanes});
    p.lanes += grid_max / W;
  }
  return p;
}

void release(cb_batch *b) {
  if (b->exec) cudaGraphExecDestroy(b->exec);
  if (b->graph) cudaGraphDestroy(b->graph);
  b->exec = nullptr;
  b->graph = nullptr;
  for (void *p : {(void *)b->pool, (void *)b->geom, (void *)b->rgeom, b->geom_t, (void *)b->maps, (void *)b->records, (void *)b->slots, (void *)b->d_desc,
                  (void *)b->d_plan, (void *)b->d_sync, (void *)b->d_flags})
    if (p) cudaFree(p);
  if (b->h_desc) cudaFreeHost(b->h_desc);
  if (b->ev0) cudaEventDestroy(b->ev0);
  if (b->ev1) cudaEventDestroy(b->ev1);
  if (b->stream) cudaStreamDestroy(b->stream);
  b->pool = nullptr;
  b->geom = nullptr;
  b->rgeom = nullptr;
  b->geom_t = nullptr;
  b->maps = nullptr;
  b->records = nullptr;
  b->slots = nullptr;
  b->d_desc = nullptr;
  b->d_plan = nullptr;
  b->d_sync = nullptr;
  b->d_flags = nullptr;
  b->h_desc = nullptr;
  b->ev0 = b->ev1 = nullptr;
  b->stream = nullptr;
}

int check_deck(const cb_deck &d, int k) {
  const std::string w = "cb_batch_create: deck " + std::to_string(k) + ": ";
  if (d.nx < 8 || d.ny < 8) return fail(CB_EINVAL, w + "mesh must have at least 8 cells per direction");
  if (d.nx > 16384 || d.ny > 16384) return fail(CB_EINVAL, w + "mesh side above 16384 cells");
  if (!(d.xmax > d.xmin) || !(d.ymax > d.ymin)) return fail(CB_EINVAL, w + "empty domain");
  if (!(d.gamma > 1.0) || !std::isfinite(d.gamma)) return fail(CB_EINVAL, w + "gamma must be a finite value above 1");
  if (d.nstates < 1 || d.nstates > CB_DECK_MAX_STATES) return fail(CB_EINVAL, w + "needs 1 to 8 states");
  if (!(d.dtinit > 0.0) || !(d.dtmax > 0.0) || !(d.dtrise > 0.0)) return fail(CB_EINVAL, w + "dtinit, dtmax and dtrise must be positive");
  if (d.end_step < 1 && !(d.end_time > 0.0)) return fail(CB_EINVAL, w + "needs an end time or an end step");
  if (d.summary_frequency < 0) return fail(CB_EINVAL, w + "summary_frequency must not be negative");
  return CB_OK;
}

// Enqueues one run: descriptors reset, barrier counters and flags cleared,
// the persistent launch.  Captured once into the batch's graph.
cudaError_t enqueue_run(cb_batch *b) {
  cudaError_t e;
  if ((e = cudaMemcpyAsync(b->d_desc, b->h_desc, sizeof(BatchDeck) * b->n, cudaMemcpyHostToDevice, b->stream)) != cudaSuccess) return e;
  if ((e = cudaMemsetAsync(b->d_sync, 0, sizeof(unsigned) * b->sync_words, b->stream)) != cudaSuccess) return e;
  if ((e = cudaMemsetAsync(b->d_flags, 0, sizeof(int) * 2, b->stream)) != cudaSuccess) return e;
  BatchLaunch a{};
  a.decks = b->d_desc;
  a.queue = b->d_plan;
  a.level = a.queue + b->n;
  a.nlevels = b->nlevels;
  a.lane_sync = b->d_sync;
  a.lane_deck = reinterpret_cast<int *>(b->d_sync + b->nlanes);
  a.next = b->d_sync + 2 * b->nlanes;
  a.abort = b->d_flags;
  a.err = b->d_flags + 1;
  const int v = b->sched.variant;
  return b->precision == CB_FP64 ? BatchOps<double>::launch(v, a, b->grid, b->stream) : BatchOps<float>::launch(v, a, b->grid, b->stream);
}

} // namespace

extern "C" {

int cb_batch_create(int ndecks, const cb_deck *decks, int precision, int device, cb_batch **out) {
  if (!out) return fail(CB_EINVAL, "cb_batch_create: null out");
  *out = nullptr;
  if (ndecks < 1 || !decks) return fail(CB_EINVAL, "cb_batch_create: need at least one deck");
  if (precision != CB_FP64 && precision != CB_FP32) return fail(CB_EINVAL, "cb_batch_create: precision must be CB_FP64 or CB_FP32");
  for (int k = 0; k < ndecks; ++k)
    if (int r = check_deck(decks[k], k)) return r;
  int ndev = 0;
  cudaError_t e = cudaGetDeviceCount(&ndev);
  if (e != cudaSuccess) return cuda_fail(e, "cb_batch_create");
  if (device < 0 || device >= ndev) return fail(CB_EINVAL, "cb_batch_create: no CUDA device " + std::to_string(device));
  if ((e = cudaSetDevice(device)) != cudaSuccess) return cuda_fail(e, "cb_batch_create");
  cb_batch *b = new (std::nothrow) cb_batch();
  if (!b) return fail(CB_ENOMEM, "cb_batch_create: out of host memory");
  b->n = ndecks;
  b->precision = precision;
  b->device = device;
  b->esize = precision == CB_FP64 ? 8 : 4;
  b->decks.assign(decks, decks + ndecks);
  b->desc.resize(ndecks);
  b->work.resize(ndecks);
  cudaDeviceGetAttribute(&b->sms, cudaDevAttrMultiProcessorCount, device);
  auto bail = [&](cudaError_t err, const char *what) {
    release(b);
    delete b;
    if (err == cudaErrorMemoryAllocation) return fail(CB_ENOMEM, std::string("cb_batch_create: out of device memory allocating ") + what);
    return cuda_fail(err, "cb_batch_create");
  };
  // layouts (cb_create's: element (i, j) at buffer + off + j * pitch + i)
  const long long align = 256 / (long long)b->esize;
  std::vector<size_t> pool_off(ndecks), geom_off(ndecks), rec_off(ndecks);
  size_t pool_bytes = 0, geom_elems = 0, rec_elems = 0;
  for (int k = 0; k < ndecks; ++k) {
    const cb_deck &d = decks[k];
    BatchDeck &D = b->desc[k];
    std::memset(&D, 0, sizeof(D));
    D.nx = d.nx;
    D.ny = d.ny;
    D.off = (int)(align - 2);
    D.pitch = (int)((D.off + d.nx + 5 + align - 1) / align * align);
    const size_t elems = (size_t)D.off + (size_t)D.pitch * (size_t)(d.ny + 6) + (size_t)align;
    D.buf_bytes = round_up(elems * b->esize, 256);
    pool_off[k] = pool_bytes;
    pool_bytes += D.buf_bytes * BATCH_BUF;
    geom_off[k] = geom_elems;
    geom_elems += (size_t)NUM_GEOM * (std::max(d.nx, d.ny) + 6);
    b->work[k] = estimate_steps(d) * (double)d.nx * d.ny;
    D.max_steps = (int)std::min<double>(d.end_step, 4.0 * estimate_steps(d) + 1000.0);
    D.max_summaries = (d.summary_frequency > 0 ? D.max_steps / d.summary_frequency : 0) + 3;
    rec_off[k] = rec_elems;
    rec_elems += (size_t)D.max_summaries * BATCH_RECORD + (size_t)D.max_steps + 5 * BATCH_MAX_LANE;
  }
  if ((e = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking)) != cudaSuccess) return bail(e, "stream");
  if ((e = cudaEventCreate(&b->ev0)) != cudaSuccess || (e = cudaEventCreate(&b->ev1)) != cudaSuccess) return bail(e, "events");
  if ((e = cudaMalloc(&b->pool, pool_bytes)) != cudaSuccess) return bail(e, "fields");
  if ((e = cudaMalloc(&b->geom, geom_elems * sizeof(double))) != cudaSuccess) return bail(e, "geometry");
  if ((e = cudaMalloc(&b->rgeom, geom_elems / 2 * sizeof(double))) != cudaSuccess) return bail(e, "geometry");
  if (precision == CB_FP32 && (e = cudaMalloc(&b->geom_t, geom_elems * sizeof(float))) != cudaSuccess) return bail(e, "geometry");
  if ((e = cudaMalloc(&b->maps, sizeof(CUtensorMap) * BATCH_BUF * NUM_BOX_H * ndecks)) != cudaSuccess) return bail(e, "tensor maps");
  if ((e = cudaMalloc(&b->records, sizeof(double) * rec_elems)) != cudaSuccess) return bail(e, "records");
  if ((e = cudaMalloc(&b->slots, sizeof(unsigned long long) * 4 * ndecks)) != cudaSuccess) return bail(e, "scratch");
  if ((e = cudaMalloc(&b->d_desc, sizeof(BatchDeck) * ndecks)) != cudaSuccess) return bail(e, "descriptors");
  if ((e = cudaMallocHost(&b->h_desc, sizeof(BatchDeck) * ndecks)) != cudaSuccess) return bail(e, "descriptors");
  if ((e = cudaMalloc(&b->d_flags, sizeof(int) * 2)) != cudaSuccess) return bail(e, "scratch");
  std::vector<double> gh(geom_elems, 0.0), rh(geom_elems / 2, 0.0);
  std::vector<CUtensorMap> maps((size_t)BATCH_BUF * NUM_BOX_H * ndecks);
  for (int k = 0; k < ndecks; ++k) {
    const cb_deck &d = decks[k];
    BatchDeck &D = b->desc[k];
    const int glen = std::max(d.nx, d.ny) + 6;
    for (int bb = 0; bb < BATCH_BUF; ++bb) D.buf[bb] = (char *)b->pool + pool_off[k] + (size_t)bb * D.buf_bytes;
    double *g[NUM_GEOM];
    for (int q = 0; q < NUM_GEOM; ++q) {
      g[q] = gh.data() + geom_off[k] + (size_t)q * glen;
      D.geom_d[q] = b->geom + geom_off[k] + (size_t)q * glen;
      D.geom_t[q] = precision == CB_FP64 ? (const void *)D.geom_d[q] : (const void *)((float *)b->geom_t + geom_off[k] + (size_t)q * glen);
    }
    chunk_geometry(d.nx, d.ny, d.xmin, d.ymin, d.xmax, d.ymax, g);
    // reciprocals of the widths, rounded to nearest (the divisors of width_ratio)
    const int rsrc[4] = {CELLDX, CELLDY, VERTEXDX, VERTEXDY};
    double *rk = rh.data() + geom_off[k] / 2;
    for (int q = 0; q < 4; ++q)
      for (int x = 0; x < glen; ++x) rk[(size_t)q * glen + x] = g[rsrc[q]][x] != 0.0 ? 1.0 / g[rsrc[q]][x] : 0.0;
    D.rgeom = b->rgeom + geom_off[k] / 2;
    D.geom_len = glen;
    std::string err;
    if (!encode_buffer_maps(D.buf, BATCH_BUF, D.pitch, d.ny, precision,
                            reinterpret_cast<CUtensorMap(*)[NUM_BOX_H]>(&maps[(size_t)k * BATCH_BUF * NUM_BOX_H]), &err)) {
      release(b);
      delete b;
      return fail(CB_ECUDA, "cb_batch_create: " + err);
    }
    D.maps = b->maps + (size_t)k * BATCH_BUF * NUM_BOX_H;
    D.gm1 = d.gamma - 1.0;
    D.nstates = d.nstates;
    for (int s = 0; s < d.nstates; ++s) {
      const cb_state &st = d.states[s];
      D.states[s] = DevState{st.density, st.energy, st.xvel, st.yvel, st.geometry, st.xmin, st.ymin, st.xmax, st.ymax, st.radius};
    }
    D.dtinit = d.dtinit;
    D.dtmin = d.dtmin;
    D.dtmax = d.dtmax;
    D.dtrise = d.dtrise;
    D.end_time = d.end_time;
    D.end_step = d.end_step;
    D.summary_frequency = d.summary_frequency;
    D.k = DtConsts{d.dtc_safe, d.dtu_safe, d.dtv_safe, d.dtdiv_safe};
    D.summaries = b->records + rec_off[k];
    D.dt_trace = D.summaries + (size_t)D.max_summaries * BATCH_RECORD;
    D.partials = D.dt_trace + D.max_steps;
    D.dt_slots = b->slots + 4 * (size_t)k;
  }
  if ((e = cudaMemcpy(b->geom, gh.data(), sizeof(double) * geom_elems, cudaMemcpyHostToDevice)) != cudaSuccess) return bail(e, "geometry");
  if ((e = cudaMemcpy(b->rgeom, rh.data(), sizeof(double) * rh.size(), cudaMemcpyHostToDevice)) != cudaSuccess) return bail(e, "geometry");
  if (precision == CB_FP32) {
    std::vector<float> gf(gh.begin(), gh.end());
    if ((e = cudaMemcpy(b->geom_t, gf.data(), sizeof(float) * geom_elems, cudaMemcpyHostToDevice)) != cudaSuccess) return bail(e, "geometry");
  }
  if ((e = cudaMemcpy(b->maps, maps.data(), sizeof(CUtensorMap) * maps.size(), cudaMemcpyHostToDevice)) != cudaSuccess)
    return bail(e, "tensor maps");
  std::memcpy(b->h_desc, b->desc.data(), sizeof(BatchDeck) * ndecks);
  cb_batch_schedule s{16384, 16, 0, 0};
  if (int r = cb_batch_set_schedule(b, &s)) {
    const std::string msg = "cb_batch_create: " + std::string(cb_last_error());
    release(b);
    delete b;
    return fail(r, msg);
  }
  *out = b;
  return CB_OK;
}

int cb_batch_destroy(cb_batch *b) {
  if (!b) return CB_OK;
  select_device(b);
  if (b->stream) cudaStreamSynchronize(b->stream);
  release(b);
  delete b;
  return CB_OK;
}

int cb_batch_set_schedule(cb_batch *b, const cb_batch_schedule *s) {
  if (!b || !s) return fail(CB_EINVAL, "cb_batch_set_schedule: null argument");
  if (s->variant < 0 || s->variant >= BATCH_VARIANTS) return fail(CB_EINVAL, "cb_batch_set_schedule: variant must be 0 or 1");
  if (s->cells_per_cta < 0 || s->ctas_per_sm < 0 || s->max_lane_width < 0)
    return fail(CB_EINVAL, "cb_batch_set_schedule: negative schedule parameter");
  BCUDA(select_device(b));
  BCUDA(cudaStreamSynchronize(b->stream));
  int per_sm = 0;
  BCUDA(occupancy(b, s->variant, &per_sm));
  if (per_sm < 1) return fail(CB_ECUDA, "cb_batch_set_schedule: the ensemble kernel does not fit on an SM");
  const int use_sm = s->ctas_per_sm > 0 ? std::min(s->ctas_per_sm, per_sm) : per_sm;
  const Plan p = make_plan(b, *s, use_sm * b->sms);
  // plan arrays: queue[n] | level[4 K]; counters: lane_sync[lanes] | lane_deck[lanes] | next[K]
  std::vector<int> h(p.queue);
  h.insert(h.end(), p.level.begin(), p.level.end());
  const int K = (int)p.level.size() / 4;
  if (b->d_plan) cudaFree(b->d_plan);
  if (b->d_sync) cudaFree(b->d_sync);
  b->d_plan = nullptr;
  b->d_sync = nullptr;
  BCUDA(cudaMalloc(&b->d_plan, sizeof(int) * h.size()));
  BCUDA(cudaMemcpy(b->d_plan, h.data(), sizeof(int) * h.size(), cudaMemcpyHostToDevice));
  BCUDA(cudaMalloc(&b->d_sync, sizeof(unsigned) * (2 * (size_t)p.lanes + K)));
  b->sched = *s;
  b->sched.ctas_per_sm = use_sm;
  b->grid = p.ctas;
  b->nlanes = p.lanes;
  b->nlevels = K;
  b->sync_words = 2 * (size_t)p.lanes + K;
  // capture the run in a graph; a capture the runtime refuses (the
  // cooperative launch attribute) leaves direct launches in use
  if (b->exec) cudaGraphExecDestroy(b->exec);
  if (b->graph) cudaGraphDestroy(b->graph);
  b->exec = nullptr;
  b->graph = nullptr;
  b->use_graph = false;
  if (cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal) == cudaSuccess) {
    cudaError_t le = enqueue_run(b);
    cudaGraph_t g = nullptr;
    cudaError_t ce = cudaStreamEndCapture(b->stream, &g);
    if (le == cudaSuccess && ce == cudaSuccess && g) {
      if (cudaGraphInstantiate(&b->exec, g, 0) == cudaSuccess) {
        b->graph = g;
        b->use_graph = true;
      } else {
        cudaGraphDestroy(g);
      }
    } else if (g) {
      cudaGraphDestroy(g);
    }
    cudaGetLastError(); // clear a refused capture's error
  }
  b->ran = false;
  return CB_OK;
}

int cb_batch_get_schedule(const cb_batch *b, cb_batch_schedule *s, int *lanes, int *ctas) {
  if (!b) return fail(CB_EINVAL, "cb_batch_get_schedule: null batch");
  if (s) *s = b->sched;
  if (lanes) *lanes = b->nlanes;
  if (ctas) *ctas = b->grid;
  return CB_OK;
}

int cb_batch_run(cb_batch *b) {
  if (!b) return fail(CB_EINVAL, "cb_batch_run: null batch");
  BCUDA(select_device(b));
  BCUDA(cudaEventRecord(b->ev0, b->stream));
  if (b->use_graph) {
    BCUDA(cudaGraphLaunch(b->exec, b->stream));
  } else {
    BCUDA(enqueue_run(b));
  }
  BCUDA(cudaEventRecord(b->ev1, b->stream));
  b->launches += 1;
  b->ran = true;
  b->results_ok = false;
  return CB_OK;
}

int cb_batch_synchronize(cb_batch *b, float *ms) {
  if (!b) return fail(CB_EINVAL, "cb_batch_synchronize: null batch");
  BCUDA(select_device(b));
  BCUDA(cudaStreamSynchronize(b->stream));
  if (!b->ran) return fail(CB_ESTATE, "cb_batch_synchronize: no run enqueued");
  int flags[2] = {0, 0};
  BCUDA(cudaMemcpy(flags, b->d_flags, sizeof(flags), cudaMemcpyDeviceToHost));
  BCUDA(cudaMemcpy(b->desc.data(), b->d_desc, sizeof(BatchDeck) * b->n, cudaMemcpyDeviceToHost));
  b->results_ok = true;
  if (ms) BCUDA(cudaEventElapsedTime(ms, b->ev0, b->ev1));
  if (flags[0]) return fail(CB_ECUDA, "cb_batch_synchronize: a lane barrier gave up (wait limit reached); the run is incomplete");
  if (flags[1]) return fail(CB_ECUDA, "cb_batch_synchronize: a tile's staging did not complete (TMA wait limit reached)");
  return CB_OK;
}

int cb_batch_autotune(cb_batch *b, int repeats, cb_batch_trial *trials, int max_trials, int *ntrials, cb_batch_schedule *best) {
  if (!b) return fail(CB_EINVAL, "cb_batch_autotune: null batch");
  if (repeats < 1) repeats = 1;
  std::vector<cb_batch_schedule> cand;
  const int cpc[] = {1024, 2048, 4096, 8192, 16384, 32768, 65536};
  for (int v = 0; v < BATCH_VARIANTS; ++v)
    for (int c : cpc) cand.push_back(cb_batch_schedule{c, BATCH_MAX_LANE, 0, v});
  float best_ms = 1e30f;
  cb_batch_schedule bs = b->sched;
  int nt = 0;
  for (const cb_batch_schedule &s : cand) {
    if (int r = cb_batch_set_schedule(b, &s)) return r;
    float tot = 0.0f;
    for (int rep = 0; rep <= repeats; ++rep) {
      if (int r = cb_batch_run(b)) return r;
      float ms = 0.0f;
      if (int r = cb_batch_synchronize(b, &ms)) return r;
      if (rep > 0) tot += ms; // the first run warms up
    }
    const float mean = tot / repeats;
    if (trials && nt < max_trials) trials[nt] = cb_batch_trial{b->sched, b->nlanes, b->grid, mean};
    ++nt;
    if (mean < best_ms) best_ms = mean, bs = b->sched;
  }
  if (ntrials) *ntrials = nt;
  if (int r = cb_batch_set_schedule(b, &bs)) return r;
  if (best) *best = b->sched;
  return CB_OK;
}

int cb_batch_deck_result(cb_batch *b, int deck, int *status, int *steps, double *time, int *nsummaries) {
  if (!b) return fail(CB_EINVAL, "cb_batch_deck_result: null batch");
  if (deck < 0 || deck >= b->n) return fail(CB_EINVAL, "cb_batch_deck_result: no deck " + std::to_string(deck));
  if (!b->results_ok) return fail(CB_ESTATE, "cb_batch_deck_result: no synchronised run");
  const BatchDeck &D = b->desc[deck];
  if (status) *status = D.status;
  if (steps) *steps = D.steps;
  if (time) *time = D.time;
  if (nsummaries) *nsummaries = D.nsummaries;
  return CB_OK;
}

int cb_batch_read_summaries(cb_batch *b, int deck, double *out, int max_records, int *count) {
  if (!b || !out) return fail(CB_EINVAL, "cb_batch_read_summaries: null argument");
  if (deck < 0 || deck >= b->n) return fail(CB_EINVAL, "cb_batch_read_summaries: no deck " + std::to_string(deck));
  if (!b->results_ok) return fail(CB_ESTATE, "cb_batch_read_summaries: no synchronised run");
  const BatchDeck &D = b->desc[deck];
  const int n = std::min(std::min(D.nsummaries, D.max_summaries), max_records);
  if (n > 0) BCUDA(cudaMemcpy(out, D.summaries, sizeof(double) * BATCH_RECORD * n, cudaMemcpyDeviceToHost));
  if (count) *count = n;
  return CB_OK;
}

int cb_batch_read_dt(cb_batch *b, int deck, double *out, int max_steps, int *count) {
  if (!b || !out) return fail(CB_EINVAL, "cb_batch_read_dt: null argument");
  if (deck < 0 || deck >= b->n) return fail(CB_EINVAL, "cb_batch_read_dt: no deck " + std::to_string(deck));
  if (!b->results_ok) return fail(CB_ESTATE, "cb_batch_read_dt: no synchronised run");
  const BatchDeck &D = b->desc[deck];
  const int n = std::min(std::min(D.steps, D.max_steps), max_steps);
  if (n > 0) BCUDA(cudaMemcpy(out, D.dt_trace, sizeof(double) * n, cudaMemcpyDeviceToHost));
  if (count) *count = n;
  return CB_OK;
}

int cb_batch_read_field(cb_batch *b, int deck, int field, double *host, size_t n, int layout) {
  if (!b || !host) return fail(CB_EINVAL, "cb_batch_read_field: null argument");
  if (deck < 0 || deck >= b->n) return fail(CB_EINVAL, "cb_batch_read_field: no deck " + std::to_string(deck));
  if (field < 0 || field >= 15) return fail(CB_EINVAL, "cb_batch_read_field: field must be a state field (0..14)");
  if (layout != CB_LAYOUT_XFAST && layout != CB_LAYOUT_YFAST) return fail(CB_EINVAL, "cb_batch_read_field: bad layout");
  BCUDA(select_device(b));
  BCUDA(cudaStreamSynchronize(b->stream));
  const BatchDeck &D = b->desc[deck];
  int sx = D.nx + 4, sy = D.ny + 4;
  switch (kind_of(field)) {
    case VERTEX: sx = D.nx + 5; sy = D.ny + 5; break;
    case XFACE: sx = D.nx + 5; break;
    case YFACE: sy = D.ny + 5; break;
    default: break;
  }
  if (n != (size_t)sx * sy) return fail(CB_EINVAL, "cb_batch_read_field: buffer size does not match the field");
  std::vector<double> xf((size_t)sx * sy);
  const char *base = (const char *)D.buf[field] + (size_t)D.off * b->esize; // the identity mapping a finished step leaves
  if (b->precision == CB_FP64) {
    BCUDA(cudaMemcpy2D(xf.data(), sizeof(double) * sx, base, sizeof(double) * D.pitch, sizeof(double) * sx, sy, cudaMemcpyDeviceToHost));
  } else {
    std::vector<float> t((size_t)sx * sy);
    BCUDA(cudaMemcpy2D(t.data(), sizeof(float) * sx, base, sizeof(float) * D.pitch, sizeof(float) * sx, sy, cudaMemcpyDeviceToHost));
    for (size_t q = 0; q < t.size(); ++q) xf[q] = t[q];
  }
  if (layout == CB_LAYOUT_XFAST) {
    std::memcpy(host, xf.data(), sizeof(double) * xf.size());
  } else {
    for (int i = 0; i < sx; ++i)
      for (int j = 0; j < sy; ++j) host[(size_t)i * sy + j] = xf[(size_t)j * sx + i];
  }
  return CB_OK;
}

int cb_batch_get_stream(cb_batch *b, void **stream) {
  if (!b || !stream) return fail(CB_EINVAL, "cb_batch_get_stream: null argument");
  *stream = (void *)b->stream;
  return CB_OK;
}

int cb_batch_launch_count(const cb_batch *b, long long *count) {
  if (!b || !count) return fail(CB_EINVAL, "cb_batch_launch_count: null argument");
  *count = b->launches;
  return CB_OK;
}

} // extern "C"
