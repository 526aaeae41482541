// cb_noalloc.cu -- cb_field_summary_noalloc: the field summary over arrays
// the caller owns, with no memory allocation of any kind.
//
// Who needs it: code that may not allocate device memory at the point it
// wants the summary -- a host program whose device memory is handed out by
// its own pool or arena (so a stray cudaMalloc would break its accounting
// or fragment it), or a caller running where cudaMalloc is not allowed to
// happen at all, such as between the steps of a loop that is being timed
// or checked for allocation-free operation.  cb_field_summary needs a
// cb_chunk, whose creation allocates every field and the reduction scratch;
// this entry point needs neither.
//
// The reduction's block partial sums and its completion counter live in one
// file-scope __device__ array of fixed size: NOALLOC_MAX_TILES blocks of
// 32 x 8 cells, one block per tile.  A mesh is accepted when
// ceil(nx / 32) * ceil(ny / 8) <= NOALLOC_MAX_TILES (16384): 4,194,304 cells
// when nx is a multiple of 32 and ny of 8, fewer otherwise (2050 x 2040 needs
// 16575 blocks and is rejected).  Every GPU that loads the library holds that
// array until the process exits.  Host code cannot use the array's name as a
// device address, so the first call on each device asks the runtime for the
// address with cudaGetSymbolAddress (with that device current) and caches it.
// The address belongs to the device's primary context: the entry point must
// not be called across cudaDeviceReset or from another context created on
// the same device (cuCtxCreate), and its first call on a device should come
// before any stream capture.  All calls on a device share the array: the
// counter is cleared on the stream before each launch, and calls whose work
// overlaps on the GPU (different streams, no ordering between them) race on
// it and give wrong sums.
//
// Compiled with -fmad=false like the FP64 kernels: per-cell terms are
// bit-identical to cb_field_summary's; only the grouping of the sums differs.
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "../../include/cloverb200.h"
#include "cb_phase.cuh"

namespace {

constexpr int NOALLOC_TILE_X = 32, NOALLOC_TILE_Y = 8;
constexpr int NOALLOC_MAX_TILES = 16384;
constexpr int NOALLOC_MAX_DEVICES = 64;

// [0, 5 * NOALLOC_MAX_TILES): block partials; then the completion counter.
static __device__ __align__(256) double g_summary_scratch[5 * NOALLOC_MAX_TILES + 32];

std::mutex g_mu;
void *g_scratch_addr[NOALLOC_MAX_DEVICES] = {};

} // namespace

namespace cb {
// Defined in cb_api.cu: records the message cb_last_error() returns.
int set_last_error(int code, const std::string &msg);
} // namespace cb

extern "C" int cb_field_summary_noalloc(int nx, int ny, long long pitch, const double *density0, const double *energy0,
                                        const double *xvel0, const double *yvel0, const double *celldx, const double *celldy,
                                        double *pressure, double *soundspeed, double gamma, double *sums, void *stream) {
  using namespace cb;
  if (nx < 1 || ny < 1) return set_last_error(CB_EINVAL, "cb_field_summary_noalloc: mesh must have at least one cell per direction");
  if (pitch < (long long)nx + 5)
    return set_last_error(CB_EINVAL, "cb_field_summary_noalloc: pitch " + std::to_string(pitch) + " is below nx + 5");
  if (!density0 || !energy0 || !xvel0 || !yvel0 || !celldx || !celldy || !pressure || !soundspeed || !sums)
    return set_last_error(CB_EINVAL, "cb_field_summary_noalloc: null array");
  if (!(gamma > 1.0)) return set_last_error(CB_EINVAL, "cb_field_summary_noalloc: gamma must be above 1");
  const long long tiles_x = (nx + NOALLOC_TILE_X - 1) / NOALLOC_TILE_X, tiles_y = (ny + NOALLOC_TILE_Y - 1) / NOALLOC_TILE_Y;
  if (tiles_x * tiles_y > NOALLOC_MAX_TILES)
    return set_last_error(CB_EINVAL, "cb_field_summary_noalloc: a " + std::to_string(nx) + " x " + std::to_string(ny) + " mesh needs " +
                                         std::to_string(tiles_x * tiles_y) + " reduction blocks; the fixed scratch holds " +
                                         std::to_string(NOALLOC_MAX_TILES) + " (ceil(nx/32) * ceil(ny/8) must not exceed it)");
  if (pitch * (long long)(ny + 5) >= (1ll << 31)) return set_last_error(CB_EINVAL, "cb_field_summary_noalloc: arrays above 2^31 elements");
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return set_last_error(CB_ECUDA, std::string("cb_field_summary_noalloc: ") + cudaGetErrorString(e));
  if (dev < 0 || dev >= NOALLOC_MAX_DEVICES) return set_last_error(CB_EINVAL, "cb_field_summary_noalloc: device ordinal out of range");
  void *scratch = nullptr;
  {
    std::lock_guard<std::mutex> lock(g_mu);
    if (!g_scratch_addr[dev]) {
      // the device address of the static array on the current device
      e = cudaGetSymbolAddress(&g_scratch_addr[dev], g_summary_scratch);
      if (e != cudaSuccess) {
        g_scratch_addr[dev] = nullptr;
        return set_last_error(CB_ECUDA, std::string("cb_field_summary_noalloc: cudaGetSymbolAddress: ") + cudaGetErrorString(e));
      }
    }
    scratch = g_scratch_addr[dev];
  }
  double *partials = (double *)scratch;
  unsigned int *counter = (unsigned int *)(partials + 5 * NOALLOC_MAX_TILES);
  cudaStream_t s = (cudaStream_t)stream;
  e = cudaMemsetAsync(counter, 0, sizeof(unsigned int), s); // the completion counter must start at zero
  if (e != cudaSuccess) return set_last_error(CB_ECUDA, std::string("cb_field_summary_noalloc: ") + cudaGetErrorString(e));

  Fields<double> F{};
  F.f[DENSITY0] = const_cast<double *>(density0);
  F.f[ENERGY0] = const_cast<double *>(energy0);
  F.f[XVEL0] = const_cast<double *>(xvel0);
  F.f[YVEL0] = const_cast<double *>(yvel0);
  F.f[PRESSURE] = pressure;
  F.f[SOUNDSPEED] = soundspeed;
  Mesh<double> m{};
  m.nx = nx;
  m.ny = ny;
  m.pitch = pitch;
  m.celldx = celldx;
  m.celldy = celldy;
  m.celldx_t = celldx;
  m.celldy_t = celldy;
  const int nt = (int)(tiles_x * tiles_y);
  k_field_summary<double><<<nt, dim3(NOALLOC_TILE_X, NOALLOC_TILE_Y), 0, s>>>(F, m, gamma - 1.0, partials, counter, sums, (int)tiles_x, nt,
                                                                          nullptr);
  e = cudaGetLastError();
  if (e != cudaSuccess) return set_last_error(CB_ECUDA, std::string("cb_field_summary_noalloc: launch: ") + cudaGetErrorString(e));
  return CB_OK;
}
