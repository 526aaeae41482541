// cb_phase.cuh -- one CUDA kernel per hydro phase (the "phase" path).
//
// Each kernel is one pass over the mesh that does the whole of the
// reference routine it replaces (all of its loops fused, intermediate work
// arrays kept on chip) and, when asked, also writes the reflective halo of
// its outputs so that the update_halo call that follows becomes a no-op.
// The arithmetic of every expression keeps the reference's operation order;
// built with -fmad=false the FP64 instantiation is bit-identical to the
// reference serial model.
//
// Kernels are templated on the storage type T (double, or float for the
// FP32 form).  Where the FP32 form keeps FP64 (calc_dt's minimum, the
// summary sums, cell-advection mass/energy accumulation) the code says
// `double` explicitly.
#pragma once

#include <cstring>

#include "cb_mesh.cuh"
#include "cb_ops.h"

namespace cb {

// Fields of one chunk as seen by a kernel launch.
template <typename T> struct Fields {
  T *f[NUM_FIELDS];
};

// ---------------------------------------------------------------------------
// generate_chunk: src/serial/generate_chunk.cpp:31-131.  Later states
// overwrite earlier ones; a node takes the velocity of the last state that
// paints any of the (up to four) cells whose loop iteration writes it.
template <typename T>
__device__ __forceinline__ bool state_hits(const DevState &s, const Mesh<T> &m, const double *cellx, const double *celly,
                                           const double *vertexx, const double *vertexy, int i, int j) {
  if (s.geometry == 1) {
    return (vertexx[i + 1] >= s.xmin && vertexx[i] < s.xmax) && (vertexy[j + 1] >= s.ymin && vertexy[j] < s.ymax);
  } else if (s.geometry == 2) {
    double x_cent = s.xmin, y_cent = s.ymin;
    double radius = sqrt((cellx[i] - x_cent) * (cellx[i] - x_cent) + (celly[j] - y_cent) * (celly[j] - y_cent));
    return radius <= s.radius;
  } else if (s.geometry == 3) {
    return vertexx[i] == s.xmin && vertexy[j] == s.ymin;
  }
  return false;
}

// Element (i, j) of the full extents (cells [0, nx+4) x [0, ny+4), nodes up
// to nx+4 / ny+4).
template <typename T>
__device__ __forceinline__ void generate_element(const Fields<T> &F, const Mesh<T> &m, const DevState *st, int nstates, const double *cellx,
                                                 const double *celly, const double *vertexx, const double *vertexy, int i, int j) {
  const int xr = m.nx + 4, yr = m.ny + 4;
  if (i > xr || j > yr) return;
  // cell part (cells cover [0, xr) x [0, yr))
  if (i < xr && j < yr) {
    double e = st[0].energy, d = st[0].density;
    for (int s = 1; s < nstates; ++s) {
      if (state_hits(st[s], m, cellx, celly, vertexx, vertexy, i, j)) {
        e = st[s].energy;
        d = st[s].density;
      }
    }
    F.f[ENERGY0][m.at(i, j)] = (T)e;
    F.f[DENSITY0][m.at(i, j)] = (T)d;
  }
  // node part: node (i, j) is written by cells (i-1..i, j-1..j)
  bool painted = false;
  double u = 0.0, v = 0.0;
  if (i < xr && j < yr) {
    u = st[0].xvel;
    v = st[0].yvel;
    painted = true;
  }
  for (int s = 1; s < nstates; ++s) {
    bool hit = false;
    for (int cj = j - 1; cj <= j; ++cj)
      for (int ci = i - 1; ci <= i; ++ci)
        if (ci >= 0 && cj >= 0 && ci < xr && cj < yr && state_hits(st[s], m, cellx, celly, vertexx, vertexy, ci, cj)) hit = true;
    if (hit) {
      u = st[s].xvel;
      v = st[s].yvel;
      painted = true;
    }
  }
  if (painted) {
    F.f[XVEL0][m.at(i, j)] = (T)u;
    F.f[YVEL0][m.at(i, j)] = (T)v;
  }
}

template <typename T>
__global__ void k_generate_chunk(Fields<T> F, Mesh<T> m, const DevState *st, int nstates, const double *cellx,
                                 const double *celly, const double *vertexx, const double *vertexy) {
  generate_element(F, m, st, nstates, cellx, celly, vertexx, vertexy, blockIdx.x * blockDim.x + threadIdx.x,
                   blockIdx.y * blockDim.y + threadIdx.y);
}

// ---------------------------------------------------------------------------
// ideal_gas: src/serial/ideal_gas.cpp:28-48.  gm1 = gamma - 1 (0.4 at the
// reference's hard-coded gamma = 1.4).
template <typename T>
__device__ __forceinline__ void eos(T density, T energy, T gm1, T &pressure, T &soundspeed) {
  T v = lim_div(T(1.0), density); // feeds the sound speed only
  pressure = gm1 * density * energy;
  T pressurebyenergy = gm1 * density;
  T pressurebyvolume = -density * pressure;
  T sound_speed_squared = v * v * (pressure * pressurebyenergy - pressurebyvolume);
  soundspeed = sqrt(sound_speed_squared);
}

// 16-byte vectors of the storage type for the pointwise kernels.  The
// first interior column (i = 2) of every field sits on a 256-byte
// boundary, so elements i = 2 + N k start aligned vectors.
template <typename T> struct Vec16;
template <> struct Vec16<double> {
  using type = double2;
  static constexpr int N = 2;
};
template <> struct Vec16<float> {
  using type = float4;
  static constexpr int N = 4;
};

// True when the block of a pointwise kernel (columns [ilo, ihi], rows
// [jlo, jhi]) lies within 8 elements of a mesh edge, where folds happen.
__device__ __forceinline__ bool near_edge(int nx, int ny, int ilo, int ihi, int jlo, int jhi) {
  return ilo < 10 || ihi > nx - 8 || jlo < 10 || jhi > ny - 8;
}

// Blocks of the pointwise phases are 32 x 8 threads.
constexpr int PW_X = 32, PW_Y = 8;

// One 32 x 8 block (block coordinates (bx, by), thread (tx, ty)); each
// thread handles N consecutive cells of one row.
template <typename T>
__device__ __forceinline__ void ideal_gas_block(const Fields<T> &F, const Mesh<T> &m, int predict, T gm1, int fold, int bx, int by, int tx,
                                                int ty) {
  constexpr int N = Vec16<T>::N;
  using V = typename Vec16<T>::type;
  const int i0 = 2 + (bx * PW_X + tx) * N;
  const int j = 2 + by * PW_Y + ty;
  const bool edge = fold && near_edge(m.nx, m.ny, 2 + bx * PW_X * N, 2 + (bx + 1) * PW_X * N, 2 + by * PW_Y, 2 + (by + 1) * PW_Y);
  if (i0 >= m.nx + 2 || j >= m.ny + 2) return;
  const long long id = m.at(i0, j);
  const T *den = F.f[predict ? DENSITY1 : DENSITY0], *ene = F.f[predict ? ENERGY1 : ENERGY0];
  T d[N], e[N], p[N], c[N];
  const bool whole = i0 + N - 1 <= m.nx + 1;
  if (whole) {
    const V dv = *reinterpret_cast<const V *>(den + id), ev = *reinterpret_cast<const V *>(ene + id);
    memcpy(d, &dv, sizeof(V));
    memcpy(e, &ev, sizeof(V));
  } else {
#pragma unroll
    for (int k = 0; k < N; ++k) {
      d[k] = i0 + k <= m.nx + 1 ? den[id + k] : T(1);
      e[k] = i0 + k <= m.nx + 1 ? ene[id + k] : T(0);
    }
  }
#pragma unroll
  for (int k = 0; k < N; ++k) eos(d[k], e[k], gm1, p[k], c[k]);
  if (whole) {
    V pv, cv;
    memcpy(&pv, p, sizeof(V));
    memcpy(&cv, c, sizeof(V));
    *reinterpret_cast<V *>(F.f[PRESSURE] + id) = pv;
    *reinterpret_cast<V *>(F.f[SOUNDSPEED] + id) = cv;
  } else {
#pragma unroll
    for (int k = 0; k < N; ++k)
      if (i0 + k <= m.nx + 1) {
        F.f[PRESSURE][id + k] = p[k];
        F.f[SOUNDSPEED][id + k] = c[k];
      }
  }
  if (edge) {
#pragma unroll
    for (int k = 0; k < N; ++k)
      if (i0 + k <= m.nx + 1) fold_halo(F.f[PRESSURE], m, halo_rule(PRESSURE), fold, i0 + k, j, p[k]);
  }
}

template <typename T>
__global__ void k_ideal_gas(Fields<T> F, Mesh<T> m, int predict, T gm1, int fold) {
  ideal_gas_block(F, m, predict, gm1, fold, blockIdx.x, blockIdx.y, threadIdx.x, threadIdx.y);
}

// ---------------------------------------------------------------------------
// Block-wide FP64 minimum (calc_dt's reduction).
__device__ __forceinline__ double warp_min(double v) {
  for (int o = 16; o > 0; o >>= 1) v = fmin(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

// Block-wide min of v (any block size that is a multiple of 32, <= 1024);
// thread 0 then folds it into *out with one 64-bit atomicMin.
__device__ __forceinline__ void block_min_to(double v, unsigned long long *out) {
  __shared__ double wmin[32];
  v = warp_min(v);
  const int lane = (threadIdx.y * blockDim.x + threadIdx.x) & 31;
  const int warp = (threadIdx.y * blockDim.x + threadIdx.x) >> 5;
  const int nw = (blockDim.x * blockDim.y) >> 5;
  if (lane == 0) wmin[warp] = v;
  __syncthreads();
  if (warp == 0) {
    v = lane < nw ? wmin[lane] : g_big;
    v = warp_min(v);
    if (lane == 0 && v >= 0.0) atomicMin(out, (unsigned long long)__double_as_longlong(v));
  }
}

// ---------------------------------------------------------------------------
// revert: src/serial/revert.cpp:29-41.
template <typename T>
__global__ void k_revert(Fields<T> F, Mesh<T> m) {
  const int i = 2 + blockIdx.x * blockDim.x + threadIdx.x;
  const int j = 2 + blockIdx.y * blockDim.y + threadIdx.y;
  if (i >= m.nx + 2 || j >= m.ny + 2) return;
  const long long id = m.at(i, j);
  F.f[DENSITY1][id] = F.f[DENSITY0][id];
  F.f[ENERGY1][id] = F.f[ENERGY0][id];
}

// ---------------------------------------------------------------------------
// reset_field: src/serial/reset_field.cpp:28-51.
// With a fold, level 0 also gets the halo update_halo(depth) would give it.
// Each thread copies N consecutive elements of one row (block 32 x 8):
// cells [2, nx+1] x [2, ny+1] for density/energy, nodes [2, nx+2] x
// [2, ny+2] for the velocities.
template <typename T>
__device__ __forceinline__ void reset_field_block(const Fields<T> &F, const Mesh<T> &m, int fold, int bx, int by, int tx, int ty) {
  constexpr int N = Vec16<T>::N;
  using V = typename Vec16<T>::type;
  const int i0 = 2 + (bx * PW_X + tx) * N;
  const int j = 2 + by * PW_Y + ty;
  const bool edge = fold && near_edge(m.nx, m.ny, 2 + bx * PW_X * N, 2 + (bx + 1) * PW_X * N, 2 + by * PW_Y, 2 + (by + 1) * PW_Y);
  if (i0 > m.nx + 2 || j > m.ny + 2) return;
  const long long id = m.at(i0, j);
  const bool cell_row = j <= m.ny + 1;
  auto copy = [&](int src, int dst, int imax) {
    if (i0 + N - 1 <= imax) {
      *reinterpret_cast<V *>(F.f[dst] + id) = *reinterpret_cast<const V *>(F.f[src] + id);
    } else {
#pragma unroll
      for (int k = 0; k < N; ++k)
        if (i0 + k <= imax) F.f[dst][id + k] = F.f[src][id + k];
    }
  };
  if (cell_row) {
    copy(DENSITY1, DENSITY0, m.nx + 1);
    copy(ENERGY1, ENERGY0, m.nx + 1);
  }
  copy(XVEL1, XVEL0, m.nx + 2);
  copy(YVEL1, YVEL0, m.nx + 2);
  if (edge) {
#pragma unroll
    for (int k = 0; k < N; ++k) {
      const int i = i0 + k;
      if (cell_row && i <= m.nx + 1) {
        fold_halo(F.f[DENSITY0], m, halo_rule(DENSITY0), fold, i, j, F.f[DENSITY0][id + k]);
        fold_halo(F.f[ENERGY0], m, halo_rule(ENERGY0), fold, i, j, F.f[ENERGY0][id + k]);
      }
      if (i <= m.nx + 2) {
        fold_halo(F.f[XVEL0], m, halo_rule(XVEL0), fold, i, j, F.f[XVEL0][id + k]);
        fold_halo(F.f[YVEL0], m, halo_rule(YVEL0), fold, i, j, F.f[YVEL0][id + k]);
      }
    }
  }
}

// Copies the elements of `src` outside the rectangle [ilo, ihi] x [jlo, jhi]
// (the ring of width 2 or 3 around it) into `dst`, so a double-buffered
// update leaves dst's halo exactly as the in-place reference leaves it.
// Threads enumerate the ring only: the rows below jlo, the rows above jhi,
// then the left and right pieces of the rows in between.  blockIdx.y picks
// one of up to two (src, dst) pairs.
struct RingPair {
  const void *src[2];
  void *dst[2];
};

template <typename T>
__global__ void k_copy_ring(RingPair rp, Mesh<T> m, int ilo, int ihi, int jlo, int jhi, int ext_x, int ext_y) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int w = ext_x, h = ext_y;
  const long long nb = (long long)jlo * w, nt = (long long)(h - 1 - jhi) * w;
  const int side = ilo + (w - 1 - ihi); // ring elements per middle row
  const long long nm = (long long)(jhi - jlo + 1) * side;
  int i, j;
  if (t < nb) {
    i = (int)(t % w), j = (int)(t / w);
  } else if (t < nb + nt) {
    const long long u = t - nb;
    i = (int)(u % w), j = jhi + 1 + (int)(u / w);
  } else if (t < nb + nt + nm) {
    const long long u = t - nb - nt;
    const int c = (int)(u % side);
    j = jlo + (int)(u / side);
    i = c < ilo ? c : ihi + 1 + (c - ilo);
  } else {
    return;
  }
  const T *src = (const T *)rp.src[blockIdx.y];
  T *dst = (T *)rp.dst[blockIdx.y];
  dst[m.at(i, j)] = src[m.at(i, j)];
}

template <typename T>
__global__ void k_reset_field(Fields<T> F, Mesh<T> m, int fold) {
  reset_field_block(F, m, fold, blockIdx.x, blockIdx.y, threadIdx.x, threadIdx.y);
}

// The interior of level 1 as the step's last sweeps and reset_field leave it
// (energy1 = energy0 on cells [2, nx+1] x [2, ny+1]; xvel1 = xvel0, yvel1 =
// yvel0 on nodes [2, nx+2] x [2, ny+2]): the end of a resident loop whose
// second sweeps wrote those to level 0 only.  One thread per node.
template <typename T> __global__ void k_level1_from_level0(Fields<T> F, Mesh<T> m) {
  const int i = 2 + blockIdx.x * blockDim.x + threadIdx.x, j = 2 + blockIdx.y * blockDim.y + threadIdx.y;
  if (i > m.nx + 2 || j > m.ny + 2) return;
  const long long g = m.at(i, j);
  F.f[XVEL1][g] = F.f[XVEL0][g];
  F.f[YVEL1][g] = F.f[YVEL0][g];
  if (i <= m.nx + 1 && j <= m.ny + 1) F.f[ENERGY1][g] = F.f[ENERGY0][g];
}

// ---------------------------------------------------------------------------
// update_halo: src/serial/update_halo.cpp:33-684 in two launches: pass 0 does
// bottom then top for every column, pass 1 left then right for every row, so
// corner and tiny-mesh semantics are the reference's exactly.
// Column (pass 0) or row (pass 1) t of field f's halo fill.
// Only the faces in `faces` (bits 1 left, 2 right, 4 bottom, 8 top) are
// filled: a tile's faces that border another tile get that tile's values
// instead (k_tile_halo), as the reference fills only faces whose chunk and
// tile neighbours are both external (src/serial/update_halo.cpp:41-71).
template <typename T>
__device__ __forceinline__ void halo_fill(const Fields<T> &F, const Mesh<T> &m, int f, int depth, int pass, int t, int faces = 15) {
  const HaloRule r = halo_rule(f);
  T *a = F.f[f];
  const int d = depth;
  if (pass == 0) {
    const int jcol = 2 - d + t;
    if (jcol >= m.nx + r.xe + d + 2) return;
    if (faces & 4)
      for (int k = 0; k < d; ++k) {
        int src = r.soundspeed_bottom_quirk ? k : r.bot_src + k;
        a[m.at(jcol, 1 - k)] = (T)(r.sign_bt * (double)a[m.at(jcol, src)]);
      }
    if (faces & 8)
      for (int k = 0; k < d; ++k) a[m.at(jcol, m.ny + r.top_dst + k)] = (T)(r.sign_bt * (double)a[m.at(jcol, m.ny + r.top_src - k)]);
  } else {
    const int krow = 2 - d + t;
    if (krow >= m.ny + r.ye + d + 2) return;
    if (faces & 1)
      for (int k = 0; k < d; ++k) a[m.at(1 - k, krow)] = (T)(r.sign_lr * (double)a[m.at(r.left_src + k, krow)]);
    if (faces & 2)
      for (int k = 0; k < d; ++k) a[m.at(m.nx + r.right_dst + k, krow)] = (T)(r.sign_lr * (double)a[m.at(m.nx + r.right_src - k, krow)]);
  }
}

template <typename T>
__global__ void k_update_halo(Fields<T> F, Mesh<T> m, HaloJob job, int depth, int pass, int faces) {
  if ((int)blockIdx.y >= job.nfields) return;
  halo_fill(F, m, job.field[blockIdx.y], depth, pass, blockIdx.x * blockDim.x + threadIdx.x, faces);
}

// ---------------------------------------------------------------------------
// Tile halo exchange: src/serial/update_tile_halo_kernel.cpp.  The halo of
// `dst` on one side, `depth` deep, from the interior of `src`, the tile on
// that side (they share the extent along the strip).  Along the strip the
// copy runs over [2 - depth, n + depth + 1], one element further for the
// arrays that extend one past the cells that way (nodes; y faces for a left /
// right strip, x faces for a bottom / top one).  Across it, element k of the
// halo (k = 0 nearest the interior):
//   left   dst(1 - k, .)              <- src(src.nx + 1 - k, .)
//   right  dst(nx + 2 + e + k, .)     <- src(2 + e + k, .)      e = 1 for nodes and x faces
//   bottom dst(., 1 - k)              <- src(., src.ny + 1 - k)
//   top    dst(., ny + 2 + e + k)     <- src(., 2 + e + k)      e = 1 for nodes and y faces
// One thread per (strip position, k), blockIdx.y the field.
template <typename T>
__global__ void k_tile_halo(Fields<T> D, Mesh<T> md, Fields<T> S, Mesh<T> ms, HaloJob job, int side, int depth) {
  if ((int)blockIdx.y >= job.nfields) return;
  const int f = job.field[blockIdx.y];
  const Kind kd = kind_of(f);
  const bool lr = side == 1 || side == 2;
  const int along_extra = lr ? (kd == VERTEX || kd == YFACE) : (kd == VERTEX || kd == XFACE);
  const int across_extra = lr ? (kd == VERTEX || kd == XFACE) : (kd == VERTEX || kd == YFACE);
  const int n_along = (lr ? md.ny : md.nx) + 2 * depth + along_extra; // positions 2 - depth .. n + depth + 1 (+1)
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n_along * depth) return;
  const int p = 2 - depth + t % n_along, k = t / n_along;
  int di, dj, si, sj;
  if (side == 1) {
    di = 1 - k, si = ms.nx + 1 - k, dj = sj = p;
  } else if (side == 2) {
    di = md.nx + 2 + across_extra + k, si = 2 + across_extra + k, dj = sj = p;
  } else if (side == 4) {
    dj = 1 - k, sj = ms.ny + 1 - k, di = si = p;
  } else {
    dj = md.ny + 2 + across_extra + k, sj = 2 + across_extra + k, di = si = p;
  }
  D.f[f][md.at(di, dj)] = S.f[f][ms.at(si, sj)];
}

// ---------------------------------------------------------------------------
// Face strips of a decomposed run: driver/comms.cpp:clover_exchange with the
// index rules of src/serial/pack_kernel.cpp (the same elements as
// k_tile_halo's, between a chunk and a linear buffer).  Along the face the
// strip runs over [2 - depth, n + depth + 1], one element further for the
// arrays that extend one past the cells that way; across it, element k
// (k = 0 nearest the face):
//   pack, the strip for the neighbour on    left (2 + e + k, .)   right (nx + 1 - k, .)
//                                           bottom (., 2 + e + k)  top (., ny + 1 - k)
//   unpack, the chunk's own halo on         left (1 - k, .)       right (nx + 2 + e + k, .)
//                                           bottom (., 1 - k)      top (., ny + 2 + e + k)
// with e = 1 for the arrays one longer across the face.  Element (p, k) of
// field slot s sits at buf[off[s] + k * n_along + p - (2 - depth)].  One
// thread per element, blockIdx.y the field slot.
template <typename T>
__global__ void k_face_strip(Fields<T> F, Mesh<T> m, StripJob job, int side, int depth, T *buf, int pack) {
  if ((int)blockIdx.y >= job.nfields) return;
  const int f = job.field[blockIdx.y];
  const Kind kd = kind_of(f);
  const bool lr = side == 1 || side == 2;
  const int along_extra = lr ? (kd == VERTEX || kd == YFACE) : (kd == VERTEX || kd == XFACE);
  const int e = lr ? (kd == VERTEX || kd == XFACE) : (kd == VERTEX || kd == YFACE);
  const int n_along = (lr ? m.ny : m.nx) + 2 * depth + along_extra;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n_along * depth) return;
  const int p = 2 - depth + t % n_along, k = t / n_along;
  int across;
  if (side == 1)
    across = pack ? 2 + e + k : 1 - k;
  else if (side == 2)
    across = pack ? m.nx + 1 - k : m.nx + 2 + e + k;
  else if (side == 4)
    across = pack ? 2 + e + k : 1 - k;
  else
    across = pack ? m.ny + 1 - k : m.ny + 2 + e + k;
  const long long id = lr ? m.at(across, p) : m.at(p, across);
  T *b = buf + job.off[blockIdx.y] + t;
  if (pack)
    *b = F.f[f][id];
  else
    F.f[f][id] = *b;
}

// ---------------------------------------------------------------------------
// field_summary: src/serial/field_summary.cpp:44-104 -- ideal_gas on level 0
// (writing pressure and soundspeed as the reference does), then the five
// sums.  Per-cell terms are formed exactly as the reference forms them; the
// sums are FP64 block partials, reduced by the last block in block order, so
// the result does not depend on scheduling.
// The cell's ideal_gas (pressure and soundspeed written) and its terms of
// the five sums, added to s.
template <typename T>
__device__ __forceinline__ void summary_cell(const Fields<T> &F, const Mesh<T> &m, T gm1, int i, int j, double s[5], bool store_ps = true) {
  const long long id = m.at(i, j);
  const T d0 = F.f[DENSITY0][id], e0 = F.f[ENERGY0][id];
  T p, c;
  eos(d0, e0, gm1, p, c);
  if (store_ps) { // ideal_gas's stores (the resident loop keeps them for its last step only)
    F.f[PRESSURE][id] = p;
    F.f[SOUNDSPEED][id] = c;
  }
  const T *u = F.f[XVEL0], *v = F.f[YVEL0];
  double vsqrd = 0.0;
  for (int kv = j; kv <= j + 1; ++kv)
    for (int jv = i; jv <= i + 1; ++jv) {
      const double uu = u[m.at(jv, kv)], vv = v[m.at(jv, kv)];
      vsqrd += 0.25 * (uu * uu + vv * vv);
    }
  const double cell_vol = m.celldx[i] * m.celldy[j];
  const double cell_mass = cell_vol * (double)d0;
  s[0] += cell_vol;
  s[1] += cell_mass;
  s[2] += cell_mass * (double)e0;
  s[3] += cell_mass * 0.5 * vsqrd;
  s[4] += cell_vol * (double)p;
}

template <typename T>
__global__ void k_field_summary(Fields<T> F, Mesh<T> m, T gm1, double *partials, unsigned int *counter, double *out,
                                int tiles_x, int ntiles, const int *store_ps) {
  double s[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
  const bool st = !store_ps || *store_ps != 0;
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const int i = 2 + (t % tiles_x) * blockDim.x + threadIdx.x;
    const int j = 2 + (t / tiles_x) * blockDim.y + threadIdx.y;
    if (i >= m.nx + 2 || j >= m.ny + 2) continue;
    summary_cell(F, m, gm1, i, j, s, st);
  }
  // block reduction (fixed tree order)
  __shared__ double red[5][256];
  const int tid = threadIdx.y * blockDim.x + threadIdx.x;
  const int nt = blockDim.x * blockDim.y;
  for (int q = 0; q < 5; ++q) red[q][tid] = s[q];
  __syncthreads();
  for (int w = nt / 2; w > 0; w >>= 1) {
    if (tid < w)
      for (int q = 0; q < 5; ++q) red[q][tid] += red[q][tid + w];
    __syncthreads();
  }
  const unsigned int nb = gridDim.x;
  const unsigned int b = blockIdx.x;
  __shared__ bool last;
  if (tid == 0) {
    for (int q = 0; q < 5; ++q) partials[(size_t)q * nb + b] = red[q][0];
    __threadfence();
    last = atomicAdd(counter, 1u) == nb - 1;
  }
  __syncthreads();
  if (!last) return;
  __threadfence();
  // the last block sums the partials: each thread a strided slice, then a tree
  for (int q = 0; q < 5; ++q) {
    double acc = 0.0;
    for (unsigned int p = tid; p < nb; p += nt) acc += ((volatile double *)partials)[(size_t)q * nb + p];
    red[q][tid] = acc;
  }
  __syncthreads();
  for (int w = nt / 2; w > 0; w >>= 1) {
    if (tid < w)
      for (int q = 0; q < 5; ++q) red[q][tid] += red[q][tid + w];
    __syncthreads();
  }
  if (tid == 0) {
    for (int q = 0; q < 5; ++q) out[q] = red[q][0];
    *counter = 0u;
  }
}

} // namespace cb
