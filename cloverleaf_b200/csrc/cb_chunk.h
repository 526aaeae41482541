// cb_chunk.h -- host-side state of one mesh chunk owned by the C-ABI library.
#pragma once

#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>
#include <string>

#include "cb_mesh.cuh"

namespace cb {

constexpr int NUM_SPARE = 4; // second buffers for the double-buffered in-place phases

struct Chunk {
  int nx = 0, ny = 0;
  int precision = 0; // 0 FP64, 1 FP32
  int device = 0;
  size_t esize = 8;       // bytes per element
  long long pitch = 0;    // elements per row
  size_t off = 0;         // elements before logical (0, 0) in an allocation
  size_t alloc_elems = 0; // elements per allocation
  double gamma = 1.4;

  void *field_mem[NUM_FIELDS] = {};  // allocation backing each field (nullptr = not allocated)
  void *spare_mem[NUM_SPARE] = {};
  // geometry: FP64 on device for every precision, plus a copy in the storage type
  double *geom_d[NUM_GEOM] = {};
  void *geom_t[NUM_GEOM] = {};
  double *geom_h[NUM_GEOM] = {};
  int geom_len = 0;

  cudaStream_t stream = nullptr;
  unsigned long long *d_dt_bits = nullptr;
  double *d_partials = nullptr;
  unsigned int *d_counter = nullptr;
  double *d_sums = nullptr;
  double *h_scalars = nullptr; // pinned: [0] dt, [1..5] sums
  int summary_grid = 0;

  int halo_fresh[15] = {};     // depth to which each field's halo matches update_halo
  bool fold_enabled = true;    // fold halos into producers when the mesh allows it
  bool reset_by_swap = false;  // reset_field swaps level buffers instead of copying

  long long launches = 0; // kernels launched for this chunk

  bool can_fold() const { return fold_enabled && nx >= 8 && ny >= 8; }
  void *base(int f) const { return field_mem[f] ? (char *)field_mem[f] + off * esize : nullptr; }
  void *spare_base(int s) const { return (char *)spare_mem[s] + off * esize; }
};

} // namespace cb
