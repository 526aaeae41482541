// context.h -- the b200 model's context and buffer types, as the reference
// driver expects every model to provide them (driver/definitions.h:22
// includes this file and embeds the buffers by value in field_type).
//
// The buffers hold no memory of their own.  All field storage lives on the
// B200 inside libcloverb200 (one cb_chunk per tile); build_field binds each
// Buffer2D / geometry Buffer1D of the tile to its slot in that chunk, and
// mirrored() copies the slot out through the C ABI.  Copies of a buffer are
// cheap handles to the same slot (the reference CUDA model's buffers are
// handles too, src/cuda/context.h:146-160).
#pragma once

#include <cstddef>
#include <iostream>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "cloverb200.h"
#include "shared.h"

namespace clover {

struct Runtime; // per-run state of the b200 model (model/b200_runtime.h)

struct context {
  int device = 0;
  int precision = CB_FP64;
  std::shared_ptr<Runtime> rt;
};

struct chunk_context {};

[[noreturn]] void b200_fatal(const std::string &where);

template <typename T> struct Buffer1D {
  size_t size;
  cb_chunk *chunk = nullptr;
  int geom = -1;             // 1-D geometry slot when bound
  std::shared_ptr<std::vector<T>> host; // plain host storage otherwise

  Buffer1D(context &, size_t size) : size(size), host(std::make_shared<std::vector<T>>(size)) {}
  T &operator[](size_t i) const { return (*host)[i]; }
  template <size_t D> [[nodiscard]] size_t extent() const {
    static_assert(D < 1);
    return size;
  }
  void bind(cb_chunk *c, int g) {
    chunk = c;
    geom = g;
  }
  std::vector<T> mirrored() const {
    if (chunk && geom >= 0) {
      std::vector<double> out(size);
      if (cb_read_geom(chunk, geom, out.data(), size) != 0) b200_fatal("Buffer1D::mirrored");
      return std::vector<T>(out.begin(), out.end());
    }
    return *host;
  }
};

template <typename T> struct Buffer2D {
  size_t sizeX, sizeY;
  cb_chunk *chunk = nullptr;
  int field = -1;

  Buffer2D(context &, size_t sizeX, size_t sizeY) : sizeX(sizeX), sizeY(sizeY) {}
  template <size_t D> [[nodiscard]] size_t extent() const {
    if constexpr (D == 0) {
      return sizeX;
    } else if (D == 1) {
      return sizeY;
    } else {
      static_assert(D < 2);
      return 0;
    }
  }
  void bind(cb_chunk *c, int f) {
    chunk = c;
    field = f;
  }
  // The reference Buffer2D order, data[j + i * sizeY] (src/serial/context.h:73).
  std::vector<T> mirrored() const {
    std::vector<double> out(sizeX * sizeY, 0.0);
    if (chunk && field >= 0 && cb_read_field(chunk, field, out.data(), out.size(), CB_LAYOUT_YFAST) != 0)
      b200_fatal("Buffer2D::mirrored");
    return std::vector<T>(out.begin(), out.end());
  }
  clover::BufferMirror2D<T> mirrored2() { return {mirrored(), extent<0>(), extent<1>()}; }
};

template <typename T> using StagingBuffer1D = Buffer1D<T> &;

} // namespace clover

using clover::Range1d;
using clover::Range2d;
