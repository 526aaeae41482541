// initialise.cpp -- create_context / report_context (driver/initialise.h:160-162)
// for the b200 model: lists the CUDA devices and selects one with --device,
// as the reference CUDA model does (src/cuda/initialise.cpp:25-45).
//
// Model settings come from the environment (the driver's command line and
// deck reader are unchanged and reject / ignore unknown options):
//   CLOVER_B200_PRECISION = fp64 (default) | fp32  storage form
//   CLOVER_B200_FOLD      = 1 (default) | 0        fold update_halo into producers
//   CLOVER_B200_FUSE      = 1 (default) | 0        the driver's phase calls as fused passes
//                                                  (with folding; results unchanged)
//   CLOVER_B200_AHEAD     = 1 (default) | 0        with fused calls: calc_dt runs the
//                                                  Lagrangian pass ahead (not with --dump)
#include "initialise.h"
#include "b200_runtime.h"

#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

model create_context(bool silent, const std::vector<std::string> &args) {
  int count = 0;
  if (cb_device_count(&count) != 0 || count == 0) {
    std::cerr << "b200 model: no CUDA device: " << cb_last_error() << std::endl;
    std::exit(EXIT_FAILURE);
  }
  std::vector<int> devices;
  for (int d = 0; d < count; ++d) devices.push_back(d);
  auto [device, parsed] = list_and_parse<int>(
      silent, devices,
      [](const int &d) {
        char name[256] = {0};
        if (cb_device_name(d, name, sizeof name) != 0) return std::string("CUDA device ") + std::to_string(d);
        return std::string(name);
      },
      args);
  clover::context ctx;
  ctx.device = device;
  ctx.rt = std::make_shared<clover::Runtime>();
  if (const char *p = std::getenv("CLOVER_B200_PRECISION")) {
    if (std::strcmp(p, "fp32") == 0) ctx.precision = CB_FP32;
    else if (std::strcmp(p, "fp64") == 0) ctx.precision = CB_FP64;
    else {
      std::cerr << "b200 model: CLOVER_B200_PRECISION must be fp64 or fp32, got " << p << std::endl;
      std::exit(EXIT_FAILURE);
    }
  }
  if (const char *f = std::getenv("CLOVER_B200_FOLD")) ctx.rt->fold = std::strcmp(f, "0") != 0;
  if (const char *f = std::getenv("CLOVER_B200_FUSE")) ctx.rt->fuse = std::strcmp(f, "0") != 0;
  if (const char *f = std::getenv("CLOVER_B200_AHEAD")) ctx.rt->ahead = std::strcmp(f, "0") != 0;
  return {ctx, "B200 (sm_100a CUDA, libcloverb200)", true, parsed};
}

void report_context(const clover::context &ctx) {
  char name[256] = {0};
  cb_device_name(ctx.device, name, sizeof name);
  std::cout << " - Device:    " << name << "\n"
            << " - Precision: " << (ctx.precision == CB_FP64 ? "fp64" : "fp32") << "\n"
            << " - Halo fold: " << (ctx.rt && ctx.rt->fold ? "on" : "off") << "\n"
            << " - Fused calls: " << (ctx.rt && ctx.rt->fold && ctx.rt->fuse ? "on" : "off")
            << ", Lagrangian pass ahead of its calls: " << (ctx.rt && ctx.rt->fold && ctx.rt->fuse && ctx.rt->ahead ? "on" : "off")
            << std::endl;
}
