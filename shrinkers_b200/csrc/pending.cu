// Entry points whose kernels are not written yet: they fail loudly with
// SHRK_ENOTIMPL (there is no CPU fallback).  Each is replaced by its own
// kernel file as it lands.
#include "common.cuh"
#include "internal.h"

namespace shrk {

static shrk_status pending(const char* what) {
  set_error(std::string(what) + " is not implemented on the GPU yet");
  return SHRK_ENOTIMPL;
}

shrk_status batched(const double*, const int64_t*, const int64_t*, int64_t, const double*, int,
                    double*, double*, cudaStream_t) {
  return pending("batched transform");
}

shrk_status nufft_points(const double*, int64_t, const double*, int64_t, double, double, double,
                         double*, double*, cudaStream_t) {
  return pending("nufft");
}
size_t nufft_grid_size(double, double) { return 0; }

bool cheb_preset(int method, ChebParams* out) {
  switch (method) {
    case SHRK_M_CHEBCODE: *out = {0.5, 11, 32, false}; return true;
    case SHRK_M_CHEBCODE_FAST: *out = {1.0, 8, 32, true}; return true;
    case SHRK_M_CHEBCODE_XTREME: *out = {0.25, 11, 16, false}; return true;
    case SHRK_M_CHEBCODE_BALANCED: *out = {0.55, 11, 32, false}; return true;
    default: return false;
  }
}
size_t grid_leaf_cap(size_t, size_t, size_t, size_t preset_leaf) { return preset_leaf; }
shrk_status chebcode_points(const double*, int64_t, const double*, const double*, int64_t, double,
                            const ChebParams&, double*, double*, cudaStream_t) {
  return pending("chebcode");
}

}  // namespace shrk
