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


}  // namespace shrk
