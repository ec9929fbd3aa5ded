// Allocation-free exact Stieltjes sums at query points.
//
// Every other entry point of the library keeps its device temporaries in
// per-device scratch slots that grow on demand: a call larger than any before
// it frees the old slot and allocates a bigger one.  Some callers cannot let a
// library do that:
//   * hosts whose framework has reserved (nearly) all device memory for its
//     own pool -- JAX preallocates most of the GPU by default, and a PyTorch
//     process under memory pressure holds its cache -- so a library
//     allocation can fail at an arbitrary point of their loop;
//   * latency-bound loops, because freeing device memory synchronises the
//     whole device and stalls the caller's other streams;
//   * long-running services that forbid allocations after start-up so that
//     device memory use stays fixed and fragmentation cannot build up.
// shrk_stieltjes_at_points_noalloc serves them.  It computes the same raw
// sums as shrk_stieltjes_at_points_dev with an exact method (FP64 or MIXED
// arithmetic), and takes all its temporaries from one file-scope device array
// of SHRK_NOALLOC_SCRATCH_BYTES that the CUDA runtime reserves when it loads
// this module.  The call never allocates and never frees.
//
// Layout of the array: [0, 256) the device error word, then the per-256-block
// source bounds of the MIXED kernel (up to SHRK_NOALLOC_MAX_EIGS eigenvalues),
// then the (re, im) split partials (at least SHRK_NOALLOC_MAX_POINTS query
// points).  Each call fully overwrites the bounds and the partials it reads;
// only the error word must start at zero, and each call clears it first.
#include "common.cuh"
#include "internal.h"

#include <cmath>
#include <mutex>
#include <string>

namespace shrk {
namespace {

constexpr size_t kScratchBytes = SHRK_NOALLOC_SCRATCH_BYTES;
constexpr size_t kErrBytes = 256;
constexpr size_t kBoundsEntries = (size_t)SHRK_NOALLOC_MAX_EIGS / 256 + 2;
constexpr size_t kBoundsBytes = (kBoundsEntries * sizeof(double2) + 255) / 256 * 256;
constexpr size_t kPartOffset = kErrBytes + kBoundsBytes;
constexpr int64_t kPartCapacity = (int64_t)((kScratchBytes - kPartOffset) / (2 * sizeof(double)));
static_assert(kPartCapacity >= (int64_t)SHRK_NOALLOC_MAX_POINTS,
              "static scratch too small for one split of the largest query set");

constexpr int kMaxDevices = 64;

}  // namespace

// Shared by every call on a device; contents persist from call to call.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

namespace {

struct FixedScratch {
  char* base = nullptr;  // device address of g_noalloc_scratch on that device
  int sms = 0;
};
std::mutex g_setup_mu;
FixedScratch g_fixed[kMaxDevices];

// Once per device, with that device current: look up the array's device
// address (this is also when the runtime loads the module onto the device if
// nothing has loaded it yet) and the multiprocessor count.
shrk_status fixed_scratch(int dev, FixedScratch* out) {
  std::lock_guard<std::mutex> lk(g_setup_mu);
  FixedScratch& f = g_fixed[dev];
  if (!f.base) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(g_noalloc_scratch)");
    int sms = 0;
    e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return cuda_fail(e, "cudaDeviceGetAttribute(multiprocessors)");
    f.sms = sms;
    f.base = (char*)p;
  }
  *out = f;
  return SHRK_OK;
}

shrk_status invalid(const std::string& msg) {
  set_error(msg);
  return SHRK_EINVAL;
}

}  // namespace
}  // namespace shrk

extern "C" shrk_status shrk_stieltjes_at_points_noalloc(const double* d_q, size_t nq,
                                                        const double* d_ev, size_t p, double eta,
                                                        int precision, double* d_re, double* d_im,
                                                        void* stream) {
  using namespace shrk;
  if (p == 0) return invalid("eigenvalues must be non-empty");
  if (!(std::isfinite(eta) && eta > 0.0)) return invalid("eta must be a positive finite number");
  if (precision != SHRK_PREC_F64 && precision != SHRK_PREC_MIXED)
    return invalid("precision must be SHRK_PREC_F64 or SHRK_PREC_MIXED");
  if (nq > (size_t)SHRK_NOALLOC_MAX_POINTS)
    return invalid("shrk_stieltjes_at_points_noalloc: " + std::to_string(nq) +
                   " query points exceed the static scratch limit of " +
                   std::to_string((long long)SHRK_NOALLOC_MAX_POINTS) +
                   "; split the query set or use shrk_stieltjes_at_points_dev");
  if (p > (size_t)SHRK_NOALLOC_MAX_EIGS)
    return invalid("shrk_stieltjes_at_points_noalloc: " + std::to_string(p) +
                   " eigenvalues exceed the static scratch limit of " +
                   std::to_string((long long)SHRK_NOALLOC_MAX_EIGS) +
                   "; use shrk_stieltjes_at_points_dev");
  if (nq == 0) return SHRK_OK;
  if (!d_q || !d_ev || !d_re || !d_im) return invalid("null device pointer");
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return cuda_fail(e, "cudaGetDevice");
  if (dev < 0 || dev >= kMaxDevices) return invalid("device ordinal out of range");
  FixedScratch f;
  SHRK_TRY(fixed_scratch(dev, &f));
  cudaStream_t s = (cudaStream_t)stream;  // null = the legacy default stream
  int* err = (int*)f.base;
  double2* bounds = (double2*)(f.base + kErrBytes);
  double* part = (double*)(f.base + kPartOffset);
  SHRK_CUDA(cudaMemsetAsync(err, 0, sizeof(int), s));
  return exact_pair_sums_fixed(d_q, (int64_t)nq, d_ev, (int64_t)p, eta, precision, d_re, d_im,
                               part, kPartCapacity, bounds, err, f.sms, s);
}
