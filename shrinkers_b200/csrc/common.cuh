// Shared internals of libshrinkers_b200: error state, per-device scratch,
// kernel timing, and the sm_100a primitives used by every kernel
// (mbarrier + bulk-copy staging with bounded waits, reciprocals).
#pragma once

#include <cuda_runtime.h>
#include <cstdint>
#include <cstddef>
#include <string>
#include <vector>

#include "../../include/shrinkers_b200.h"

namespace shrk {

// ----------------------------------------------------------- host side --
void set_error(const std::string& msg);
shrk_status cuda_fail(cudaError_t e, const char* what);

#define SHRK_CUDA(call)                                  \
  do {                                                   \
    cudaError_t _e = (call);                             \
    if (_e != cudaSuccess) return cuda_fail(_e, #call);  \
  } while (0)

#define SHRK_TRY(call)                        \
  do {                                        \
    shrk_status _s = (call);                  \
    if (_s != SHRK_OK) return _s;             \
  } while (0)

// Grow-only device scratch owned by the library (one set per device).
struct Scratch {
  void* ptr = nullptr;
  size_t bytes = 0;
};
shrk_status scratch_get(int slot, size_t bytes, void** out);  // slot in [0, 64)
// Per-context module state: the object in slot k (a CtxExt) of the running
// call's context, made by `make` on first use and deleted by `del` when the
// context is released.  Contexts are never shared by concurrent calls.
enum CtxExt : int { EXT_FFT_TABLES = 0, EXT_BATCHED_GRAPH = 1 };
void* ctx_ext(int k, void* (*make)(), void (*del)(void*));
template <typename T>
T& ctx_state(int k) {
  return *static_cast<T*>(
      ctx_ext(k, []() -> void* { return new T(); }, [](void* q) { delete static_cast<T*>(q); }));
}
int* device_error_word();  // the running call's context; cleared when a host call reads it

// Host-side facts about a source array a host-pointer entry point has just
// uploaded (sortedness, first and last entry in the caller's order), so the
// methods that need sorted sources skip the device check and its read-back.
// Valid for the running call only (cleared when a host-pointer call enters).
void set_source_hint(const double* d_src, const double* h_src, int64_t n);
// lo / hi (optional): the smallest and largest entry.  NaN input makes the
// array unsorted (the comparison v[i-1] <= v[i] fails), as on the device.
bool source_hint(const double* d_src, int64_t n, bool* sorted, double* first, double* last,
                 double* lo = nullptr, double* hi = nullptr);
int sm_count();
cudaStream_t library_stream();

// Kernel launch bookkeeping (launch count, optional CUDA-event timing).
struct LaunchScope {
  LaunchScope(const char* family, cudaStream_t s);
  ~LaunchScope();
  const char* family;
  cudaStream_t stream;
  cudaEvent_t start = nullptr, stop = nullptr;
};

// Adds kernels launched outside a LaunchScope (inside a CUDA graph) to the
// library's launch count.
void add_launches(int64_t n);

// Read back and clear the device error word; maps a set word to a status.
shrk_status check_device_error(cudaStream_t s);

// ------------------------------------------------------- device side --
enum DeviceError : int {
  DEV_ERR_NONE = 0,
  DEV_ERR_TIMEOUT = 1,   // an mbarrier / queue wait ran out of iterations
  DEV_ERR_BOUNDS = 2,    // a self-check found an index out of range
};

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count)
               : "memory");
}

__device__ __forceinline__ void fence_mbar_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void fence_proxy_async() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile(
      "{ .reg .b64 st; mbarrier.arrive.expect_tx.shared::cta.b64 st, [%0], %1; }" ::"r"(
          smem_u32(bar)),
      "r"(bytes)
      : "memory");
}

// One-dimensional TMA bulk copy global -> shared, completing on `bar`.
// Both addresses 16-byte aligned, bytes a multiple of 16.  No multicast.
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes,
                                         uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::
          "r"(smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}

// Default budget of a bounded wait: 2e9 clock cycles, about a second.
constexpr long long WAIT_CYCLES_DEFAULT = 2000000000LL;

// Bounded wait on an mbarrier phase: gives up after `max_cycles` clock
// cycles (about a second at the default limit) and returns false.  A budget
// of zero or less gives up at once without looking at the barrier (the
// failure path's test setting).
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity,
                                          long long max_cycles = WAIT_CYCLES_DEFAULT) {
  if (max_cycles <= 0) return false;
  const uint32_t addr = smem_u32(bar);
  const long long t0 = clock64();
  while (true) {
    uint32_t done;
    asm volatile(
        "{ .reg .pred p; mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2; selp.u32 %0, 1, 0, "
        "p; }"
        : "=r"(done)
        : "r"(addr), "r"(parity)
        : "memory");
    if (done) return true;
    if (clock64() - t0 > max_cycles) return false;
  }
}

// FP64 reciprocal: hardware seed (rcp.approx.ftz.f64) refined by one
// third-order Newton-Raphson step r' = r + r (e + e^2), e = 1 - a r
// (error ~ e^3, i.e. below one ulp from a 2^-22 seed).  a must be a
// normal positive number (the pair denominators are >= eta^2).
__device__ __forceinline__ double rcp_f64(double a) {
  double r;
  asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(r) : "d"(a));
  double e = fma(-a, r, 1.0);
  e = fma(e, e, e);
  return fma(r, e, r);
}

// FP32 reciprocal on the MUFU pipe (rcp.approx.ftz.f32, <= 1 ulp).
__device__ __forceinline__ float rcp_f32(float a) {
  float r;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(a));
  return r;
}

// Error-free transformation s + e = a + b (Knuth TwoSum, six FP32 adds).
__device__ __forceinline__ void two_sum_acc(float& hi, float& lo, float b) {
  float s = hi + b;
  float bb = s - hi;
  float e = (hi - (s - bb)) + (b - bb);
  hi = s;
  lo += e;
}

}  // namespace shrk
