// Pipe-rate probes: measured FP32 and FP64 FMA lane-op rates of the current
// device, the denominators of the exact kernels' roofline fractions; and the
// mean error of the MUFU reciprocal that the mixed kernel corrects for.  Each
// thread runs independent dependency chains of FMAs whose operands stay in
// registers, sized so that issue (not latency) limits the rate.
#include "common.cuh"
#include "internal.h"

#include <vector>

namespace shrk {
namespace {

template <typename T>
__global__ void __launch_bounds__(256) fma_rate_kernel(int iters, T a, T b, T* sink) {
  T x0 = (T)threadIdx.x, x1 = x0 + (T)1, x2 = x0 + (T)2, x3 = x0 + (T)3;
  T x4 = x0 + (T)4, x5 = x0 + (T)5, x6 = x0 + (T)6, x7 = x0 + (T)7;
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int k = 0; k < 16; ++k) {
      x0 = fma(x0, a, b); x1 = fma(x1, a, b); x2 = fma(x2, a, b); x3 = fma(x3, a, b);
      x4 = fma(x4, a, b); x5 = fma(x5, a, b); x6 = fma(x6, a, b); x7 = fma(x7, a, b);
    }
  }
  T s = ((x0 + x1) + (x2 + x3)) + ((x4 + x5) + (x6 + x7));
  if (s == (T)-1.2345) sink[0] = s;  // never true; keeps the chains live
}

template <typename T>
shrk_status rate(double* out, cudaStream_t s) {
  const int blocks = sm_count() * 8, iters = 4096;
  void* sink = nullptr;
  SHRK_TRY(scratch_get(15, 64, &sink));
  cudaEvent_t e0, e1;
  SHRK_CUDA(cudaEventCreate(&e0));
  SHRK_CUDA(cudaEventCreate(&e1));
  fma_rate_kernel<T><<<blocks, 256, 0, s>>>(64, (T)0.999, (T)0.001, (T*)sink);  // warm-up
  SHRK_CUDA(cudaEventRecord(e0, s));
  fma_rate_kernel<T><<<blocks, 256, 0, s>>>(iters, (T)0.999, (T)0.001, (T*)sink);
  SHRK_CUDA(cudaEventRecord(e1, s));
  SHRK_CUDA(cudaEventSynchronize(e1));
  float ms = 0.f;
  SHRK_CUDA(cudaEventElapsedTime(&ms, e0, e1));
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  const double ops = (double)blocks * 256.0 * iters * 16.0 * 8.0;  // FMA lane-ops
  *out = ops / (ms * 1e-3);
  return SHRK_OK;
}

// Relative error of the MUFU reciprocal over every mantissa of [1, 2):
// a = 1 + k 2^-23, rel = r a - 1 (the product of two floats is exact in
// FP64).  Per block: the plain sum of rel, the sum of rel / a and the sum of
// 1 / a (the log-uniform weight), reduced in a fixed order.
constexpr int BIAS_PER = 16, BIAS_NT = 256, BIAS_BLOCKS = (1 << 23) / (BIAS_NT * BIAS_PER);

__global__ void __launch_bounds__(BIAS_NT) rcp_bias_kernel(double* part) {
  __shared__ double red[3][BIAS_NT];
  double su = 0.0, sl = 0.0, wl = 0.0;
  for (int i = 0; i < BIAS_PER; ++i) {
    const uint32_t k = (uint32_t)(blockIdx.x * BIAS_NT + threadIdx.x) * BIAS_PER + i;
    const float a = __uint_as_float(0x3F800000u | k);
    const float r = -rcp_f32(-a);  // the negated form the pair kernel uses
    const double rel = (double)r * (double)a - 1.0;
    su += rel;
    sl += rel / (double)a;
    wl += 1.0 / (double)a;
  }
  red[0][threadIdx.x] = su;
  red[1][threadIdx.x] = sl;
  red[2][threadIdx.x] = wl;
  __syncthreads();
  for (int h = BIAS_NT / 2; h > 0; h >>= 1) {
    if ((int)threadIdx.x < h)
      for (int c = 0; c < 3; ++c) red[c][threadIdx.x] += red[c][threadIdx.x + h];
    __syncthreads();
  }
  if (threadIdx.x < 3) part[blockIdx.x * 3 + threadIdx.x] = red[threadIdx.x][0];
}

}  // namespace

shrk_status measure_rcp_bias(double* uniform_mean, double* log_mean) {
  cudaStream_t s = library_stream();
  void* part = nullptr;
  SHRK_TRY(scratch_get(15, (size_t)BIAS_BLOCKS * 3 * sizeof(double), &part));
  rcp_bias_kernel<<<BIAS_BLOCKS, BIAS_NT, 0, s>>>((double*)part);
  SHRK_CUDA(cudaGetLastError());
  std::vector<double> h((size_t)BIAS_BLOCKS * 3);
  SHRK_CUDA(cudaMemcpyAsync(h.data(), part, h.size() * sizeof(double), cudaMemcpyDeviceToHost, s));
  SHRK_CUDA(cudaStreamSynchronize(s));
  double su = 0.0, sl = 0.0, wl = 0.0;
  for (int b = 0; b < BIAS_BLOCKS; ++b) {
    su += h[b * 3];
    sl += h[b * 3 + 1];
    wl += h[b * 3 + 2];
  }
  *uniform_mean = su / (double)(1 << 23);
  *log_mean = sl / wl;
  return SHRK_OK;
}

shrk_status measure_pipe_rates(double* fp32, double* fp64) {
  cudaStream_t s = library_stream();
  SHRK_TRY(rate<float>(fp32, s));
  SHRK_TRY(rate<double>(fp64, s));
  return SHRK_OK;
}

}  // namespace shrk
