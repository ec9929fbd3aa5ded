// Smaller exact kernels: the value+derivative sum (src/stieltjes/autovec.rs:
// 38-77), the f32 full-square kernel (src/stieltjes/cacheblock.rs:1525-1572),
// the windowed cutoff sums (cacheblock.rs:452-577) and the scaled-ray sums of
// inverse nonlinear shrinkage (src/stieltjes/mod.rs:304-319).  The forward
// pair-sum kernels live in pairsum.cu, the adjoint in adjoint.cu.
#include "common.cuh"
#include "internal.h"
#include "pairs.cuh"

#include <algorithm>
#include <cmath>

namespace shrk {

namespace {

// --------------------------------------------------------------- E7 ----
// autovec.rs:38-59: value + derivative.  One target per thread, sources
// through shared memory tiles.
__global__ void __launch_bounds__(256) deriv_kernel(const double* __restrict__ ev, int64_t p,
                                                    double eta, double* re_o, double* im_o,
                                                    double* dre_o, double* dim_o) {
  __shared__ double tile[1024];
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const double x = ev[min(t, p - 1)];
  const double eta2 = eta * eta;
  double s_re = 0.0, s_inv = 0.0, d_re = 0.0, d_im = 0.0;
  for (int64_t j0 = 0; j0 < p; j0 += 1024) {
    const int len = (int)min((int64_t)1024, p - j0);
    __syncthreads();
    for (int i = threadIdx.x; i < len; i += blockDim.x) tile[i] = ev[j0 + i];
    __syncthreads();
    for (int j = 0; j < len; ++j) {
      const double d = x - tile[j];
      const double den = d * d + eta2;
      const double inv = rcp_f64(den);
      s_re = s_re + d * inv;
      s_inv = s_inv + inv;
      d_re = d_re - (d * d - eta2) * inv * inv;
      d_im = d_im - (2.0 * d * eta) * inv * inv;
    }
  }
  if (t < p) {
    re_o[t] = s_re;
    im_o[t] = eta * s_inv;
    dre_o[t] = d_re;
    dim_o[t] = d_im;
  }
}

// --------------------------------------------------------------- E6 ----
// cacheblock.rs:1525-1572 + mod.rs:805-848: FP32 full square, fused f32
// mul_add, IEEE f32 reciprocal, 1/p applied in f32.
__global__ void __launch_bounds__(256) f32_kernel(const float* __restrict__ ev, int64_t p,
                                                  float eta, float* re_o, float* im_o) {
  __shared__ float tile[2048];
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const float x = ev[min(t, p - 1)];
  const float eta2 = eta * eta;
  float r = 0.0f, s = 0.0f;
  for (int64_t j0 = 0; j0 < p; j0 += 2048) {
    const int len = (int)min((int64_t)2048, p - j0);
    __syncthreads();
    for (int i = threadIdx.x; i < len; i += blockDim.x) tile[i] = ev[j0 + i];
    __syncthreads();
    for (int j = 0; j < len; ++j) {
      const float d = x - tile[j];
      const float inv = __frcp_rn(fmaf(d, d, eta2));
      r = fmaf(d, inv, r);
      s = fmaf(eta, inv, s);
    }
  }
  if (t < p) {
    const float inv_p = 1.0f / (float)p;
    re_o[t] = r * inv_p;
    im_o[t] = s * inv_p;
  }
}

// --------------------------------------------------------------- E5 ----
// cacheblock.rs:531-577 windowed sum per target: binary-searched window of
// sorted sources within +-window, fused accumulation as in the reference.
__global__ void windowed_kernel(const double* __restrict__ tgt, int64_t nt,
                                const double* __restrict__ src, int64_t ns, double eta,
                                double window, double scale, double* re_o, double* im_o) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nt) return;
  const double x = tgt[t], eta2 = eta * eta;
  const double lo_v = x - window, hi_v = x + window;
  int64_t lo = 0, hi = ns;  // first index with src >= lo_v
  while (lo < hi) {
    const int64_t mid = (lo + hi) >> 1;
    if (src[mid] < lo_v) lo = mid + 1;
    else hi = mid;
  }
  const int64_t first = lo;
  lo = first;
  hi = ns;  // first index with src > hi_v
  while (lo < hi) {
    const int64_t mid = (lo + hi) >> 1;
    if (src[mid] <= hi_v) lo = mid + 1;
    else hi = mid;
  }
  double sr = 0.0, si = 0.0;
  for (int64_t j = first; j < lo; ++j) {
    const double d = x - src[j];
    const double inv = rcp_f64(fma(d, d, eta2));
    sr = fma(d, inv, sr);
    si = fma(eta, inv, si);
  }
  re_o[t] = sr * scale;
  im_o[t] = si * scale;
}

// ------------------------------------------------------ scaled ray ----
// mod.rs:304-319 compute_stieltjes_scaled_ray: RAW sums at z_t = x_t (1 + i h),
// i.e. every target has its own eta_t = h x_t.  FP64 pairs; a CTA of 256
// threads holds 4 targets per thread (and their eta^2), source chunks of
// 1024 are staged in shared memory; source splits write partial slabs that
// ray_reduce_kernel adds in a fixed order.
constexpr int RAY_NT = 256, RAY_R = 4, RAY_CH = 1024;

__global__ void __launch_bounds__(RAY_NT, 2) ray_kernel(const double* __restrict__ ev, int64_t p,
                                                       double scale, int64_t n_tiles,
                                                       int n_splits, int64_t split_len,
                                                       double* part_re, double* part_im) {
  __shared__ double sb[RAY_CH];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int64_t n_items = n_tiles * n_splits;
  for (int64_t item = blockIdx.x; item < n_items; item += gridDim.x) {
    const int64_t tile = item / n_splits;
    const int split = (int)(item % n_splits);
    const int64_t wbase = tile * RAY_NT * RAY_R + (int64_t)warp * 32 * RAY_R;
    double x[RAY_R], eta2[RAY_R], re[RAY_R], iv[RAY_R];
#pragma unroll
    for (int r = 0; r < RAY_R; ++r) {
      const int64_t idx = wbase + r * 32 + lane;
      x[r] = idx < p ? ev[idx] : ev[0];
      const double eta = scale * x[r];
      eta2[r] = eta * eta;
      re[r] = iv[r] = 0.0;
    }
    const int64_t s0 = (int64_t)split * split_len, s1 = min(p, s0 + split_len);
    for (int64_t cs = s0; cs < s1; cs += RAY_CH) {
      const int len = (int)min((int64_t)RAY_CH, s1 - cs);
      __syncthreads();
      for (int i = threadIdx.x; i < len; i += RAY_NT) sb[i] = ev[cs + i];
      __syncthreads();
#pragma unroll 4
      for (int j = 0; j < len; ++j) {
        const double l = sb[j];
#pragma unroll
        for (int r = 0; r < RAY_R; ++r) {
          const double d = x[r] - l;
          const double inv = rcp_f64(fma(d, d, eta2[r]));
          re[r] = fma(d, inv, re[r]);
          iv[r] += inv;
        }
      }
    }
#pragma unroll
    for (int r = 0; r < RAY_R; ++r) {
      const int64_t idx = wbase + r * 32 + lane;
      if (idx < p) {
        part_re[(int64_t)split * p + idx] = re[r];
        part_im[(int64_t)split * p + idx] = scale * x[r] * iv[r];
      }
    }
  }
}

__global__ void ray_reduce_kernel(const double* __restrict__ part_re,
                                  const double* __restrict__ part_im, int n_splits, int64_t p,
                                  double* out_re, double* out_im) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= p) return;
  double re = 0.0, im = 0.0;
  for (int k = 0; k < n_splits; ++k) {
    re += part_re[(int64_t)k * p + t];
    im += part_im[(int64_t)k * p + t];
  }
  out_re[t] = re;
  out_im[t] = im;
}

}  // namespace

shrk_status scaled_ray_sums(const double* d_ev, int64_t p, double scale, double* d_re,
                            double* d_im, cudaStream_t s) {
  if (p <= 0) return SHRK_OK;
  const SplitPlan pl = plan_splits(p, p, RAY_NT * RAY_R, RAY_CH, 2);
  void* part = nullptr;
  SHRK_TRY(scratch_get(0, sizeof(double) * 2 * (size_t)pl.n_splits * (size_t)p, &part));
  double* pre = (double*)part;
  double* pim = pre + (size_t)pl.n_splits * p;
  {
    LaunchScope ls("scaled_ray", s);
    ray_kernel<<<pl.grid, RAY_NT, 0, s>>>(d_ev, p, scale, pl.n_tiles, pl.n_splits, pl.split_len,
                                          pre, pim);
    SHRK_CUDA(cudaGetLastError());
  }
  LaunchScope ls("split_reduce", s);
  ray_reduce_kernel<<<(unsigned)((p + 255) / 256), 256, 0, s>>>(pre, pim, pl.n_splits, p, d_re,
                                                                d_im);
  SHRK_CUDA(cudaGetLastError());
  return SHRK_OK;
}

shrk_status windowed_sums(const double* d_tgt, int64_t nt, const double* d_src, int64_t ns,
                          double eta, double window, double scale, double* d_re, double* d_im,
                          cudaStream_t s) {
  if (nt <= 0) return SHRK_OK;
  LaunchScope ls("windowed", s);
  windowed_kernel<<<(unsigned)((nt + 255) / 256), 256, 0, s>>>(d_tgt, nt, d_src, ns, eta, window,
                                                               scale, d_re, d_im);
  SHRK_CUDA(cudaGetLastError());
  return SHRK_OK;
}

shrk_status with_deriv(const double* d_ev, int64_t p, double eta, double* d_re, double* d_im,
                       double* d_dre, double* d_dim, cudaStream_t s) {
  if (p <= 0) return SHRK_OK;
  LaunchScope ls("with_deriv", s);
  deriv_kernel<<<(unsigned)((p + 255) / 256), 256, 0, s>>>(d_ev, p, eta, d_re, d_im, d_dre, d_dim);
  SHRK_CUDA(cudaGetLastError());
  return SHRK_OK;
}

shrk_status all_f32(const float* d_ev, int64_t p, float eta, float* d_re, float* d_im,
                    cudaStream_t s) {
  if (p <= 0) return SHRK_OK;
  LaunchScope ls("all_f32", s);
  f32_kernel<<<(unsigned)((p + 255) / 256), 256, 0, s>>>(d_ev, p, eta, d_re, d_im);
  SHRK_CUDA(cudaGetLastError());
  return SHRK_OK;
}

}  // namespace shrk
