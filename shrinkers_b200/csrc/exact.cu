// Smaller exact kernels: the value+derivative sum (src/stieltjes/autovec.rs:
// 38-77), the f32 full-square kernel (src/stieltjes/cacheblock.rs:1525-1572),
// the windowed cutoff sums (cacheblock.rs:452-577) and the adjoint of the
// all-points transform (no reference counterpart).  The forward pair-sum
// kernels live in pairsum.cu.
#include "common.cuh"
#include "internal.h"
#include "pairs.cuh"

#include <algorithm>
#include <cmath>

namespace shrk {

namespace {

constexpr int NT = 256;
constexpr int R = 4;             // targets per thread (adjoint)
constexpr int TT = NT * R;
constexpr int WT = 32 * R;
constexpr int ACH = 512;         // sources per staged adjoint chunk
constexpr int FOLD = 16;

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

// ------------------------------------------------------------ adjoint ----
// dL/dev_k = (1/p) sum_j [ (w_k - w_j)(a^2 - eta^2) - (v_k + v_j) 2 a eta ] / (a^2+eta^2)^2,
// a = ev_k - ev_j, for L = sum_j (w_j Re m_j + v_j Im m_j) with
// m_j = (1/p) sum_i 1/(ev_i - ev_j - i eta).  Four source sums per target:
//   A1 = sum (a^2-eta^2)/D^2, A2 = sum w_j (a^2-eta^2)/D^2,
//   B1 = sum 2 a eta/D^2,     B2 = sum v_j 2 a eta/D^2.
// Pairs are recomputed, never stored; sources (ev, w, v) stream through
// shared memory.  MIXED: far pairs in FP32 (split separation, unbiased
// reciprocal, FP32 partials folded into FP64), near pairs in FP64.
struct AdjArgs {
  const double* ev;
  const double* w;
  const double* v;
  int64_t p;
  const double2* bounds;
  const double2* gminmax;
  double eta;
  double near_dist;
  int64_t n_tiles;
  int n_splits;
  int64_t split_len;
  double* part;  // [n_splits][4][p]
};

template <bool MIXED>
__global__ void __launch_bounds__(NT, 2) adjoint_kernel(const AdjArgs a) {
  __shared__ __align__(16) double sl[ACH], sw[ACH], sv[ACH];
  __shared__ __align__(16) float fmu[MIXED ? ACH : 4], fml[MIXED ? ACH : 4];
  __shared__ __align__(16) float fw[MIXED ? ACH : 4], fv[MIXED ? ACH : 4];
  __shared__ double red[NT / 32];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const double eta = a.eta, eta2 = eta * eta, teta = 2.0 * eta;
  const float eta2f = (float)eta2, tetaf = (float)teta;
  const int64_t n_items = a.n_tiles * (int64_t)a.n_splits;
  for (int64_t item = blockIdx.x; item < n_items; item += gridDim.x) {
    const int64_t tile = item / a.n_splits;
    const int split = (int)(item % a.n_splits);
    const int64_t tile0 = tile * TT, wbase = tile0 + (int64_t)warp * WT;
    const double x0 = a.ev[tile0];
    double x[R];
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const int64_t idx = wbase + r * 32 + lane;
      x[r] = idx < a.p ? a.ev[idx] : x0;
    }
    double acc[R][4];
    float xh[R], xl[R];
#pragma unroll
    for (int r = 0; r < R; ++r) {
#pragma unroll
      for (int q = 0; q < 4; ++q) acc[r][q] = 0.0;
      xh[r] = xl[r] = 0.0f;
    }
    const double c = x0;
    double wlo = 0, whi = 0, thr = INFINITY;
    if (MIXED) {
      double spread = 0.0, mn = x[0], mx = x[0];
#pragma unroll
      for (int r = 0; r < R; ++r) {
        spread = fmax(spread, fabs(x[r] - c));
        mn = fmin(mn, x[r]);
        mx = fmax(mx, x[r]);
      }
      wlo = warp_min(mn);
      whi = warp_max(mx);
      spread = warp_max(spread);
      if (lane == 0) red[warp] = spread;
      __syncthreads();
      double wd = 0.0;
      for (int i = 0; i < NT / 32; ++i) wd = fmax(wd, red[i]);
      const double2 g = *a.gminmax;
      const double u = snap_unit(fmax(fmax(g.y - c, c - g.x), wd));
      thr = (wd < 0x1p22 * u) ? fmax(a.near_dist, wd) : INFINITY;
#pragma unroll
      for (int r = 0; r < R; ++r) split_target(x[r], c, u, xh[r], xl[r]);
    }
    const int64_t s0 = (int64_t)split * a.split_len, s1 = min(a.p, s0 + a.split_len);
    for (int64_t cs = s0; cs < s1; cs += ACH) {
      const int len = (int)min((int64_t)ACH, s1 - cs);
      __syncthreads();
      for (int i = tid; i < len; i += NT) {
        sl[i] = a.ev[cs + i];
        sw[i] = a.w[cs + i];
        sv[i] = a.v[cs + i];
        if (MIXED) {
          split_source(sl[i], c, fmu[i], fml[i]);
          fw[i] = (float)sw[i];
          fv[i] = (float)sv[i];
        }
      }
      __syncthreads();
      for (int sub = 0; sub < len; sub += SUB) {
        const int slen = min(SUB, len - sub);
        bool far32 = false;
        if (MIXED && slen == SUB) {
          const double2 bd = a.bounds[(cs + sub) / SUB];
          const double gap = fmax(fmax(bd.x - whi, wlo - bd.y), 0.0);
          const double span = fmax(bd.y - wlo, whi - bd.x);
          far32 = gap >= thr && span <= 1e9;
        }
        if (MIXED && far32) {
          for (int j = sub; j < sub + SUB; j += FOLD) {
            float pp[R][4];
#pragma unroll
            for (int r = 0; r < R; ++r)
#pragma unroll
              for (int q = 0; q < 4; ++q) pp[r][q] = 0.0f;
#pragma unroll 4
            for (int jj = j; jj < j + FOLD; ++jj) {
              const float mh = fmu[jj], ml = fml[jj], wj = fw[jj], vj = fv[jj];
#pragma unroll
              for (int r = 0; r < R; ++r) {
                const float d = sep32(xh[r], xl[r], mh, ml);
                const float d2 = d * d;
                const float inv = rcp32_unbiased(d2 + eta2f);
                const float i2 = inv * inv;
                const float A = (d2 - eta2f) * i2;
                const float B = tetaf * d * i2;
                pp[r][0] += A;
                pp[r][1] = fmaf(wj, A, pp[r][1]);
                pp[r][2] += B;
                pp[r][3] = fmaf(vj, B, pp[r][3]);
              }
            }
#pragma unroll
            for (int r = 0; r < R; ++r)
#pragma unroll
              for (int q = 0; q < 4; ++q) acc[r][q] += (double)pp[r][q];
          }
        } else {
          for (int j = sub; j < sub + slen; ++j) {
            const double l = sl[j], wj = sw[j], vj = sv[j];
#pragma unroll
            for (int r = 0; r < R; ++r) {
              const double d = x[r] - l;
              const double d2 = d * d;
              const double inv = rcp_f64(d2 + eta2);
              const double i2 = inv * inv;
              const double A = (d2 - eta2) * i2;
              const double B = teta * d * i2;
              acc[r][0] += A;
              acc[r][1] = fma(wj, A, acc[r][1]);
              acc[r][2] += B;
              acc[r][3] = fma(vj, B, acc[r][3]);
            }
          }
        }
      }
    }
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const int64_t idx = wbase + r * 32 + lane;
      if (idx >= a.p) continue;
#pragma unroll
      for (int q = 0; q < 4; ++q) a.part[((int64_t)split * 4 + q) * a.p + idx] = acc[r][q];
    }
    __syncthreads();
  }
}

__global__ void adjoint_reduce_kernel(const double* __restrict__ part, int n_splits, int64_t p,
                                      const double* __restrict__ w, const double* __restrict__ v,
                                      double inv_p, double* __restrict__ grad) {
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= p) return;
  double s[4] = {0, 0, 0, 0};
  for (int sp = 0; sp < n_splits; ++sp)
    for (int q = 0; q < 4; ++q) s[q] += part[((int64_t)sp * 4 + q) * p + k];
  grad[k] = (w[k] * s[0] - s[1] - v[k] * s[2] - s[3]) * inv_p;
}

}  // namespace

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

shrk_status adjoint(const double* d_ev, int64_t p, double eta, const double* d_gre,
                    const double* d_gim, int precision, double* d_grad, cudaStream_t s) {
  if (p <= 0) return SHRK_OK;
  const bool mixed = (precision == SHRK_PREC_MIXED);
  const SplitPlan pl = plan_splits(p, p, TT, ACH, 2);
  void* part = nullptr;
  SHRK_TRY(scratch_get(2, sizeof(double) * 4 * (size_t)pl.n_splits * (size_t)p, &part));
  double2* bounds = nullptr;
  const int64_t nblocks = (p + SUB - 1) / SUB;
  if (mixed) {
    void* b = nullptr;
    SHRK_TRY(scratch_get(1, sizeof(double2) * (size_t)(nblocks + 1), &b));
    bounds = (double2*)b;
    SHRK_TRY(source_bounds(d_ev, p, nblocks, bounds, s));
  }
  AdjArgs a;
  a.ev = d_ev;
  a.w = d_gre;
  a.v = d_gim;
  a.p = p;
  a.bounds = bounds;
  a.gminmax = bounds ? bounds + nblocks : nullptr;
  a.eta = eta;
  a.near_dist = std::max(mixed_near_k() * eta, 1e-9);
  a.n_tiles = pl.n_tiles;
  a.n_splits = pl.n_splits;
  a.split_len = pl.split_len;
  a.part = (double*)part;
  {
    LaunchScope ls(mixed ? "adjoint_mixed" : "adjoint_f64", s);
    if (mixed) adjoint_kernel<true><<<pl.grid, NT, 0, s>>>(a);
    else adjoint_kernel<false><<<pl.grid, NT, 0, s>>>(a);
    SHRK_CUDA(cudaGetLastError());
  }
  {
    LaunchScope ls("adjoint_reduce", s);
    adjoint_reduce_kernel<<<(unsigned)((p + 255) / 256), 256, 0, s>>>(
        (const double*)part, pl.n_splits, p, d_gre, d_gim, 1.0 / (double)p, d_grad);
    SHRK_CUDA(cudaGetLastError());
  }
  return SHRK_OK;
}

}  // namespace shrk
