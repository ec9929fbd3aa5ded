// Exact O(nt*ns) Stieltjes pair sums on sm_100a.
//
// Replaces the exact family of the shrinkers crate: symmetric_sweep
// (src/stieltjes/cacheblock.rs:841-954), the tiled full-square kernels
// (cacheblock.rs:1286-1513), the at-points kernel (cacheblock.rs:167-437),
// the windowed cutoff kernels (cacheblock.rs:452-577), the f32 kernel
// (cacheblock.rs:1525-1572) and the value+derivative sum
// (src/stieltjes/autovec.rs:38-77).  The pair term is term.rs:26-31:
//     1/((x - s) - i eta) = (d + i eta)/(d^2 + eta^2),  d = x - s.
//
// Work decomposition: a CTA of 256 threads owns a tile of 1024 targets
// (4 per thread, 128 consecutive targets per warp) and one split of the
// sources.  Source chunks of 1024 doubles are staged into shared memory by
// TMA bulk copies (cp.async.bulk + mbarrier, double-buffered) and read by
// all threads as broadcasts.  Each (tile, split) item writes its partial
// sums to a scratch slab; a second kernel reduces the splits in a fixed
// order in FP64 (deterministic) and applies the fused epilogue.
//
// MIXED precision: a source sub-chunk of 256 whose interval lies at least
// max(K*eta, W) away from the warp's targets (W = spread of the CTA's
// targets around their centre c) is summed in FP32: d = (xh - mu_j) + xl
// with mu_j = float(s_j - c) and x - c split into a hi/lo float pair, the
// reciprocal on the MUFU pipe, 16-term FP32 partials folded into a
// compensated (TwoSum hi/lo) accumulator.  Every other pair -- the near
// field, where d cancels -- is summed in FP64, as are all reductions.
#include "common.cuh"
#include "epilogue.cuh"
#include "internal.h"

#include <algorithm>
#include <cmath>

namespace shrk {

namespace {

constexpr int NT = 256;        // threads per CTA
constexpr int R = 4;           // targets per thread
constexpr int TT = NT * R;     // targets per tile
constexpr int WT = 32 * R;     // targets per warp
constexpr int CH = 1024;       // sources per staged chunk
constexpr int SUB = 256;       // sources per near/far classification block
// FP32 far-field arithmetic of the MIXED kernel (compile-time choices; the
// defaults are the measured best):
//   SHRK_RCP  0: rcp.approx alone (biased: ~1.5e-9 median error at p = 1e6)
//             1: rcp.approx + one Newton step (unbiased)
//   SHRK_FOLDMODE 0: FP32 partials folded into a TwoSum hi/lo FP32 pair
//                 1: FP32 partials folded into the FP64 accumulators
//   SHRK_FOLD: sources per FP32 partial (two interleaved chains)
#ifndef SHRK_RCP
#define SHRK_RCP 1
#endif
#ifndef SHRK_FOLDMODE
#define SHRK_FOLDMODE 1
#endif
#ifndef SHRK_FOLD
#define SHRK_FOLD 16
#endif
#ifndef SHRK_NEAR_K
#define SHRK_NEAR_K 32.0
#endif
constexpr int FOLD = SHRK_FOLD;  // FP32 partial length before a fold

// Near-field radius in units of eta for the MIXED kernel.
double g_near_k = SHRK_NEAR_K;

struct PairArgs {
  const double* tgt;
  int64_t nt;
  const double* src;
  int64_t ns;
  const double2* bounds;  // per SUB block of sources: (min, max)
  const double2* gminmax; // (min, max) over all sources
  double eta;
  double near_dist;
  int64_t n_tiles;
  int n_splits;
  int64_t split_len;      // multiple of CH
  double* part_re;        // [n_splits][nt]
  double* part_im;
  int* err;
  int use_tma;
};

// Power of two u >= ulp_float(M): the grid on which target offsets are
// snapped so that (xh - mh) is exact for every |mh| <= M.  IEEE-754 bit
// layout only (exponent field of M, shifted by the 23 fraction bits).
__device__ __forceinline__ double snap_unit(double M) {
  const long long bits = __double_as_longlong(M) & 0x7FF0000000000000LL;
  return __longlong_as_double(bits) * 0x1p-23;
}

// Split x - c into xh + xl with xh a multiple of u (exact in float while
// |x - c| < 2^23 u, which the caller guarantees).
__device__ __forceinline__ void split_target(double x, double c, double u, float& xh, float& xl) {
  const double xo = x - c;
  const double h = rint(xo / u) * u;
  xh = (float)h;
  xl = (float)(xo - h);
}

__device__ __forceinline__ void pair64(double x, double s, double eta2, double& re, double& iv) {
  const double d = x - s;
  const double inv = rcp_f64(fma(d, d, eta2));
  re = fma(d, inv, re);
  iv = iv + inv;
}

// FP32 separation of a target and a source, both split around the CTA
// centre c: x - c = xh + xl and s - c = mh + ml, with xh a multiple of a
// power of two u >= ulp(max |s - c|).  Then xh - mh is exact (or rounds on
// mh's own bits), and the final rounding of (xh - mh) + (xl - ml) depends on
// the source's low bits ml -- the errors of different pairs are independent.
// (Rounding a FIXED target offset onto each source's float grid instead
// shifts the target coherently by up to half an ulp of d: a systematic error
// that no accumulation scheme can remove.)
__device__ __forceinline__ float sep32(float xh, float xl, float mh, float ml) {
  return (xh - mh) + (xl - ml);
}

// Unbiased FP32 reciprocal: the MUFU seed's error has a nonzero mean (a
// few 1e-9 relative, measured), which would add coherently over a far field
// of ~1e6 same-signed terms; one Newton step r + r (1 - a r) removes it.
__device__ __forceinline__ float rcp32_unbiased(float a) {
  const float r = rcp_f32(a);
#if SHRK_RCP == 1
  return fmaf(r, fmaf(-a, r, 1.0f), r);
#else
  return r;
#endif
}

__device__ __forceinline__ void pair32(float xh, float xl, float mh, float ml, float eta2f,
                                       float& re, float& iv) {
  const float d = sep32(xh, xl, mh, ml);
  const float inv = rcp32_unbiased(fmaf(d, d, eta2f));
  re = fmaf(d, inv, re);
  iv = iv + inv;
}

__device__ __forceinline__ double warp_max(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}
__device__ __forceinline__ double warp_min(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmin(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

template <bool MIXED>
__global__ void __launch_bounds__(NT, 2) pair_sum_kernel(const PairArgs a) {
  __shared__ __align__(16) double sbuf[2][CH];
  __shared__ __align__(16) float smu[MIXED ? CH : 4];   // high part of s - c
  __shared__ __align__(16) float smul[MIXED ? CH : 4];  // low part of s - c
  __shared__ __align__(8) uint64_t bar[2];
  __shared__ double red[NT / 32];

  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  if (tid == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    fence_mbar_init();
  }
  __syncthreads();
  uint32_t phase = 0u;    // bit b: expected parity of bar[b]
  uint32_t pending = 0u;  // bit b: thread 0 issued a copy into sbuf[b]

  const double eta = a.eta, eta2 = eta * eta;
  const float eta2f = (float)eta2;
  const int64_t n_items = a.n_tiles * (int64_t)a.n_splits;

  for (int64_t item = blockIdx.x; item < n_items; item += gridDim.x) {
    const int64_t tile = item / a.n_splits;
    const int split = (int)(item % a.n_splits);
    const int64_t tile0 = tile * TT;
    const int64_t wbase = tile0 + (int64_t)warp * WT;
    const double x0 = a.tgt[tile0];
    double x[R];
    bool valid[R];
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const int64_t idx = wbase + r * 32 + lane;
      valid[r] = idx < a.nt;
      x[r] = valid[r] ? a.tgt[idx] : x0;
    }
    const int64_t s0 = (int64_t)split * a.split_len;
    const int64_t s1 = min(a.ns, s0 + a.split_len);
    const int nchunks = (int)((s1 - s0 + CH - 1) / CH);

    double re64[R], iv64[R];
    float hr[R], lr[R], hv[R], lv[R], xh[R], xl[R];
#pragma unroll
    for (int r = 0; r < R; ++r) {
      re64[r] = 0.0; iv64[r] = 0.0;
      hr[r] = lr[r] = hv[r] = lv[r] = 0.0f;
      xh[r] = xl[r] = 0.0f;
    }
    const double c = x0;
    double wlo = 0.0, whi = 0.0, thr = 0.0;
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
      double w = 0.0;
#pragma unroll
      for (int i = 0; i < NT / 32; ++i) w = fmax(w, red[i]);
      const double2 g = *a.gminmax;
      const double u = snap_unit(fmax(fmax(g.y - c, c - g.x), w));
      // The far path needs the targets' snapped offsets to stay exact floats.
      thr = (w < 0x1p22 * u) ? fmax(a.near_dist, w) : INFINITY;
#pragma unroll
      for (int r = 0; r < R; ++r) split_target(x[r], c, u, xh[r], xl[r]);
    }

    auto chunk_is_tma = [&](int k) -> bool {
      const int64_t cs = s0 + (int64_t)k * CH;
      return a.use_tma && k < nchunks && (s1 - cs) >= CH;
    };
    if (tid == 0) {
#pragma unroll
      for (int k = 0; k < 2; ++k) {
        if (chunk_is_tma(k)) {
          mbar_arrive_expect_tx(&bar[k], CH * 8);
          bulk_g2s(sbuf[k], a.src + s0 + (int64_t)k * CH, CH * 8, &bar[k]);
          pending |= 1u << k;
        }
      }
    }

    for (int k = 0; k < nchunks; ++k) {
      const int b = k & 1;
      const int64_t cs = s0 + (int64_t)k * CH;
      const int len = (int)min((int64_t)CH, s1 - cs);
      const bool tma = chunk_is_tma(k);
      bool ok = true;
      if (tma) {
        ok = mbar_wait(&bar[b], (phase >> b) & 1u);
        phase ^= 1u << b;
        pending &= ~(1u << b);
      } else {
        for (int i = tid; i < len; i += NT) sbuf[b][i] = a.src[cs + i];
      }
      if (!__syncthreads_and(ok)) {
        // A bulk copy never completed: record it, drain what thread 0 still
        // has in flight (bounded), and leave the kernel uniformly.
        if (tid == 0) {
          atomicExch(a.err, DEV_ERR_TIMEOUT);
          for (int q = 0; q < 2; ++q)
            if ((pending >> q) & 1u) mbar_wait(&bar[q], (phase >> q) & 1u, 200000000LL);
        }
        return;
      }
      if (MIXED) {
        for (int i = tid; i < len; i += NT) {
          const double so = sbuf[b][i] - c;
          const float h = (float)so;
          smu[i] = h;
          smul[i] = (float)(so - (double)h);
        }
        __syncthreads();
      }

      for (int sub = 0; sub < len; sub += SUB) {
        const int slen = min(SUB, len - sub);
        bool far32 = false;
        if (MIXED && slen == SUB) {
          const double2 bd = a.bounds[(cs + sub) / SUB];
          const double gap = fmax(fmax(bd.x - whi, wlo - bd.y), 0.0);
          const double span = fmax(bd.y - wlo, whi - bd.x);
          // far enough for FP32, and every product of two denominators stays a
          // normal float (thr >= 1e-9 is enforced on the host)
          far32 = gap >= thr && span <= 1e9;
        }
        if (MIXED && far32) {
          const float* mp = &smu[sub];
          const float* lp = &smul[sub];
          for (int j = 0; j < SUB; j += FOLD) {
            // Two interleaved FP32 chains per target (even / odd sources)
            // halve the partials' accumulation error at no extra work.
            float pr[2][R], pv[2][R];
#pragma unroll
            for (int r = 0; r < R; ++r) {
              pr[0][r] = pv[0][r] = 0.0f;
              pr[1][r] = pv[1][r] = 0.0f;
            }
#pragma unroll
            for (int q = 0; q < FOLD; q += 4) {
              const float4 m4 = *reinterpret_cast<const float4*>(mp + j + q);
              const float4 l4 = *reinterpret_cast<const float4*>(lp + j + q);
              const float ms[4] = {m4.x, m4.y, m4.z, m4.w};
              const float ls[4] = {l4.x, l4.y, l4.z, l4.w};
#pragma unroll
              for (int u = 0; u < 4; ++u) {
#pragma unroll
                for (int r = 0; r < R; ++r)
                  pair32(xh[r], xl[r], ms[u], ls[u], eta2f, pr[u & 1][r], pv[u & 1][r]);
              }
            }
#pragma unroll
            for (int r = 0; r < R; ++r) {
              const float sr = pr[0][r] + pr[1][r], sv = pv[0][r] + pv[1][r];
#if SHRK_FOLDMODE == 1
              re64[r] += (double)sr;
              iv64[r] += (double)sv;
#else
              two_sum_acc(hr[r], lr[r], sr);
              two_sum_acc(hv[r], lv[r], sv);
#endif
            }
          }
        } else {
          const double* sp = &sbuf[b][sub];
          int j = 0;
#pragma unroll 2
          for (; j + 2 <= slen; j += 2) {
            const double2 l2 = *reinterpret_cast<const double2*>(sp + j);
#pragma unroll
            for (int r = 0; r < R; ++r) {
              pair64(x[r], l2.x, eta2, re64[r], iv64[r]);
              pair64(x[r], l2.y, eta2, re64[r], iv64[r]);
            }
          }
          if (j < slen) {
            const double l = sp[j];
#pragma unroll
            for (int r = 0; r < R; ++r) pair64(x[r], l, eta2, re64[r], iv64[r]);
          }
        }
      }
      __syncthreads();
      if (tid == 0 && chunk_is_tma(k + 2)) {
        fence_proxy_async();
        mbar_arrive_expect_tx(&bar[b], CH * 8);
        bulk_g2s(sbuf[b], a.src + s0 + (int64_t)(k + 2) * CH, CH * 8, &bar[b]);
        pending |= 1u << b;
      }
    }

    double* pre = a.part_re + (int64_t)split * a.nt;
    double* pim = a.part_im + (int64_t)split * a.nt;
#pragma unroll
    for (int r = 0; r < R; ++r) {
      if (!valid[r]) continue;
      const int64_t idx = wbase + r * 32 + lane;
      double re = re64[r], iv = iv64[r];
      if (MIXED) {
        re = re + ((double)hr[r] + (double)lr[r]);
        iv = iv + ((double)hv[r] + (double)lv[r]);
      }
      pre[idx] = re;
      pim[idx] = eta * iv;
    }
  }
}

// (min, max) over the block bounds, written after them (one CTA).
__global__ void __launch_bounds__(1024) minmax_kernel(double2* __restrict__ bounds, int64_t nblocks) {
  __shared__ double smin[32], smax[32];
  double mn = INFINITY, mx = -INFINITY;
  for (int64_t i = threadIdx.x; i < nblocks; i += blockDim.x) {
    mn = fmin(mn, bounds[i].x);
    mx = fmax(mx, bounds[i].y);
  }
  mn = warp_min(mn);
  mx = warp_max(mx);
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (lane == 0) { smin[w] = mn; smax[w] = mx; }
  __syncthreads();
  if (w == 0) {
    const int nw = blockDim.x >> 5;
    mn = lane < nw ? smin[lane] : INFINITY;
    mx = lane < nw ? smax[lane] : -INFINITY;
    mn = warp_min(mn);
    mx = warp_max(mx);
    if (lane == 0) bounds[nblocks] = make_double2(mn, mx);
  }
}

// (min, max) of every SUB-block of sources.
__global__ void block_bounds_kernel(const double* __restrict__ src, int64_t ns,
                                    double2* __restrict__ out, int64_t nblocks) {
  const int64_t blk = (int64_t)blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (blk >= nblocks) return;
  const int64_t b0 = blk * SUB, b1 = min(ns, b0 + SUB);
  double mn = INFINITY, mx = -INFINITY;
  for (int64_t i = b0 + lane; i < b1; i += 32) {
    const double v = src[i];
    mn = fmin(mn, v);
    mx = fmax(mx, v);
  }
  mn = warp_min(mn);
  mx = warp_max(mx);
  if (lane == 0) out[blk] = make_double2(mn, mx);
}

struct ReduceArgs {
  const double* part_re;
  const double* part_im;
  int n_splits;
  int64_t nt;
  const double* tgt;
  Epilogue epi;
};

// Fixed-order FP64 reduction of the split partials + fused epilogue.  The
// epilogue arithmetic is written operation by operation as in the
// reference (the library is compiled without FMA contraction).
__global__ void reduce_kernel(const ReduceArgs a) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= a.nt) return;
  double re = 0.0, im = 0.0;
  for (int s = 0; s < a.n_splits; ++s) {
    re += a.part_re[(int64_t)s * a.nt + t];
    im += a.part_im[(int64_t)s * a.nt + t];
  }
  epi_store(a.epi, t, a.tgt[t], re, im);
}

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
    if (src[mid] < lo_v) lo = mid + 1; else hi = mid;
  }
  int64_t a = lo;
  lo = a; hi = ns;          // first index with src > hi_v
  while (lo < hi) {
    const int64_t mid = (lo + hi) >> 1;
    if (src[mid] <= hi_v) lo = mid + 1; else hi = mid;
  }
  double sr = 0.0, si = 0.0;
  for (int64_t j = a; j < lo; ++j) {
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
// shared memory.  MIXED: far pairs in FP32 (compensated), near in FP64.
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
  double* part;   // [n_splits][4][p]
};

template <bool MIXED>
__global__ void __launch_bounds__(NT, 2) adjoint_kernel(const AdjArgs a) {
  constexpr int ACH = 512;
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
    bool valid[R];
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const int64_t idx = wbase + r * 32 + lane;
      valid[r] = idx < a.p;
      x[r] = valid[r] ? a.ev[idx] : x0;
    }
    double acc[R][4];
    float hs[R][4], ls[R][4], xh[R], xl[R];
#pragma unroll
    for (int r = 0; r < R; ++r)
#pragma unroll
      for (int q = 0; q < 4; ++q) { acc[r][q] = 0.0; hs[r][q] = 0.0f; ls[r][q] = 0.0f; }
    const double c = x0;
    double wlo = 0, whi = 0, thr = 0;
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
          const double so = sl[i] - c;
          const float h = (float)so;
          fmu[i] = h;
          fml[i] = (float)(so - (double)h);
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
          far32 = gap >= thr;
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
              for (int q = 0; q < 4; ++q) two_sum_acc(hs[r][q], ls[r][q], pp[r][q]);
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
      if (!valid[r]) continue;
      const int64_t idx = wbase + r * 32 + lane;
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        double v = acc[r][q];
        if (MIXED) v = v + ((double)hs[r][q] + (double)ls[r][q]);
        a.part[((int64_t)split * 4 + q) * a.p + idx] = v;
      }
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

struct SplitPlan {
  int64_t n_tiles;
  int n_splits;
  int64_t split_len;
  int grid;
};

SplitPlan plan_splits(int64_t nt, int64_t ns, int chunk) {
  SplitPlan pl;
  pl.n_tiles = (nt + TT - 1) / TT;
  const int ctas = std::max(1, sm_count() * 2);
  const int64_t max_splits = std::max<int64_t>(1, (ns + chunk - 1) / chunk);
  int64_t want = (8LL * ctas + pl.n_tiles - 1) / pl.n_tiles;
  want = std::min(std::max<int64_t>(want, 1), max_splits);
  int64_t per = (ns + want - 1) / want;
  pl.split_len = ((per + chunk - 1) / chunk) * chunk;
  pl.n_splits = (int)((ns + pl.split_len - 1) / pl.split_len);
  const int64_t items = pl.n_tiles * pl.n_splits;
  pl.grid = (int)std::min<int64_t>(items, ctas);
  return pl;
}

}  // namespace

double mixed_near_k() { return g_near_k; }

// Block bounds of the sources and, after them, the global (min, max).
static shrk_status source_bounds(const double* d_src, int64_t ns, int64_t nblocks,
                                 double2* bounds, cudaStream_t s) {
  {
    LaunchScope ls("block_bounds", s);
    block_bounds_kernel<<<(unsigned)((nblocks + 7) / 8), 256, 0, s>>>(d_src, ns, bounds, nblocks);
    SHRK_CUDA(cudaGetLastError());
  }
  {
    LaunchScope ls("block_bounds", s);
    minmax_kernel<<<1, 1024, 0, s>>>(bounds, nblocks);
    SHRK_CUDA(cudaGetLastError());
  }
  return SHRK_OK;
}

shrk_status exact_pair_sums(const double* d_tgt, int64_t nt, const double* d_src, int64_t ns,
                            double eta, int precision, const Epilogue& epi, cudaStream_t s) {
  if (nt <= 0) return SHRK_OK;
  if (ns <= 0) {
    set_error("exact_pair_sums: empty source set");
    return SHRK_EINVAL;
  }
  const bool mixed = (precision == SHRK_PREC_MIXED);
  const SplitPlan pl = plan_splits(nt, ns, CH);
  void* part = nullptr;
  SHRK_TRY(scratch_get(0, sizeof(double) * 2 * (size_t)pl.n_splits * (size_t)nt, &part));
  double2* bounds = nullptr;
  const int64_t nblocks = (ns + SUB - 1) / SUB;
  if (mixed) {
    void* b = nullptr;
    SHRK_TRY(scratch_get(1, sizeof(double2) * (size_t)(nblocks + 1), &b));
    bounds = (double2*)b;
    SHRK_TRY(source_bounds(d_src, ns, nblocks, bounds, s));
  }
  PairArgs a;
  a.tgt = d_tgt;
  a.nt = nt;
  a.src = d_src;
  a.ns = ns;
  a.bounds = bounds;
  a.gminmax = bounds ? bounds + nblocks : nullptr;
  a.eta = eta;
  a.near_dist = std::max(g_near_k * eta, 1e-9);
  a.n_tiles = pl.n_tiles;
  a.n_splits = pl.n_splits;
  a.split_len = pl.split_len;
  a.part_re = (double*)part;
  a.part_im = (double*)part + (size_t)pl.n_splits * nt;
  a.err = device_error_word();
  a.use_tma = ((uintptr_t)d_src % 16 == 0) ? 1 : 0;
  {
    LaunchScope ls(mixed ? "pair_sum_mixed" : "pair_sum_f64", s);
    if (mixed) pair_sum_kernel<true><<<pl.grid, NT, 0, s>>>(a);
    else pair_sum_kernel<false><<<pl.grid, NT, 0, s>>>(a);
    SHRK_CUDA(cudaGetLastError());
  }
  ReduceArgs ra;
  ra.part_re = a.part_re;
  ra.part_im = a.part_im;
  ra.n_splits = pl.n_splits;
  ra.nt = nt;
  ra.tgt = d_tgt;
  ra.epi = epi;
  {
    LaunchScope ls("split_reduce", s);
    reduce_kernel<<<(unsigned)((nt + 255) / 256), 256, 0, s>>>(ra);
    SHRK_CUDA(cudaGetLastError());
  }
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

shrk_status adjoint(const double* d_ev, int64_t p, double eta, const double* d_gre,
                    const double* d_gim, int precision, double* d_grad, cudaStream_t s) {
  if (p <= 0) return SHRK_OK;
  const bool mixed = (precision == SHRK_PREC_MIXED);
  const SplitPlan pl = plan_splits(p, p, 512);
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
  a.near_dist = std::max(g_near_k * eta, 1e-9);
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

namespace shrk {
shrk_status apply_epilogue(const double* d_tgt, const double* d_raw_re, const double* d_raw_im,
                           int64_t n, const Epilogue& epi, cudaStream_t s) {
  if (n <= 0) return SHRK_OK;
  ReduceArgs ra;
  ra.part_re = d_raw_re;
  ra.part_im = d_raw_im;
  ra.n_splits = 1;
  ra.nt = n;
  ra.tgt = d_tgt;
  ra.epi = epi;
  LaunchScope ls("epilogue", s);
  reduce_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(ra);
  SHRK_CUDA(cudaGetLastError());
  return SHRK_OK;
}
}  // namespace shrk
