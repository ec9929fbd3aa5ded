// Adjoint of the all-points transform (no reference counterpart):
//   dL/dev_k = (1/p) sum_j G(k, j),
//   G(k, j) = (w_k - w_j)(a^2 - eta^2)/D^2 - (v_k + v_j) 2 a eta/D^2,
//   a = ev_k - ev_j, D = a^2 + eta^2,
// for L = sum_j (w_j Re m_j + v_j Im m_j), m_j = (1/p) sum_i 1/(ev_i - z_j),
// z_j = ev_j + i eta: the source term of each m_j plus the dependence of z_k
// on ev_k (the target derivative of autovec.rs:38-59).  Pairs are recomputed,
// never stored.
//
// G is antisymmetric (G(j, k) = -G(k, j)), so the main kernel evaluates each
// unordered pair once and adds it to both ends; the row-sum kernel (every
// ordered pair, four source sums per target) remains for sizes whose column
// slabs would not fit.
#include "common.cuh"
#include "internal.h"
#include "pairs.cuh"

#include <algorithm>
#include <cmath>

namespace shrk {

namespace {

constexpr int NT = 256;
constexpr int R = 4;             // targets per thread (row-sum adjoint)
constexpr int TT = NT * R;
constexpr int WT = 32 * R;
constexpr int ACH = 512;         // sources per staged chunk (row-sum adjoint)
constexpr int FOLD = 16;         // FP32 partial length before the FP64 fold

// ------------------------------------------------- row-sum adjoint ----
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

// ------------------------------------------------- symmetric adjoint ----
// With r = 1/D, A = (a^2 - eta^2)/D^2 = r - 2 eta^2 r^2, B = a r^2 and
// v' = 2 eta v:  G(k, j) = (w_k - w_j) A - (v'_k + v'_j) B.
// Work item (T, S), T <= S: target tile T (R targets per thread, in
// registers) against source tile S (staged in chunks of SUB).  Each pair's G
// is added to the row of k and, negated, to the column of j; column sums are
// reduced across the warp by shuffles and across the CTA in a fixed order.
// Rows of item (T, S) go to slab S and columns to slab T, so every target
// receives exactly one value per slab (no clearing, deterministic).  The
// diagonal items (T, T) sum their tile as a full square, rows only
// (G(k, k) = 0).  MIXED: a source block at least near_dist from all of the
// warp's targets is summed in FP32 (block-centred separation as in the
// forward kernel, unbiased reciprocal, partials folded into FP64).
struct AdjSymArgs {
  const double* ev;
  const double* w;
  const double* v;
  int64_t p;
  const double2* bounds;  // MIXED: (min, max) per SUB-block
  double eta;
  double near_dist;
  int n_tiles;
  int64_t n_items;        // n_tiles (n_tiles + 1) / 2
  double* part;           // [n_tiles][p]
};

// item -> (T, S), T <= S, row-major over the upper triangle.
__device__ __forceinline__ void tri_decode(int64_t item, int n, int& T, int& S) {
  const int64_t total = (int64_t)n * (n + 1) / 2;
  const int64_t m = total - 1 - item;  // index counted from the last row
  int64_t q = (int64_t)((sqrt(8.0 * (double)m + 1.0) - 1.0) * 0.5);
  while ((q + 1) * (q + 2) / 2 <= m) ++q;
  while (q * (q + 1) / 2 > m) --q;
  T = n - 1 - (int)q;
  S = n - 1 - (int)(m - q * (q + 1) / 2);
}

// Warp sums of four per-lane values c[0..3] (one per source) by
// reduce-scatter: the two lane halves exchange the pair they do not keep,
// then the quarter-halves the value they do not keep, then the remaining
// 8-lane groups reduce by butterflies -- 6 shuffles instead of 20.  Returns
// the full sum of c[q] in lanes 8q (q = 0..3); other lanes hold partials.
template <typename F>
__device__ __forceinline__ F warp_sum4(const F (&c)[4], int lane) {
  const bool hi16 = (lane & 16) != 0, hi8 = (lane & 8) != 0;
  const F s0 = hi16 ? c[0] : c[2], s1 = hi16 ? c[1] : c[3];
  const F k0 = (hi16 ? c[2] : c[0]) + __shfl_xor_sync(0xffffffffu, s0, 16);
  const F k1 = (hi16 ? c[3] : c[1]) + __shfl_xor_sync(0xffffffffu, s1, 16);
  F v = (hi8 ? k1 : k0) + __shfl_xor_sync(0xffffffffu, hi8 ? k0 : k1, 8);
#pragma unroll
  for (int o = 4; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

template <bool MIXED, int RS>
__global__ void __launch_bounds__(NT, 2) adjoint_sym_kernel(const AdjSymArgs a) {
  constexpr int STT = NT * RS, SWT = 32 * RS;
  __shared__ __align__(16) double sl[SUB], sw[SUB], sv[SUB];
  __shared__ __align__(16) float fsm[MIXED ? SUB : 1], fw[MIXED ? SUB : 1], fv[MIXED ? SUB : 1];
  __shared__ double colw[NT / 32][SUB];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const double eta = a.eta, eta2 = eta * eta, teta = 2.0 * eta, m2e2 = -2.0 * eta2;
  const float eta2f = (float)eta2, m2e2f = (float)m2e2;
  for (int64_t item = blockIdx.x; item < a.n_items; item += gridDim.x) {
    int T, S;
    tri_decode(item, a.n_tiles, T, S);
    const bool diag = T == S;
    const int64_t tile0 = (int64_t)T * STT, wbase = tile0 + (int64_t)warp * SWT;
    double x[RS], wk[RS], vk[RS], row[RS];
    bool valid[RS];
#pragma unroll
    for (int r = 0; r < RS; ++r) {
      const int64_t idx = wbase + r * 32 + lane;
      valid[r] = idx < a.p;
      x[r] = valid[r] ? a.ev[idx] : a.ev[tile0];
      wk[r] = valid[r] ? a.w[idx] : 0.0;
      vk[r] = valid[r] ? teta * a.v[idx] : 0.0;
      row[r] = 0.0;
    }
    double wlo = 0.0, whi = 0.0;
    if (MIXED) {
      double mn = x[0], mx = x[0];
#pragma unroll
      for (int r = 0; r < RS; ++r) {
        mn = fmin(mn, x[r]);
        mx = fmax(mx, x[r]);
      }
      wlo = warp_min(mn);
      whi = warp_max(mx);
    }
    const int64_t src0 = (int64_t)S * STT, src1 = min(a.p, src0 + STT);
    for (int64_t cs = src0; cs < src1; cs += SUB) {
      const int len = (int)min((int64_t)SUB, src1 - cs);
      __syncthreads();  // the previous chunk's readers are done
      const double cb = a.ev[cs];
      for (int i = tid; i < len; i += NT) {
        const double l = a.ev[cs + i], wj = a.w[cs + i], vj = teta * a.v[cs + i];
        sl[i] = l;
        sw[i] = wj;
        sv[i] = vj;
        if (MIXED) {
          fsm[i] = (float)(l - cb);
          fw[i] = (float)wj;
          fv[i] = (float)vj;
        }
      }
      __syncthreads();
      bool far32 = false;
      if (MIXED && len == SUB) {
        const double2 bd = a.bounds[cs / SUB];
        const double gap = fmax(fmax(bd.x - whi, wlo - bd.y), 0.0);
        const double span = fmax(bd.y - wlo, whi - bd.x);
        far32 = gap >= a.near_dist && span <= 1e9;
      }
      if (MIXED && far32) {
        float th[RS], tl[RS], wkf[RS], vkf[RS];
#pragma unroll
        for (int r = 0; r < RS; ++r) {
          const double o = x[r] - cb;
          th[r] = (float)o;
          tl[r] = (float)(o - (double)th[r]);
          wkf[r] = (float)wk[r];
          vkf[r] = (float)vk[r];
        }
        for (int j0 = 0; j0 < SUB; j0 += FOLD) {
          float rowf[RS];
#pragma unroll
          for (int r = 0; r < RS; ++r) rowf[r] = 0.0f;
#pragma unroll 1
          for (int j = j0; j < j0 + FOLD; j += 4) {
            float col[4];
#pragma unroll
            for (int q = 0; q < 4; ++q) {
              const float sm = fsm[j + q], wj = fw[j + q], vj = fv[j + q];
              col[q] = 0.0f;
#pragma unroll
              for (int r = 0; r < RS; ++r) {
                const float d = th[r] - (sm - tl[r]);
                const float rr = rcp32_unbiased(fmaf(d, d, eta2f));
                const float r2 = rr * rr;
                const float A = fmaf(m2e2f, r2, rr);
                const float g = fmaf(-(vkf[r] + vj), d * r2, (wkf[r] - wj) * A);
                rowf[r] += g;
                if (valid[r]) col[q] += g;
              }
            }
            if (!diag) {
              const float c = warp_sum4(col, lane);
              if ((lane & 7) == 0) colw[warp][j + (lane >> 3)] = (double)c;
            }
          }
#pragma unroll
          for (int r = 0; r < RS; ++r) row[r] += (double)rowf[r];
        }
      } else {
        // Groups of 4 sources; a ragged last group skips the sources past len.
        for (int j = 0; j < len; j += 4) {
          double col[4];
#pragma unroll
          for (int q = 0; q < 4; ++q) {
            col[q] = 0.0;
            if (j + q < len) {
              const double l = sl[j + q], wj = sw[j + q], vj = sv[j + q];
#pragma unroll
              for (int r = 0; r < RS; ++r) {
                const double d = x[r] - l;
                const double rr = rcp_f64(fma(d, d, eta2));
                const double r2 = rr * rr;
                const double A = fma(m2e2, r2, rr);
                const double g = fma(-(vk[r] + vj), d * r2, (wk[r] - wj) * A);
                row[r] += g;
                if (valid[r]) col[q] += g;
              }
            }
          }
          if (!diag) {
            const double c = warp_sum4(col, lane);
            const int q = lane >> 3;
            if ((lane & 7) == 0 && j + q < len) colw[warp][j + q] = c;
          }
        }
      }
      if (!diag) {
        __syncthreads();
        for (int i = tid; i < len; i += NT) {
          double c = 0.0;
#pragma unroll
          for (int q = 0; q < NT / 32; ++q) c += colw[q][i];
          a.part[(int64_t)T * a.p + cs + i] = -c;
        }
      }
    }
#pragma unroll
    for (int r = 0; r < RS; ++r) {
      const int64_t idx = wbase + r * 32 + lane;
      if (valid[r]) a.part[(int64_t)S * a.p + idx] = row[r];
    }
  }
}

// grad_k = (1/p) sum over slabs, in slab order.
__global__ void adjoint_slab_reduce_kernel(const double* __restrict__ part, int n_slabs,
                                           int64_t p, double inv_p, double* __restrict__ grad) {
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= p) return;
  double s = 0.0;
  for (int q = 0; q < n_slabs; ++q) s += part[(int64_t)q * p + k];
  grad[k] = s * inv_p;
}

}  // namespace

namespace {

// Row-sum path (every ordered pair).
shrk_status adjoint_rows(const double* d_ev, int64_t p, double eta, const double* d_gre,
                         const double* d_gim, int precision, double* d_grad, cudaStream_t s) {
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


template <int RS>
shrk_status launch_sym(const AdjSymArgs& a, bool mixed, int grid, cudaStream_t s) {
  LaunchScope ls(mixed ? "adjoint_mixed" : "adjoint_f64", s);
  if (mixed) adjoint_sym_kernel<true, RS><<<grid, NT, 0, s>>>(a);
  else adjoint_sym_kernel<false, RS><<<grid, NT, 0, s>>>(a);
  SHRK_CUDA(cudaGetLastError());
  return SHRK_OK;
}

}  // namespace

shrk_status adjoint(const double* d_ev, int64_t p, double eta, const double* d_gre,
                    const double* d_gim, int precision, double* d_grad, cudaStream_t s) {
  if (p <= 0) return SHRK_OK;
  const bool mixed = (precision == SHRK_PREC_MIXED);
  // Targets per thread: the widest tile that still gives the grid a few
  // waves of (T, S) items.
  const int64_t ctas = (int64_t)sm_count() * 2;
  int RS = 1;
  int64_t n_t = 0;
  for (int cand : {4, 2, 1}) {
    n_t = (p + (int64_t)NT * cand - 1) / ((int64_t)NT * cand);
    RS = cand;
    if (n_t * (n_t + 1) / 2 >= (cand == 4 ? 8 : 2) * ctas) break;
  }
  const size_t slab_bytes = sizeof(double) * (size_t)n_t * (size_t)p;
  if (slab_bytes > (size_t(2) << 30))
    return adjoint_rows(d_ev, p, eta, d_gre, d_gim, precision, d_grad, s);
  void* part = nullptr;
  SHRK_TRY(scratch_get(2, slab_bytes, &part));
  double2* bounds = nullptr;
  if (mixed) {
    const int64_t nblocks = (p + SUB - 1) / SUB;
    void* b = nullptr;
    SHRK_TRY(scratch_get(1, sizeof(double2) * (size_t)(nblocks + 1), &b));
    bounds = (double2*)b;
    SHRK_TRY(source_bounds(d_ev, p, nblocks, bounds, s));
  }
  AdjSymArgs a;
  a.ev = d_ev;
  a.w = d_gre;
  a.v = d_gim;
  a.p = p;
  a.bounds = bounds;
  a.eta = eta;
  a.near_dist = std::max(mixed_near_k() * eta, 1e-9);
  a.n_tiles = (int)n_t;
  a.n_items = n_t * (n_t + 1) / 2;
  a.part = (double*)part;
  const int grid = (int)std::min<int64_t>(a.n_items, ctas);
  if (RS == 4) SHRK_TRY(launch_sym<4>(a, mixed, grid, s));
  else if (RS == 2) SHRK_TRY(launch_sym<2>(a, mixed, grid, s));
  else SHRK_TRY(launch_sym<1>(a, mixed, grid, s));
  LaunchScope ls("adjoint_reduce", s);
  adjoint_slab_reduce_kernel<<<(unsigned)((p + 255) / 256), 256, 0, s>>>(
      (const double*)part, (int)n_t, p, 1.0 / (double)p, d_grad);
  SHRK_CUDA(cudaGetLastError());
  return SHRK_OK;
}

}  // namespace shrk
