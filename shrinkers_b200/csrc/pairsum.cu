// Exact O(nt*ns) Stieltjes pair sums on sm_100a (forward transform).
//
// Replaces the exact family of the shrinkers crate: symmetric_sweep
// (src/stieltjes/cacheblock.rs:841-954), the tiled full-square kernels
// (cacheblock.rs:1286-1513) and the at-points kernel (cacheblock.rs:167-437).
// The pair term is term.rs:26-31:
//     1/((x - s) - i eta) = (d + i eta)/(d^2 + eta^2),  d = x - s.
//
// Work decomposition: a CTA of 256 threads owns a tile of 256*R targets (R
// per thread, 32*R consecutive targets per warp) and one split of the
// sources.  Source chunks of 1024 doubles are staged into shared memory by
// TMA bulk copies (cp.async.bulk + mbarrier, double-buffered) and read by all
// threads as broadcasts.  Each (tile, split) item writes partial sums to a
// scratch slab; a second kernel reduces the splits in a fixed order in FP64
// (deterministic) and applies the fused epilogue.
//
// F64 (R = 4): every pair in FP64, reciprocal = hardware seed + one
// third-order Newton step.
//
// MIXED (R = 4): a source block of 256 whose interval lies at least
// max(K*eta, 1e-9) from all of the warp's targets is summed in FP32 on the
// packed f32x2 pipe -- two targets x two sources per step, one unbiased
// reciprocal per two sources (pairs32x4 in pairs.cuh), FP32 partials folded
// into FP64 every 16 sources.  Every other pair (the near field, where the
// terms are large and d cancels) is summed in FP64, as are all reductions.
#include "common.cuh"
#include "epilogue.cuh"
#include "internal.h"
#include "pairs.cuh"

#include <algorithm>
#include <cmath>

namespace shrk {

namespace {

#ifndef SHRK_R_MIXED
#define SHRK_R_MIXED 4
#endif
#ifndef SHRK_MIXED_CTAS
#define SHRK_MIXED_CTAS 2
#endif

constexpr int NT = 256;   // threads per CTA
constexpr int CH = 1024;  // sources per staged chunk
constexpr int FOLD = 16;  // sources per FP32 partial before the FP64 fold
constexpr int R_F64 = 4;
constexpr int R_MIXED = SHRK_R_MIXED;

double g_near_k = SHRK_NEAR_K;

struct PairArgs {
  const double* tgt;
  int64_t nt;
  const double* src;
  int64_t ns;
  const double2* bounds;   // per SUB block of sources: (min, max)
  double eta;
  double near_dist;
  int64_t n_tiles;
  int n_splits;
  int64_t split_len;       // multiple of CH
  double* part_re;         // [n_splits][nt]
  double* part_im;
  int* err;
  int use_tma;
};

template <bool MIXED, int R>
__global__ void __launch_bounds__(NT, MIXED ? SHRK_MIXED_CTAS : 2) pair_sum_kernel(const PairArgs a) {
  constexpr int TT = NT * R, WT = 32 * R, R2 = R / 2;
  __shared__ __align__(16) double sbuf[2][CH];
  __shared__ __align__(16) float4 sm4[MIXED ? CH / 2 : 1];  // {sm, sm, dl, dl} per source pair
  __shared__ __align__(8) uint64_t bar[2];

  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  if (tid == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    fence_mbar_init();
  }
  __syncthreads();
  uint32_t phase = 0u;    // bit b: expected parity of bar[b]
  uint32_t pending = 0u;  // bit b: thread 0 has a copy in flight into sbuf[b]

  const double eta = a.eta, eta2 = eta * eta;
  const float eta2f = (float)eta2;
  const u64 ETA2 = pk2(eta2f, eta2f), ONE = pk2(1.0f, 1.0f);
  const int64_t n_items = a.n_tiles * (int64_t)a.n_splits;

  for (int64_t item = blockIdx.x; item < n_items; item += gridDim.x) {
    const int64_t tile = item / a.n_splits;
    const int split = (int)(item % a.n_splits);
    const int64_t tile0 = tile * TT;
    const int64_t wbase = tile0 + (int64_t)warp * WT;
    const double x0 = a.tgt[tile0];
    double x[R];
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const int64_t idx = wbase + r * 32 + lane;
      x[r] = idx < a.nt ? a.tgt[idx] : x0;
    }
    const int64_t s0 = (int64_t)split * a.split_len;
    const int64_t s1 = min(a.ns, s0 + a.split_len);
    const int nchunks = (int)((s1 - s0 + CH - 1) / CH);

    double re64[R], iv64[R];
#pragma unroll
    for (int r = 0; r < R; ++r) re64[r] = iv64[r] = 0.0;
    // Range of this warp's targets: a source block is summed in FP32 only if
    // it lies at least near_dist from all of them.
    double wlo = 0.0, whi = 0.0;
    if (MIXED) {
      double mn = x[0], mx = x[0];
#pragma unroll
      for (int r = 0; r < R; ++r) {
        mn = fmin(mn, x[r]);
        mx = fmax(mx, x[r]);
      }
      wlo = warp_min(mn);
      whi = warp_max(mx);
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
      bool ok = true;
      if (chunk_is_tma(k)) {
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
        // Source pairs of each full 256-block: (s1, s2) = (src[k], src[k+128])
        // as {SM, SM, DL, DL} relative to the block's first source.  Pairing
        // sources half a block apart keeps e1 = d1^2+eta^2 and e2 well apart:
        // adjacent sorted sources give e1 e2 ~ a square, and the rounded
        // reciprocal of a near-square carries a small systematic error
        // (~2e-11 relative, measured) that adds up coherently at large p.
        for (int i = tid; i < (len / SUB) * (SUB / 2); i += NT) {
          const int blk = i / (SUB / 2) * SUB, k = i % (SUB / 2);
          const double cb = sbuf[b][blk];
          const double s1 = sbuf[b][blk + k], s2 = sbuf[b][blk + k + SUB / 2];
          const float sm = (float)(s1 - cb), dl = (float)(s1 - s2);
          sm4[i] = make_float4(sm, sm, dl, dl);
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
          far32 = gap >= a.near_dist && span <= 1e9;
        }
        if (MIXED && far32) {
          // Block-wide target offsets x - cb = TH + TL.
          const double cb = sbuf[b][sub];
          u64 TH[R2], TL[R2];
#pragma unroll
          for (int kk = 0; kk < R2; ++kk) {
            const double o0 = x[2 * kk] - cb, o1 = x[2 * kk + 1] - cb;
            const float h0 = (float)o0, h1 = (float)o1;
            TH[kk] = pk2(h0, h1);
            TL[kk] = pk2((float)(o0 - (double)h0), (float)(o1 - (double)h1));
          }
          const float4* sp = &sm4[sub / 2];
          const u64 ETA2_ = ETA2, ONE_ = ONE;
          for (int j = 0; j < SUB / 2; j += FOLD / 2) {
            u64 RE[R2], IV[R2];
#pragma unroll
            for (int kk = 0; kk < R2; ++kk) RE[kk] = IV[kk] = 0ull;
#pragma unroll
            for (int q = 0; q < FOLD / 2; ++q) {
              const float4 s4 = sp[j + q];
              const u64 SM = pk2(s4.x, s4.y), DL = pk2(s4.z, s4.w);
#pragma unroll
              for (int kk = 0; kk < R2; ++kk)
                pairs32x4(SM, DL, TH[kk], TL[kk], ETA2_, ONE_, RE[kk], IV[kk]);
            }
            // FP32 partials of FOLD sources are folded into FP64 (negated).
#pragma unroll
            for (int kk = 0; kk < R2; ++kk) {
              float r0, r1, v0, v1;
              upk2(RE[kk], r0, r1);
              upk2(IV[kk], v0, v1);
              re64[2 * kk] -= (double)r0;
              re64[2 * kk + 1] -= (double)r1;
              iv64[2 * kk] -= (double)v0;
              iv64[2 * kk + 1] -= (double)v1;
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
      const int64_t idx = wbase + r * 32 + lane;
      if (idx < a.nt) {
        pre[idx] = re64[r];
        pim[idx] = eta * iv64[r];
      }
    }
  }
}

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

__global__ void __launch_bounds__(1024) minmax_kernel(double2* __restrict__ bounds,
                                                      int64_t nblocks) {
  __shared__ double smin[32], smax[32];
  double mn = INFINITY, mx = -INFINITY;
  for (int64_t i = threadIdx.x; i < nblocks; i += blockDim.x) {
    mn = fmin(mn, bounds[i].x);
    mx = fmax(mx, bounds[i].y);
  }
  mn = warp_min(mn);
  mx = warp_max(mx);
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (lane == 0) {
    smin[w] = mn;
    smax[w] = mx;
  }
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

struct ReduceArgs {
  const double* part_re;
  const double* part_im;
  int n_splits;
  int64_t nt;
  const double* tgt;
  Epilogue epi;
};

// Fixed-order FP64 reduction of the split partials + fused epilogue.
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

}  // namespace

double mixed_near_k() { return g_near_k; }

SplitPlan plan_splits(int64_t nt, int64_t ns, int tile, int chunk, int ctas_per_sm) {
  SplitPlan pl;
  pl.n_tiles = (nt + tile - 1) / tile;
  const int ctas = std::max(1, sm_count() * ctas_per_sm);
  const int64_t max_splits = std::max<int64_t>(1, (ns + chunk - 1) / chunk);
  int64_t want = (8LL * ctas + pl.n_tiles - 1) / pl.n_tiles;
  want = std::min(std::max<int64_t>(want, 1), max_splits);
  const int64_t per = (ns + want - 1) / want;
  pl.split_len = ((per + chunk - 1) / chunk) * chunk;
  pl.n_splits = (int)((ns + pl.split_len - 1) / pl.split_len);
  pl.grid = (int)std::min<int64_t>(pl.n_tiles * pl.n_splits, ctas);
  return pl;
}

shrk_status source_bounds(const double* d_src, int64_t ns, int64_t nblocks, double2* bounds,
                          cudaStream_t s) {
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
  const int R = mixed ? R_MIXED : R_F64;
  const SplitPlan pl = plan_splits(nt, ns, NT * R, CH, mixed ? SHRK_MIXED_CTAS : 2);
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
    if (mixed) pair_sum_kernel<true, R_MIXED><<<pl.grid, NT, 0, s>>>(a);
    else pair_sum_kernel<false, R_F64><<<pl.grid, NT, 0, s>>>(a);
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

namespace {

// Split reduction for the caller-scratch launcher: raw sums, or NaN in every
// output when the pair kernel recorded a failed bounded wait (the caller is
// not synchronised, so the failure is reported through the values).
__global__ void reduce_flagged_kernel(const double* part_re, const double* part_im, int n_splits,
                                      int64_t nt, const int* err, double* out_re,
                                      double* out_im) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nt) return;
  if (*err != DEV_ERR_NONE) {
    out_re[t] = NAN;
    out_im[t] = NAN;
    return;
  }
  double re = 0.0, im = 0.0;
  for (int s = 0; s < n_splits; ++s) {
    re += part_re[(int64_t)s * nt + t];
    im += part_im[(int64_t)s * nt + t];
  }
  out_re[t] = re;
  out_im[t] = im;
}

}  // namespace

shrk_status exact_pair_sums_fixed(const double* d_tgt, int64_t nt, const double* d_src,
                                  int64_t ns, double eta, int precision, double* d_re,
                                  double* d_im, double* part, int64_t part_capacity,
                                  double2* bounds, int* err, int sms, cudaStream_t s) {
  if (nt <= 0) return SHRK_OK;
  if (ns <= 0 || part_capacity < nt) {
    set_error("exact_pair_sums_fixed: empty source set or scratch smaller than one split");
    return SHRK_EINVAL;
  }
  const bool mixed = (precision == SHRK_PREC_MIXED);
  const int R = mixed ? R_MIXED : R_F64;
  const int ctas = std::max(1, sms * (mixed ? SHRK_MIXED_CTAS : 2));
  const int64_t n_tiles = (nt + NT * R - 1) / (NT * R);
  // Same split rule as plan_splits, additionally capped by the scratch.
  const int64_t max_splits =
      std::max<int64_t>(1, std::min<int64_t>((ns + CH - 1) / CH, part_capacity / nt));
  int64_t want = (8LL * ctas + n_tiles - 1) / n_tiles;
  want = std::min(std::max<int64_t>(want, 1), max_splits);
  const int64_t per = (ns + want - 1) / want;
  const int64_t split_len = ((per + CH - 1) / CH) * CH;
  const int n_splits = (int)((ns + split_len - 1) / split_len);
  const int grid = (int)std::min<int64_t>(n_tiles * n_splits, ctas);
  const int64_t nblocks = (ns + SUB - 1) / SUB;
  if (mixed) {
    block_bounds_kernel<<<(unsigned)((nblocks + 7) / 8), 256, 0, s>>>(d_src, ns, bounds, nblocks);
    SHRK_CUDA(cudaGetLastError());
    minmax_kernel<<<1, 1024, 0, s>>>(bounds, nblocks);
    SHRK_CUDA(cudaGetLastError());
  }
  PairArgs a;
  a.tgt = d_tgt;
  a.nt = nt;
  a.src = d_src;
  a.ns = ns;
  a.bounds = mixed ? bounds : nullptr;
  a.eta = eta;
  a.near_dist = std::max(g_near_k * eta, 1e-9);
  a.n_tiles = n_tiles;
  a.n_splits = n_splits;
  a.split_len = split_len;
  a.part_re = part;
  a.part_im = part + (size_t)n_splits * nt;
  a.err = err;
  a.use_tma = ((uintptr_t)d_src % 16 == 0) ? 1 : 0;
  if (mixed) pair_sum_kernel<true, R_MIXED><<<grid, NT, 0, s>>>(a);
  else pair_sum_kernel<false, R_F64><<<grid, NT, 0, s>>>(a);
  SHRK_CUDA(cudaGetLastError());
  reduce_flagged_kernel<<<(unsigned)((nt + 255) / 256), 256, 0, s>>>(
      a.part_re, a.part_im, n_splits, nt, err, d_re, d_im);
  SHRK_CUDA(cudaGetLastError());
  return SHRK_OK;
}

}  // namespace shrk
