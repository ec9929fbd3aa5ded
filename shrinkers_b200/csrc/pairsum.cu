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
// packed f32x2 pipe -- two targets x two sources per step, one MUFU
// reciprocal per two sources (pairs32x4 in pairs.cuh), FP32 partials folded
// into FP64 every 16 sources with the reciprocal's measured mean error taken
// out at the fold.  Every other pair (the near field, where the
// terms are large and d cancels) is summed in FP64, as are all reductions.
#include "common.cuh"
#include "epilogue.cuh"
#include "internal.h"
#include "pair_item.cuh"
#include "pairs.cuh"

#include <algorithm>
#include <atomic>
#include <cmath>

namespace shrk {

namespace {

#ifndef SHRK_R_MIXED
#define SHRK_R_MIXED 4
#endif
#ifndef SHRK_MIXED_CTAS
#define SHRK_MIXED_CTAS 2
#endif

constexpr int NT = PAIR_NT;
constexpr int CH = PAIR_CH;
constexpr int R_F64 = 4;
constexpr int R_MIXED = SHRK_R_MIXED;
constexpr int R_SMALL_F64 = 1;    // targets per thread below one full tile
constexpr int R_SMALL_MIXED = 2;  // the packed far field takes target pairs

double g_near_k = SHRK_NEAR_K;
// Budget of the pair kernels' bulk-copy waits (clock cycles); changed only by
// shrk_diag_set_wait_limit to exercise the timeout path.
std::atomic<long long> g_wait_cycles{WAIT_CYCLES_DEFAULT};

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
  int64_t split_len;       // multiple of CH (of SUB below one full tile)
  double* part_re;         // [n_splits][nt]
  double* part_im;
  int* err;
  int use_tma;
  long long wait_cycles;   // budget of each bulk-copy wait
};

template <bool MIXED, int R>
__global__ void __launch_bounds__(NT, MIXED ? SHRK_MIXED_CTAS : 2) pair_sum_kernel(const PairArgs a) {
  __shared__ PairStage st;
  pair_stage_init(st);
  uint32_t phase = 0u;    // bit b: expected parity of st.bar[b]
  uint32_t pending = 0u;  // bit b: thread 0 has a copy in flight into st.sbuf[b]
  const int64_t n_items = a.n_tiles * (int64_t)a.n_splits;
  for (int64_t item = blockIdx.x; item < n_items; item += gridDim.x) {
    const int64_t tile = item / a.n_splits;
    const int split = (int)(item % a.n_splits);
    PairItem it;
    it.tgt = a.tgt;
    it.nt = a.nt;
    it.src = a.src;
    it.s0 = (int64_t)split * a.split_len;
    it.s1 = min(a.ns, it.s0 + a.split_len);
    it.tile0 = tile * (NT * R);
    it.eta = a.eta;
    it.near_dist = a.near_dist;
    it.bounds = a.bounds;
    it.out_re = a.part_re + (int64_t)split * a.nt;
    it.out_im = a.part_im + (int64_t)split * a.nt;
    it.err = a.err;
    it.use_tma = a.use_tma != 0;
    it.wait_cycles = a.wait_cycles;
    if (!pair_item<MIXED, R>(it, st, phase, pending)) return;
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

long long set_wait_cycles(long long cycles) {
  return g_wait_cycles.exchange(cycles < 0 ? WAIT_CYCLES_DEFAULT : cycles);
}

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
  // Fewer targets than one full tile (a query grid), or a sum whose full-tile
  // plan has fewer items than the GPU holds CTAs (a small spectrum): the
  // 4-target tiles would leave most of each thread's work on padding or the
  // 1024-source splits would put the whole sum on a few CTAs, so such calls
  // take R_SMALL targets per thread and splits of SUB sources (plain loads,
  // still aligned to the mixed kernel's source blocks).
  const int Rbig = mixed ? R_MIXED : R_F64;
  const int cps = mixed ? SHRK_MIXED_CTAS : 2;
  const SplitPlan big = plan_splits(nt, ns, NT * Rbig, CH, cps);
  const bool small =
      nt < (int64_t)NT * Rbig || big.n_tiles * big.n_splits < (int64_t)sm_count() * cps;
  const int R = small ? (mixed ? R_SMALL_MIXED : R_SMALL_F64) : Rbig;
  const SplitPlan pl = small ? plan_splits(nt, ns, NT * R, SUB, cps) : big;
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
  a.wait_cycles = g_wait_cycles.load();
  {
    LaunchScope ls(mixed ? "pair_sum_mixed" : "pair_sum_f64", s);
    if (mixed && small) pair_sum_kernel<true, R_SMALL_MIXED><<<pl.grid, NT, 0, s>>>(a);
    else if (mixed) pair_sum_kernel<true, R_MIXED><<<pl.grid, NT, 0, s>>>(a);
    else if (small) pair_sum_kernel<false, R_SMALL_F64><<<pl.grid, NT, 0, s>>>(a);
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
  a.wait_cycles = g_wait_cycles.load();
  if (mixed) pair_sum_kernel<true, R_MIXED><<<grid, NT, 0, s>>>(a);
  else pair_sum_kernel<false, R_F64><<<grid, NT, 0, s>>>(a);
  SHRK_CUDA(cudaGetLastError());
  reduce_flagged_kernel<<<(unsigned)((nt + 255) / 256), 256, 0, s>>>(
      a.part_re, a.part_im, n_splits, nt, err, d_re, d_im);
  SHRK_CUDA(cudaGetLastError());
  return SHRK_OK;
}

}  // namespace shrk
