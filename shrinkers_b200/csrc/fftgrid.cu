// FFT grid convolution for the Stieltjes transform on sm_100a: the fft5
// family (fft5 / fft3 / fft2, and the real part of adaptive and dst) and the
// coarse-grid NUFFT preset over the same pipeline.
//
// Replaces the dual-convolution core of src/stieltjes/fft5.rs
// (Fft5Options 213-249, lagrange_weights 136-164, splat 175-185 / 259-318,
// fft_convolution 325-432, interp_at 191-211, interpolate_grid 440-476, entry
// points 559-625), the packing helpers of src/stieltjes/fftplan.rs:43-76 and
// the NUFFT policy of src/stieltjes/nufft.rs (33-126, entry points 164-220).
// Pipeline (all FP64), stencil width N = 2/4/6/8 a template parameter:
//
//   1. runs         a source's stencil cell is i0 = floor((v-lo)/dx); the
//                   sources are sorted, so the cells are too, and one thread
//                   per cell key bisects for first[key] = the first source
//                   with cell >= key (on an integer cell array for large
//                   grids); each run of equal cells gets the sums of its N
//                   stencil weights, from the key's thread, a warp or CTAs
//                   by the run's length.
//   2. pack         one thread per grid cell adds the weights of its sources
//                   (at most 32) run by run in ascending source order -- the
//                   order of the reference's sequential splat, so these
//                   densities are the same sums, without atomics; a denser
//                   cell adds the N run sums.  The N Lagrange weights of
//                   t = pos - i0 are recomputed where they are added
//                   (sources come from L2; no weight array).
//                   packed[c] = density[c] + i x_c/(x_c^2 + eta^2).
//   4. fft          four-step FFT m = m1*m2 (m1, m2 <= 2048): column FFTs of
//                   length m1 in shared memory with the inter-pass twiddle,
//                   then row FFTs of length m2.  Twiddles and the analytic
//                   even-kernel spectrum are device tables cached per grid.
//   5. spectral     unpack the two real spectra (conjugate symmetry), form
//                   Im_hat + i Re_hat = D*K_even + i D*K_odd.
//   6. fft          inverse transform.
//   7. interp       N-point interpolation at the query points, 1/m scale,
//                   fused FP64 epilogue.
#include "common.cuh"
#include "epilogue.cuh"
#include "internal.h"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdlib>
#include <map>
#include <string>

namespace shrk {

namespace {

// nufft.rs:33-58
constexpr double NUFFT_PAD_ETA_MULT = 2000.0;
constexpr double NUFFT_PAD_RANGE_FRAC = 0.75;
constexpr double NUFFT_RESOLUTION = 5.0;
constexpr size_t NUFFT_MIN_GRID = 8192;
constexpr size_t NUFFT_MAX_GRID = 65536;

// fft5.rs:345-353: dx <= eta/8, m >= 8p, at most 2^20 cells.
constexpr size_t FFT5_MAX_AUTO_GRID = (size_t)1 << 20;

constexpr int FFT_MAXL = 2048;                  // longest in-shared-memory transform
constexpr int64_t FFT_MAX_M = (int64_t)FFT_MAXL * FFT_MAXL;

size_t next_pow2(size_t n) {  // mod.rs:529-535
  size_t p = 1;
  while (p < n) p <<= 1;
  return p;
}

// Rust's saturating float -> usize cast (NaN and negatives -> 0).
size_t sat_usize(double v) {
  if (!(v > 0.0)) return 0;
  if (v >= 18446744073709551616.0) return SIZE_MAX;
  return (size_t)v;
}

// fft5.rs:136-164 lagrange_weights<N>, operation order preserved.
template <int N>
__device__ __forceinline__ void lagrange(double t, double w[N]) {
  const double q = (double)(N / 2);
  double pref[N], suf[N], acc = 1.0;
#pragma unroll
  for (int j = 0; j < N; ++j) {
    pref[j] = acc;
    acc *= t - (double)j + q - 1.0;
  }
  acc = 1.0;
#pragma unroll
  for (int j = N - 1; j >= 0; --j) {
    suf[j] = acc;
    acc *= t - (double)j + q - 1.0;
  }
#pragma unroll
  for (int j = 0; j < N; ++j) {
    double den = 1.0;
#pragma unroll
    for (int l = 0; l < N; ++l)
      if (l != j) den *= (double)(j - l);
    w[j] = pref[j] * suf[j] / den;
  }
}

// floor((v - lo)/dx) as a cell index clamped to [-N - 1, m + N] (every slot
// of a source beyond that range lands on the same edge cell), and the
// fraction t = pos - floor(pos) of the unclamped position.
template <int N>
__device__ __forceinline__ int64_t cell_of(double v, double lo, double dx, int64_t m, double* t) {
  const double pos = (v - lo) / dx;
  const double fl = floor(pos);
  *t = pos - fl;
  const double c = fmin(fmax(fl, -(double)N - 1.0), (double)(m + N));
  return (int64_t)c;
}

struct GridArgs {
  const double* src;  // ascending
  int64_t ns;
  int rev;            // 1: visit the sources in descending order (dx < 0)
  double lo, dx, eta;
  int64_t m;
  double2* packed;
  double* dens;       // non-null: write the density alone (the splat stage)
};

template <int N>
__device__ __forceinline__ int clamped_cell(const GridArgs& a, int64_t j, double* t) {
  const double v = a.rev ? a.src[a.ns - 1 - j] : a.src[j];
  const int64_t i0 = cell_of<N>(v, a.lo, a.dx, a.m, t);
  return (int)(i0 < -N ? -N : (i0 > a.m + N ? a.m + N : i0));
}

// Stencil weight k of visited source j (fft5.rs:136-164, 175-185): the same
// arithmetic as the k-th entry of lagrange<N>, recomputed where it is summed
// (k is a compile-time constant at every call, so only that weight's
// operations remain).  Sources are read through L2; no weight array.
template <int N, int K>
__device__ __forceinline__ double weight_of(const GridArgs& a, int64_t j) {
  double t;
  (void)clamped_cell<N>(a, j, &t);
  double w[N];
  lagrange<N>(t, w);
  return w[K];
}

// first[key + N + 1] for every key in [-N - 1, m + N + 1]: the number of
// visited sources whose clamped stencil cell is below key.  Visiting order
// makes the cells non-decreasing, so this is a lower bound found by
// bisection (the same cell computation as everywhere else, so the same runs).
// With `cells` (the clamped cell of every visited source, cells_kernel) the
// probes compare integers instead of each dividing, and start on `coarse`
// (every COARSE-th entry of cells, small enough to stay in L1): the first
// coarse entry at least key brackets the answer within COARSE sources.
constexpr int COARSE = 64;

template <int N>
__device__ __forceinline__ int64_t lower_key(const GridArgs& a, const int* __restrict__ cells,
                                             const int* __restrict__ coarse, int key, int64_t lo,
                                             int64_t hi) {
  if (cells) {
    int64_t blo = 0, bhi = (a.ns + COARSE - 1) / COARSE;
    while (blo < bhi) {
      const int64_t mid = (blo + bhi) >> 1;
      if (__ldg(coarse + mid) < key) blo = mid + 1;
      else bhi = mid;
    }
    // cells[COARSE (blo - 1)] < key <= cells[COARSE blo] (or blo = the end)
    if (blo == 0) return 0;
    lo = COARSE * (blo - 1) + 1;
    hi = COARSE * blo < a.ns ? COARSE * blo : a.ns;
  }
  while (lo < hi) {
    const int64_t mid = (lo + hi) >> 1;
    double t;
    const int c = cells ? __ldg(cells + mid) : clamped_cell<N>(a, mid, &t);
    if (c < key) lo = mid + 1;
    else hi = mid;
  }
  return lo;
}

// cells[j] = the clamped stencil cell of visited source j: one division per
// source, for grids with many keys, whose searches would otherwise divide at
// every probe.
template <int N>
__global__ void cells_kernel(const GridArgs a, int* __restrict__ cells, int* __restrict__ coarse) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j < a.ns; j += stride) {
    double t;
    const int c = clamped_cell<N>(a, j, &t);
    cells[j] = c;
    if (j % COARSE == 0) coarse[j / COARSE] = c;
  }
}

constexpr int DENSE_MIN = 32;   // cells with more sources take their density from run sums
constexpr int RUN_CHUNK = 4096; // long runs are summed in chunks of this many sources, a CTA each

// Run lengths that decide who sums a run: at most `thread_max` sources, the
// key's own thread; up to `warp_max`, a warp; longer runs, CTAs in chunks of
// RUN_CHUNK.  Each run's sum depends only on its length, so it is the same
// from call to call.
struct RunSplit {
  int thread_max;
  int warp_max;
};

// The long runs and their chunks (keys_kernel fills them, long_runs_kernel
// sums them): run r is key idx[r] with nch[r] chunks from the chunk list's
// base[r]; cnt[r] counts its finished chunks; partial[g][k] holds chunk g's
// sums; widx[] lists the keys of the warp-summed runs.  counters[0] / [1] /
// [2] = runs / chunks / warp runs listed (zero on entry).
struct LongRuns {
  int* idx;
  int* base;
  int* nch;
  int* cnt;
  int* chunk_run;  // chunk g -> its run r
  int* widx;
  int* counters;
  double* partial;
};

// Keys and run sums.  A CTA of KEYS_CTA threads serves KEYS_CTA - 1
// consecutive keys: each thread finds first[] of its key, and the end of a
// key's run, first[] of the next key, comes from the next thread through
// shared memory (the last thread of a CTA searches only for that, the next
// CTA's first key), so every thread makes one search.  Then
// S[(e + N + 1) N + k], the sum of stencil weight k over the run, computing
// each source's N weights once in ascending source order -- or, for a longer
// run (RunSplit), lists it for long_runs_kernel: as a warp run, or with its
// chunks of RUN_CHUNK sources.
constexpr int KEYS_CTA = 256;

template <int N>
__global__ void __launch_bounds__(KEYS_CTA) keys_kernel(const GridArgs a, int* __restrict__ first,
                                                        int64_t n_keys, double* __restrict__ S,
                                                        LongRuns L, const int* __restrict__ cells,
                                                        const int* __restrict__ coarse,
                                                        RunSplit rs) {
  __shared__ int first_sh[KEYS_CTA];
  const int64_t idx = (int64_t)blockIdx.x * (KEYS_CTA - 1) + threadIdx.x;
  const int key = (int)(idx - N - 1);
  int64_t j0 = a.ns;
  if (idx <= n_keys) j0 = lower_key<N>(a, cells, coarse, key, 0, a.ns);
  first_sh[threadIdx.x] = (int)j0;
  __syncthreads();
  if (idx > n_keys || threadIdx.x == KEYS_CTA - 1) return;
  first[idx] = (int)j0;
  if (idx == n_keys) return;  // the closing entry (= ns)
  // end of the run: the first source whose cell is at least key + 1 (the
  // next thread's key; idx < n_keys, so that thread searched)
  const int64_t j1 = first_sh[threadIdx.x + 1];
  double t;
  if (j1 - j0 > rs.thread_max && j1 - j0 <= rs.warp_max) {
    L.widx[atomicAdd(L.counters + 2, 1)] = (int)idx;
    return;
  }
  if (j1 - j0 > rs.thread_max) {
    const int nch = (int)((j1 - j0 + RUN_CHUNK - 1) / RUN_CHUNK);
    const int r = atomicAdd(L.counters, 1);
    const int base = atomicAdd(L.counters + 1, nch);
    L.idx[r] = (int)idx;
    L.base[r] = base;
    L.nch[r] = nch;
    L.cnt[r] = 0;
    for (int c = 0; c < nch; ++c) L.chunk_run[base + c] = r;
    return;
  }
  double acc[N];
#pragma unroll
  for (int k = 0; k < N; ++k) acc[k] = 0.0;
  for (int64_t j = j0; j < j1; ++j) {
    double w[N];
    (void)clamped_cell<N>(a, j, &t);
    lagrange<N>(t, w);
#pragma unroll
    for (int k = 0; k < N; ++k) acc[k] += w[k];
  }
#pragma unroll
  for (int k = 0; k < N; ++k) S[idx * N + k] = acc[k];
}

// Run sums of the longer runs.  Runs listed with chunks: a CTA per chunk of
// RUN_CHUNK sources (threads stride the chunk, partials added in a fixed
// order); a run of one chunk writes its sums directly, otherwise the CTA that
// finishes a run's last chunk (a ticket taken after a fence) adds the run's
// chunk partials in chunk order.  Then the warp runs, a warp each.  The
// lists' order varies from call to call; each run's sum does not.
template <int N>
__global__ void __launch_bounds__(256) long_runs_kernel(const GridArgs a,
                                                        const int* __restrict__ first,
                                                        const LongRuns L,
                                                        double* __restrict__ S) {
  __shared__ double red[8][N];
  __shared__ int last;
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  const int n_chunks = L.counters[1];
  for (int g = blockIdx.x; g < n_chunks; g += gridDim.x) {
    const int r = L.chunk_run[g];
    const int64_t idx = L.idx[r];
    const int nch = L.nch[r], c = g - L.base[r];
    const int64_t r0 = first[idx], r1 = first[idx + 1];
    const int64_t j0 = r0 + (int64_t)c * RUN_CHUNK;
    const int64_t j1 = j0 + RUN_CHUNK < r1 ? j0 + RUN_CHUNK : r1;
    double acc[N];
#pragma unroll
    for (int k = 0; k < N; ++k) acc[k] = 0.0;
    for (int64_t j = j0 + threadIdx.x; j < j1; j += blockDim.x) {
      double t, w[N];
      (void)clamped_cell<N>(a, j, &t);
      lagrange<N>(t, w);
#pragma unroll
      for (int k = 0; k < N; ++k) acc[k] += w[k];
    }
#pragma unroll
    for (int k = 0; k < N; ++k) {
      double v = acc[k];
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
      if (lane == 0) red[wib][k] = v;
    }
    __syncthreads();
    if (threadIdx.x < N) {
      double tt = 0.0;
      for (int w = 0; w < (int)(blockDim.x >> 5); ++w) tt += red[w][threadIdx.x];
      if (nch == 1) S[idx * N + threadIdx.x] = tt;
      else L.partial[(int64_t)g * N + threadIdx.x] = tt;
    }
    if (nch > 1) {
      __syncthreads();
      if (threadIdx.x == 0) {
        __threadfence();  // this chunk's partials before its ticket
        last = atomicAdd(L.cnt + r, 1) == nch - 1;
      }
      __syncthreads();
      if (last && threadIdx.x < N) {
        __threadfence();
        const int b0 = L.base[r];
        double tt = 0.0;
        for (int q = 0; q < nch; ++q) tt += __ldcg(L.partial + (int64_t)(b0 + q) * N + threadIdx.x);
        S[idx * N + threadIdx.x] = tt;
      }
    }
    __syncthreads();
  }
  // Warp runs: a warp per run, lanes striding it, the lanes' partials added
  // by a fixed butterfly.
  const int n_warp_runs = L.counters[2];
  const int warps = (int)(blockDim.x >> 5);
  for (int r = blockIdx.x * warps + wib; r < n_warp_runs; r += gridDim.x * warps) {
    const int64_t idx = L.widx[r];
    const int64_t j1 = first[idx + 1];
    double acc[N];
#pragma unroll
    for (int k = 0; k < N; ++k) acc[k] = 0.0;
    for (int64_t j = first[idx] + lane; j < j1; j += 32) {
      double t, w[N];
      (void)clamped_cell<N>(a, j, &t);
      lagrange<N>(t, w);
#pragma unroll
      for (int k = 0; k < N; ++k) acc[k] += w[k];
    }
#pragma unroll
    for (int k = 0; k < N; ++k) {
      double v = acc[k];
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
      if (lane == k) S[idx * N + k] = v;
    }
  }
}

// The density of cell c is the sum of weight k over the run of sources with
// cell c + N/2 - 1 - k, k = N-1 .. 0 (fft5.rs:175-185).  A cell with at most
// DENSE_MIN sources adds them one by one, runs in ascending cell order and
// each run in ascending source order -- the order of the reference's
// sequential splat, so these densities are the same sums, without atomics;
// a denser cell adds the N run sums in that run order (deterministic, not the
// sequential order).  The two edge cells also collect every clamped slot.
// packed[c] = density[c] + i x_c/(x_c^2 + eta^2) (fft5.rs:364-376).
__device__ __forceinline__ void pack_cell(const GridArgs& a, int64_t c, double dens) {
  if (a.dens) {
    a.dens[c] = dens;
    return;
  }
  const int64_t half = a.m / 2;
  const double sd = (c <= half) ? (double)c : (double)c - (double)a.m;
  const double x = sd * a.dx;
  const double denom = x * x + a.eta * a.eta;
  a.packed[c] = make_double2(dens, x / denom);
}

// dens += weight K of every source of the run of cell c + N/2 - 1 - K, for
// K = KK .. 0 in that order.
template <int N, int KK>
__device__ __forceinline__ void run_sums(const GridArgs& a, const int* first, int64_t c,
                                         double& dens) {
  if constexpr (KK >= 0) {
    const int64_t e = c + N / 2 - 1 - KK;
    for (int64_t j = first[e], j1 = first[e + 1]; j < j1; ++j) dens += weight_of<N, KK>(a, j);
    run_sums<N, KK - 1>(a, first, c, dens);
  }
}

template <int N>
__global__ void __launch_bounds__(256) pack_kernel(const GridArgs a, const int* __restrict__ first_all,
                                                   const double* __restrict__ S) {
  constexpr int H = N / 2;
  const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t m = a.m;
  if (c >= m) return;
  const int* first = first_all + N + 1;  // first[key] for key >= -N - 1
  double dens = 0.0;
  if (c > 0 && c < m - 1) {
    const int cnt = first[c + H] - first[c - H];
    if (cnt > DENSE_MIN) {
#pragma unroll
      for (int k = N - 1; k >= 0; --k) dens += S[(c + H - 1 - k + N + 1) * N + k];
    } else {
      run_sums<N, N - 1>(a, first, c, dens);
    }
  } else {
    // edge cell: every slot whose clamped index lands here, sources then slots
    const int64_t j0 = (c == 0) ? 0 : first[m - 1 - H];
    const int64_t j1 = (c == 0) ? first[H] : a.ns;
    for (int64_t j = j0; j < j1; ++j) {
      double t;
      const int i0 = clamped_cell<N>(a, j, &t);
      double w[N];
      lagrange<N>(t, w);
#pragma unroll
      for (int k = 0; k < N; ++k) {
        int64_t cell = (int64_t)i0 - H + 1 + k;
        cell = cell < 0 ? 0 : (cell > m - 1 ? m - 1 : cell);
        if (cell == c) dens += w[k];
      }
    }
  }
  pack_cell(a, c, dens);
}

// The evaluation stage's input: packed[c] from a given density (the sum of
// the splat stages of several source sets).
__global__ void pack_density_kernel(const GridArgs a, const double* __restrict__ density) {
  const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (c < a.m) pack_cell(a, c, density[c]);
}

// ---------------------------------------------------------------- FFT --
// Unnormalised DFT, forward sign e^{-2 pi i jk/m}, inverse e^{+2 pi i jk/m}
// (the contract of the reference's transform, rustfft).  m = m1*m2 by the
// four-step method; each row transform of length L (8 <= L <= 2048) runs in
// shared memory as a mixed-radix Stockham FFT (radix 8, then one radix-4 or
// radix-2 stage): every thread owns 8 elements per stage, the stage twiddles
// come from a per-CTA table, and rows are stored with one pad slot per 8
// elements (and one more per row) so that strided accesses spread over the
// shared-memory banks.
__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double2 cadd(double2 a, double2 b) {
  return make_double2(a.x + b.x, a.y + b.y);
}
__device__ __forceinline__ double2 csub(double2 a, double2 b) {
  return make_double2(a.x - b.x, a.y - b.y);
}
// v * (sign * i)
__device__ __forceinline__ double2 mul_si(double2 v, double sign) {
  return make_double2(-sign * v.y, sign * v.x);
}
__device__ __forceinline__ int padi(int i) { return i + (i >> 3); }

// R-point DFTs in registers, W_R = e^{sign 2 pi i/R}.
__device__ __forceinline__ void dft2(double2* v) {
  const double2 a = v[0], b = v[1];
  v[0] = cadd(a, b);
  v[1] = csub(a, b);
}
__device__ __forceinline__ void dft4(double2& v0, double2& v1, double2& v2, double2& v3,
                                     double sign) {
  const double2 t0 = cadd(v0, v2), t1 = csub(v0, v2), t2 = cadd(v1, v3);
  const double2 t3 = mul_si(csub(v1, v3), sign);
  v0 = cadd(t0, t2);
  v1 = cadd(t1, t3);
  v2 = csub(t0, t2);
  v3 = csub(t1, t3);
}
__device__ __forceinline__ void dft8(double2* v, double sign) {
  const double h = 0.70710678118654752440;  // sqrt(1/2)
  double2 e0 = v[0], e1 = v[2], e2 = v[4], e3 = v[6];
  double2 o0 = v[1], o1 = v[3], o2 = v[5], o3 = v[7];
  dft4(e0, e1, e2, e3, sign);
  dft4(o0, o1, o2, o3, sign);
  o1 = cmul(o1, make_double2(h, sign * h));
  o2 = mul_si(o2, sign);
  o3 = cmul(o3, make_double2(-h, sign * h));
  v[0] = cadd(e0, o0);
  v[1] = cadd(e1, o1);
  v[2] = cadd(e2, o2);
  v[3] = cadd(e3, o3);
  v[4] = csub(e0, o0);
  v[5] = csub(e1, o1);
  v[6] = csub(e2, o2);
  v[7] = csub(e3, o3);
}

// One radix-R Stockham stage over a row of length L (sub-transform length Ns
// so far): thread q of the row does the 8/R butterflies j = q + b*L/8.
template <int R>
__device__ __forceinline__ void fft_stage(double2* row, const double2* tws, int L, int Ns, int q,
                                          double sign) {
  // tws: this stage's twiddles W_{Ns R}^{k r} at [(r - 1) * Ns + k]
  constexpr int B = 8 / R;
  const int tpr = L >> 3;
  double2 v[8];
#pragma unroll
  for (int b = 0; b < B; ++b) {
    const int j = q + b * tpr;
#pragma unroll
    for (int r = 0; r < R; ++r) v[b * R + r] = row[padi(j + r * (L / R))];
  }
  __syncthreads();
#pragma unroll
  for (int b = 0; b < B; ++b) {
    const int j = q + b * tpr;
    const int k = j & (Ns - 1);
    if (Ns > 1) {
#pragma unroll
      for (int r = 1; r < R; ++r) v[b * R + r] = cmul(v[b * R + r], tws[(r - 1) * Ns + k]);
    }
    if (R == 8) dft8(&v[b * R], sign);
    else if (R == 4) dft4(v[b * R], v[b * R + 1], v[b * R + 2], v[b * R + 3], sign);
    else dft2(&v[b * R]);
    const int base = (j - k) * R + k;
#pragma unroll
    for (int r = 0; r < R; ++r) row[padi(base + r * Ns)] = v[b * R + r];
  }
  __syncthreads();
}

// In-place FFT of a padded row of length L >= 8; every thread of the CTA
// calls it (the stages hold barriers).
__device__ void row_fft(double2* row, const double2* tws, int L, int q, double sign) {
  int Ns = 1, rem = L, off = 0;
  while (rem >= 8) {
    fft_stage<8>(row, tws + off, L, Ns, q, sign);
    if (Ns > 1) off += 7 * Ns;
    Ns *= 8;
    rem >>= 3;
  }
  if (rem == 4) fft_stage<4>(row, tws + off, L, Ns, q, sign);
  else if (rem == 2) fft_stage<2>(row, tws + off, L, Ns, q, sign);
}

// Per-stage twiddles for row_fft: for every stage after the first (Ns > 1,
// radix R), W_{Ns R}^{k r} = W_m^{k r m/(Ns R)} for r = 1..R-1, k < Ns, laid
// out [r - 1][k] so that consecutive lanes read consecutive entries; L - 8
// entries in all.  Taken from the length-m table, sign applied.
__device__ __forceinline__ void load_stage_twiddles(double2* tws, const double2* __restrict__ tw,
                                                    int L, int64_t m, double sign) {
  const int total = L - 8;  // <= 8 * blockDim
  double2 w[8];
#pragma unroll
  for (int it = 0; it < 8; ++it) {
    const int idx = threadIdx.x + it * blockDim.x;
    w[it] = make_double2(1.0, 0.0);
    if (idx < total) {
      int off = 0, Ns = 8, rem = L >> 3, R = rem >= 8 ? 8 : rem;
      while (idx >= off + (R - 1) * Ns) {
        off += (R - 1) * Ns;
        Ns *= R;
        rem /= R;
        R = rem >= 8 ? 8 : rem;
      }
      const int r = (idx - off) / Ns + 1, k = (idx - off) & (Ns - 1);
      w[it] = tw[(int64_t)k * r * (m / ((int64_t)Ns * R))];
    }
  }
#pragma unroll
  for (int it = 0; it < 8; ++it) {
    const int idx = threadIdx.x + it * blockDim.x;
    if (idx < total) tws[idx] = make_double2(w[it].x, sign * w[it].y);
  }
}

// Pass 1: Y[k1*m2 + n2] = W_m^{n2 k1} * sum_n1 x[m2 n1 + n2] W_m1^{n1 k1}, for
// G columns n2 per CTA (G*m1/8 threads).
__global__ void __launch_bounds__(256, 4) fft_pass1(const double2* __restrict__ x,
                                                 double2* __restrict__ y, int m1, int m2,
                                                 int64_t m, const double2* __restrict__ tw,
                                                 double sign) {
  extern __shared__ double2 fsm[];
  const int L = m1, Lp = L + (L >> 3) + 1, tpr = L >> 3;
  const int G = blockDim.x / tpr, gl = __ffs(G) - 1;
  double2* tws = fsm + G * Lp;
  load_stage_twiddles(tws, tw, L, m, sign);
  const int n2_0 = blockIdx.x * G;
  // G*L = 8*blockDim: every thread moves exactly 8 elements each way
  double2 v[8];
#pragma unroll
  for (int it = 0; it < 8; ++it) {
    const int e = threadIdx.x + it * blockDim.x;
    const int n1 = e >> gl, g = e & (G - 1);
    v[it] = n2_0 + g < m2 ? x[(int64_t)m2 * n1 + n2_0 + g] : make_double2(0.0, 0.0);
  }
#pragma unroll
  for (int it = 0; it < 8; ++it) {
    const int e = threadIdx.x + it * blockDim.x;
    fsm[(e & (G - 1)) * Lp + padi(e >> gl)] = v[it];
  }
  __syncthreads();
  row_fft(fsm + (threadIdx.x / tpr) * Lp, tws, L, threadIdx.x % tpr, sign);
  // W_m^a = W_m^{a - a mod 1024} * W_m^{a mod 1024}, both from the table;
  // two batches of 4 elements keep the loads in flight within 64 registers
#pragma unroll
  for (int h = 0; h < 8; h += 4) {
    double2 wh[4], wl[4];
#pragma unroll
    for (int it = 0; it < 4; ++it) {
      const int e = threadIdx.x + (h + it) * blockDim.x;
      const int64_t a = ((int64_t)(n2_0 + (e & (G - 1))) * (e >> gl)) & (m - 1);
      wh[it] = tw[a & ~(int64_t)1023];
      wl[it] = tw[a & 1023];
    }
#pragma unroll
    for (int it = 0; it < 4; ++it) {
      const int e = threadIdx.x + (h + it) * blockDim.x;
      const int k1 = e >> gl, g = e & (G - 1);
      const int n2 = n2_0 + g;
      const double2 w = cmul(wh[it], wl[it]);
      if (n2 < m2)
        y[(int64_t)k1 * m2 + n2] = cmul(fsm[g * Lp + padi(k1)], make_double2(w.x, sign * w.y));
    }
  }
}

// Pass 2: X[k1 + m1 k2] = sum_n2 Y[k1*m2 + n2] W_m2^{n2 k2}, G rows per CTA.
__global__ void __launch_bounds__(256, 4) fft_pass2(const double2* __restrict__ y,
                                                 double2* __restrict__ x, int m1, int m2,
                                                 int64_t m, const double2* __restrict__ tw,
                                                 double sign) {
  extern __shared__ double2 fsm[];
  const int L = m2, Lp = L + (L >> 3) + 1, tpr = L >> 3;
  const int G = blockDim.x / tpr, gl = __ffs(G) - 1, ll = __ffs(L) - 1;
  double2* tws = fsm + G * Lp;
  load_stage_twiddles(tws, tw, L, m, sign);
  const int k1_0 = blockIdx.x * G;
  double2 v[8];
#pragma unroll
  for (int it = 0; it < 8; ++it) {
    const int e = threadIdx.x + it * blockDim.x;
    const int g = e >> ll, n2 = e & (L - 1);
    v[it] = k1_0 + g < m1 ? y[(int64_t)(k1_0 + g) * m2 + n2] : make_double2(0.0, 0.0);
  }
#pragma unroll
  for (int it = 0; it < 8; ++it) {
    const int e = threadIdx.x + it * blockDim.x;
    fsm[(e >> ll) * Lp + padi(e & (L - 1))] = v[it];
  }
  __syncthreads();
  row_fft(fsm + (threadIdx.x / tpr) * Lp, tws, L, threadIdx.x % tpr, sign);
#pragma unroll
  for (int it = 0; it < 8; ++it) {
    const int e = threadIdx.x + it * blockDim.x;
    const int k2 = e >> gl, g = e & (G - 1);
    if (k1_0 + g < m1) x[(int64_t)(k1_0 + g) + (int64_t)m1 * k2] = fsm[g * Lp + padi(k2)];
  }
}

// Transforms shorter than 64 points: direct DFT, one thread per output.
__global__ void dft_small(const double2* __restrict__ x, double2* __restrict__ y, int m,
                          const double2* __restrict__ tw, double sign) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= m) return;
  double2 acc = make_double2(0.0, 0.0);
  for (int n = 0; n < m; ++n) {
    const double2 w = tw[((int64_t)n * k) % m];
    acc = cadd(acc, cmul(x[n], make_double2(w.x, sign * w.y)));
  }
  y[k] = acc;
}

// fftplan.rs:43-76: unpack D (density) and K (odd kernel) from the packed
// forward transform, multiply, repack as Im_hat + i Re_hat.
__global__ void spectral_kernel(const double2* __restrict__ C, const double* __restrict__ ke,
                                double2* __restrict__ out, int64_t m) {
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= m) return;
  const double2 ck = C[k];
  const double2 cn = C[(m - k) % m];
  const double2 cnc = make_double2(cn.x, -cn.y);
  const double2 s = make_double2(ck.x + cnc.x, ck.y + cnc.y);
  const double2 df = make_double2(ck.x - cnc.x, ck.y - cnc.y);
  const double2 D = make_double2(0.5 * s.x, 0.5 * s.y);
  const double2 K = make_double2(0.5 * df.y, -0.5 * df.x);  // (-0.5 i) * df
  const double ih_re = D.x * ke[k], ih_im = D.y * ke[k];
  const double2 rh = cmul(D, K);
  out[k] = make_double2(ih_re - rh.y, ih_im + rh.x);
}

struct InterpArgs {
  const double* q;
  int64_t nq;
  const double2* grid;
  int64_t m;
  double lo, dx, inv_m;
  Epilogue epi;
};

// fft5.rs:191-211 interp_at<N> + 440-476: re <- .im, im <- .re, times 1/m.
template <int N>
__global__ void interp_kernel(const InterpArgs a) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= a.nq) return;
  const double qv = a.q[t];
  double tt;
  const int64_t i0 = cell_of<N>(qv, a.lo, a.dx, a.m, &tt);
  double w[N];
  lagrange<N>(tt, w);
  double ra = 0.0, ia = 0.0;
#pragma unroll
  for (int j = 0; j < N; ++j) {
    int64_t cell = i0 - N / 2 + 1 + j;
    cell = cell < 0 ? 0 : (cell > a.m - 1 ? a.m - 1 : cell);
    const double2 g = a.grid[cell];
    ia += g.x * w[j];
    ra += g.y * w[j];
  }
  epi_store(a.epi, t, qv, ra * a.inv_m, ia * a.inv_m);
}

// Twiddles (cos 2 pi j/m, sin 2 pi j/m) for j < m.
__global__ void twiddle_kernel(double2* tw, int64_t m) {
  const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= m) return;
  double s, c;
  sincospi(2.0 * (double)j / (double)m, &s, &c);
  tw[j] = make_double2(c, s);
}

// fft5.rs:404-416: K_even[k] = (pi/dx) r^|k|, |k| = min(k, m - k),
// r = exp(-2 pi eta/(m dx)).  The power is evaluated directly, not by the
// reference's running product (the two differ by that product's rounding,
// at most |k| ulp).
__global__ void even_kernel_spectrum(double* ke, int64_t m, double ke0, double r) {
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= m) return;
  const int64_t half = m / 2;
  const int64_t kk = k <= half ? k : m - k;
  ke[k] = ke0 * pow(r, (double)kk);
}

// Grids whose size m is not a power of two (a forced fft5 grid_size; the
// reference plans any length through rustfft, fftplan.rs:21-28) take
// Bluestein's chirp-z form over the power-of-two transform of length
// M = next_pow2(2m - 1):  with c_j = e^{i pi j^2/m} and nk = (n^2 + k^2 -
// (k - n)^2)/2,
//   y_k = sum_n x_n e^{s 2 pi i nk/m} = c_k^s sum_n (x_n c_n^s) conj(c^s)_{k-n},
// a circular convolution of length M with the chirp filter, which is
// transformed once per m.  c^s is c for s = +1 and its conjugate for s = -1.

// c_j = e^{i pi (j^2 mod 2m)/m}, j < m; j^2 is exact in 64-bit integers for
// the m this path admits (m <= 2^21).
__global__ void chirp_kernel(double2* c, int64_t m) {
  const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= m) return;
  const int64_t r = (j * j) % (2 * m);
  double sn, cs;
  sincospi((double)r / (double)m, &sn, &cs);
  c[j] = make_double2(cs, sn);
}

// The forward transform's filter conj(c^{-1})_j = c_j on the circular index
// range (-m, m) of length M, scaled by 1/M (a power of two: exact) so that
// the unnormalised inverse transform of the product is the convolution.
__global__ void chirp_filter_kernel(const double2* __restrict__ c, int64_t m, int64_t M,
                                    double2* __restrict__ b) {
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= M) return;
  const int64_t j = k < m ? k : (k > M - m ? M - k : -1);
  const double inv = 1.0 / (double)M;
  b[k] = j >= 0 ? make_double2(c[j].x * inv, c[j].y * inv) : make_double2(0.0, 0.0);
}

// a_n = x_n c^s_n for n < m, zero up to M.
__global__ void chirp_in_kernel(const double2* __restrict__ x, const double2* __restrict__ c,
                                int64_t m, int64_t M, double sign, double2* __restrict__ a) {
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= M) return;
  a[k] = k < m ? cmul(x[k], make_double2(c[k].x, sign * c[k].y)) : make_double2(0.0, 0.0);
}

// a_k *= B_k for the forward transform; for the inverse the filter is the
// conjugate chirp, whose transform is conj(B_{-k mod M}).
__global__ void chirp_mul_kernel(double2* __restrict__ a, const double2* __restrict__ bhat,
                                 int64_t M, int inverse) {
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= M) return;
  double2 h = bhat[inverse ? (M - k) & (M - 1) : k];
  if (inverse) h.y = -h.y;
  a[k] = cmul(a[k], h);
}

// y_k = c^s_k a_k, k < m.
__global__ void chirp_out_kernel(const double2* __restrict__ a, const double2* __restrict__ c,
                                 int64_t m, double sign, double2* __restrict__ y) {
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= m) return;
  y[k] = cmul(a[k], make_double2(c[k].x, sign * c[k].y));
}

// Length of the power-of-two (or direct, below 64 points) transform that
// serves a grid of m cells.
int64_t transform_len(int64_t m) {
  if (m < 64 || (m & (m - 1)) == 0) return m;
  return (int64_t)next_pow2((size_t)(2 * m - 1));
}

// Constant tables, cached per call context for the last transform length,
// m and (m, dx, eta); written and read on the context's stream.
struct Tables {
  double2* tw = nullptr;     // twiddles of the transform length
  int64_t tw_m = 0;
  double2* chirp = nullptr;  // Bluestein: c_j (m) and the filter's transform (M)
  double2* bhat = nullptr;
  int64_t bs_m = 0, bs_cap = 0, bhat_cap = 0;
  double* ke = nullptr;
  int64_t ke_cap = 0;
  int64_t ke_m = 0;
  double ke_dx = 0.0, ke_eta = 0.0;
  ~Tables() {
    if (tw) cudaFree(tw);
    if (chirp) cudaFree(chirp);
    if (bhat) cudaFree(bhat);
    if (ke) cudaFree(ke);
  }
};

unsigned blocks_for(int64_t n, int t) { return (unsigned)((n + t - 1) / t); }

shrk_status fft(double2* buf, double2* tmp, int64_t m, const double2* tw, double sign,
                const char* family, cudaStream_t s);

shrk_status ensure_tables(int64_t m, double dx, double eta, const char* family, cudaStream_t s,
                          Tables** out) {
  Tables& T = ctx_state<Tables>(EXT_FFT_TABLES);
  const int64_t L = transform_len(m);
  if (T.tw_m != L) {
    if (T.tw) SHRK_CUDA(cudaFree(T.tw));
    T.tw = nullptr;
    T.tw_m = 0;
    SHRK_CUDA(cudaMalloc(&T.tw, sizeof(double2) * L));
    twiddle_kernel<<<blocks_for(L, 256), 256, 0, s>>>(T.tw, L);
    SHRK_CUDA(cudaGetLastError());
    T.tw_m = L;
  }
  if (L != m && T.bs_m != m) {
    T.bs_m = 0;
    if (T.bs_cap < m) {
      if (T.chirp) SHRK_CUDA(cudaFree(T.chirp));
      T.chirp = nullptr;
      T.bs_cap = 0;
      SHRK_CUDA(cudaMalloc(&T.chirp, sizeof(double2) * m));
      T.bs_cap = m;
    }
    if (T.bhat_cap < 2 * L) {  // the filter's transform and its scratch
      if (T.bhat) SHRK_CUDA(cudaFree(T.bhat));
      T.bhat = nullptr;
      T.bhat_cap = 0;
      SHRK_CUDA(cudaMalloc(&T.bhat, sizeof(double2) * 2 * L));
      T.bhat_cap = 2 * L;
    }
    chirp_kernel<<<blocks_for(m, 256), 256, 0, s>>>(T.chirp, m);
    SHRK_CUDA(cudaGetLastError());
    chirp_filter_kernel<<<blocks_for(L, 256), 256, 0, s>>>(T.chirp, m, L, T.bhat);
    SHRK_CUDA(cudaGetLastError());
    SHRK_TRY(fft(T.bhat, T.bhat + L, L, T.tw, -1.0, family, s));
    T.bs_m = m;
  }
  if (T.ke_m != m || T.ke_dx != dx || T.ke_eta != eta) {
    if (T.ke_cap < m) {
      if (T.ke) SHRK_CUDA(cudaFree(T.ke));
      T.ke = nullptr;
      T.ke_cap = 0;
      SHRK_CUDA(cudaMalloc(&T.ke, sizeof(double) * m));
      T.ke_cap = m;
    }
    const double r = std::exp(-2.0 * M_PI * eta / ((double)m * dx));
    even_kernel_spectrum<<<blocks_for(m, 256), 256, 0, s>>>(T.ke, m, M_PI / dx, r);
    SHRK_CUDA(cudaGetLastError());
    T.ke_m = m;
    T.ke_dx = dx;
    T.ke_eta = eta;
  }
  *out = &T;
  return SHRK_OK;
}

int ilog2(int64_t v) {
  int b = 0;
  while ((int64_t(1) << b) < v) ++b;
  return b;
}

// Rows per CTA for a pass over `rows` transforms of length L: as many as fit
// 256 threads (8 elements each), but no more than keeps ~2 CTAs per SM.
int rows_per_cta(int L, int rows) {
  const int cap = 2048 / L;
  int g = 1;
  while (g * 2 <= cap && (int64_t)rows / (g * 2) >= 296) g *= 2;
  return g;
}

size_t pass_smem(int L, int G) {
  return sizeof(double2) * ((size_t)G * (L + (L >> 3) + 1) + L);
}

shrk_status fft(double2* buf, double2* tmp, int64_t m, const double2* tw, double sign,
                const char* family, cudaStream_t s) {
  if (m < 64) {
    LaunchScope ls(family, s);
    dft_small<<<1, 64, 0, s>>>(buf, tmp, (int)m, tw, sign);
    SHRK_CUDA(cudaGetLastError());
    SHRK_CUDA(cudaMemcpyAsync(buf, tmp, sizeof(double2) * m, cudaMemcpyDeviceToDevice, s));
    return SHRK_OK;
  }
  const int bits = ilog2(m);
  const int m1 = 1 << ((bits + 1) / 2), m2 = 1 << (bits / 2);
  static std::atomic<bool> opted[64];
  int dev = 0;
  SHRK_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64 || !opted[dev].load()) {
    const int big = (int)pass_smem(FFT_MAXL, 1);
    SHRK_CUDA(cudaFuncSetAttribute(fft_pass1, cudaFuncAttributeMaxDynamicSharedMemorySize, big));
    SHRK_CUDA(cudaFuncSetAttribute(fft_pass2, cudaFuncAttributeMaxDynamicSharedMemorySize, big));
    if (dev >= 0 && dev < 64) opted[dev] = true;
  }
  {
    const int G = rows_per_cta(m1, m2);
    LaunchScope ls(family, s);
    fft_pass1<<<blocks_for(m2, G), G * (m1 >> 3), pass_smem(m1, G), s>>>(buf, tmp, m1, m2, m, tw,
                                                                        sign);
    SHRK_CUDA(cudaGetLastError());
  }
  {
    const int G = rows_per_cta(m2, m1);
    LaunchScope ls(family, s);
    fft_pass2<<<blocks_for(m1, G), G * (m2 >> 3), pass_smem(m2, G), s>>>(tmp, buf, m1, m2, m, tw,
                                                                        sign);
    SHRK_CUDA(cudaGetLastError());
  }
  return SHRK_OK;
}

// Unnormalised DFT of the m-cell grid in buf (sign -1 forward, +1 inverse):
// the power-of-two transform in place, or Bluestein's form through the
// M-point work buffers wa and wt.
shrk_status dft(double2* buf, int64_t m, const Tables* T, double sign, double2* wa, double2* wt,
                const char* family, cudaStream_t s) {
  const int64_t M = transform_len(m);
  if (M == m) return fft(buf, wt, m, T->tw, sign, family, s);
  {
    LaunchScope ls(family, s);
    chirp_in_kernel<<<blocks_for(M, 256), 256, 0, s>>>(buf, T->chirp, m, M, sign, wa);
    SHRK_CUDA(cudaGetLastError());
  }
  SHRK_TRY(fft(wa, wt, M, T->tw, -1.0, family, s));
  {
    LaunchScope ls(family, s);
    chirp_mul_kernel<<<blocks_for(M, 256), 256, 0, s>>>(wa, T->bhat, M, sign > 0.0 ? 1 : 0);
    SHRK_CUDA(cudaGetLastError());
  }
  SHRK_TRY(fft(wa, wt, M, T->tw, +1.0, family, s));
  {
    LaunchScope ls(family, s);
    chirp_out_kernel<<<blocks_for(m, 256), 256, 0, s>>>(wa, T->chirp, m, sign, buf);
    SHRK_CUDA(cudaGetLastError());
  }
  return SHRK_OK;
}

// One grid: stencil width, size, origin and spacing, and the launch families
// its kernels are timed under.
struct GridPlan {
  int order;
  int64_t m;
  double lo, dx;
  const char* fam_splat;
  const char* fam_fft;
  const char* fam_spectral;
  const char* fam_interp;
};

template <int N>
shrk_status eval_grid(double2* A, double2* B, double2* Wa, double2* Wt, const Tables* T,
                      const double* d_q, int64_t nq, const GridPlan& g, const Epilogue& epi,
                      cudaStream_t s);

// Splat tuning, read once: SHRK_SPLAT_CELLS (0 / 1: the key searches on a
// cell array off / on; default: on when the keys outnumber one wave of
// resident threads), SHRK_SPLAT_THREAD_MAX and SHRK_SPLAT_WARP_MAX (the
// RunSplit bounds; default 8 and 256, measured at p = 10^6 on the NUFFT's
// 65 536-cell grid and the fft5 grid of 2^20 cells).
struct SplatTuning {
  int cells = -1;
  RunSplit rs{8, 256};
};

const SplatTuning& splat_tuning() {
  static const SplatTuning t = [] {
    SplatTuning v;
    if (const char* e = std::getenv("SHRK_SPLAT_CELLS")) v.cells = std::atoi(e) != 0 ? 1 : 0;
    if (const char* e = std::getenv("SHRK_SPLAT_THREAD_MAX")) v.rs.thread_max = std::max(0, std::atoi(e));
    if (const char* e = std::getenv("SHRK_SPLAT_WARP_MAX")) v.rs.warp_max = std::atoi(e);
    v.rs.warp_max = std::max(v.rs.warp_max, v.rs.thread_max);
    return v;
  }();
  return t;
}

// The whole grid convolution, or one of its two stages: with dens_out the
// splat alone (the density of the sources into dens_out[m], nothing else);
// with dens_in the evaluation alone from that density (no sources read).
template <int N>
shrk_status run_grid(const double* d_q, int64_t nq, const double* d_src, int64_t ns, double eta,
                     const GridPlan& g, const Epilogue& epi, cudaStream_t s,
                     const double* dens_in, double* dens_out) {
  const int64_t m = g.m;
  Tables* T = nullptr;
  if (!dens_out) SHRK_TRY(ensure_tables(m, g.dx, eta, g.fam_fft, s, &T));
  // slot 11: A (packed grid) | B (product) | Wt | Wa, the last two of the
  // transform length (Wa only for a Bluestein grid)
  const int64_t L = transform_len(m);
  void* w = nullptr;
  SHRK_TRY(scratch_get(11, sizeof(double2) * (size_t)(2 * m + (L == m ? L : 2 * L)), &w));
  double2* A = (double2*)w;
  double2* B = A + m;
  double2* Wt = B + m;
  double2* Wa = Wt + L;
  GridArgs ga{d_src, ns, g.dx < 0.0 ? 1 : 0, g.lo, g.dx, eta, m, A, dens_out};
  if (dens_in) {
    LaunchScope ls(g.fam_splat, s);
    pack_density_kernel<<<blocks_for(m, 256), 256, 0, s>>>(ga, dens_in);
    SHRK_CUDA(cudaGetLastError());
    return eval_grid<N>(A, B, Wa, Wt, T, d_q, nq, g, epi, s);
  }
  if (ns == 0) {  // no sources: a zero density
    if (dens_out) SHRK_CUDA(cudaMemsetAsync(dens_out, 0, sizeof(double) * m, s));
    return SHRK_OK;
  }
  // slot 24: first [K + 1] | long runs: idx, base, nch, cnt, warp runs [K]
  // each | three counters | chunk list [C] | source cells [ns] (when used) |
  // run sums [K][N] | chunk partials [C][N], K = m + 2N + 2 keys from
  // -N - 1, C = ns / RUN_CHUNK + K chunks at most (a chunked run of n sources
  // has ceil(n / RUN_CHUNK)); the source cells are followed by their coarse
  // table [ceil(ns / COARSE)]
  const int64_t n_keys = m + 2 * N + 2;
  const int64_t max_chunks = ns / RUN_CHUNK + n_keys;
  const SplatTuning& st = splat_tuning();
  const bool use_cells =
      st.cells >= 0 ? st.cells != 0 : (n_keys + 1) > (int64_t)sm_count() * 2048;
  const size_t n_coarse = (size_t)((ns + COARSE - 1) / COARSE);
  const size_t int_bytes =
      ((sizeof(int) * (6 * (size_t)n_keys + 4 + (size_t)max_chunks +
                       (use_cells ? (size_t)ns + n_coarse : 0))) +
       255) & ~(size_t)255;
  void* sw = nullptr;
  SHRK_TRY(scratch_get(24, int_bytes + sizeof(double) * N * ((size_t)n_keys + (size_t)max_chunks),
                       &sw));
  int* first = (int*)sw;
  LongRuns lr;
  lr.idx = first + n_keys + 1;
  lr.base = lr.idx + n_keys;
  lr.nch = lr.base + n_keys;
  lr.cnt = lr.nch + n_keys;
  lr.widx = lr.cnt + n_keys;
  lr.counters = lr.widx + n_keys;
  lr.chunk_run = lr.counters + 3;
  int* cells = use_cells ? lr.chunk_run + max_chunks : nullptr;
  int* coarse = use_cells ? cells + ns : nullptr;
  double* runs = (double*)((char*)sw + int_bytes);
  lr.partial = runs + (size_t)N * n_keys;
  SHRK_CUDA(cudaMemsetAsync(lr.counters, 0, 3 * sizeof(int), s));
  if (use_cells) {
    LaunchScope ls(g.fam_splat, s);
    const int64_t blocks = std::min<int64_t>((ns + 255) / 256, (int64_t)sm_count() * 8);
    cells_kernel<N><<<(unsigned)blocks, 256, 0, s>>>(ga, cells, coarse);
    SHRK_CUDA(cudaGetLastError());
  }
  {
    LaunchScope ls(g.fam_splat, s);
    keys_kernel<N><<<blocks_for(n_keys + 1, KEYS_CTA - 1), KEYS_CTA, 0, s>>>(ga, first, n_keys,
                                                                             runs, lr, cells, coarse,
                                                                             st.rs);
    SHRK_CUDA(cudaGetLastError());
  }
  {
    LaunchScope ls(g.fam_splat, s);
    long_runs_kernel<N><<<sm_count() * 4, 256, 0, s>>>(ga, first, lr, runs);
    SHRK_CUDA(cudaGetLastError());
  }
  {
    LaunchScope ls(g.fam_splat, s);
    pack_kernel<N><<<blocks_for(m, 256), 256, 0, s>>>(ga, first, runs);
    SHRK_CUDA(cudaGetLastError());
  }
  if (dens_out) return SHRK_OK;
  return eval_grid<N>(A, B, Wa, Wt, T, d_q, nq, g, epi, s);
}

// Forward transform of the packed grid A, spectral product into B, inverse
// transform, interpolation at the queries with the epilogue.
template <int N>
shrk_status eval_grid(double2* A, double2* B, double2* Wa, double2* Wt, const Tables* T,
                      const double* d_q, int64_t nq, const GridPlan& g, const Epilogue& epi,
                      cudaStream_t s) {
  const int64_t m = g.m;
  SHRK_TRY(dft(A, m, T, -1.0, Wa, Wt, g.fam_fft, s));
  {
    LaunchScope ls(g.fam_spectral, s);
    spectral_kernel<<<blocks_for(m, 256), 256, 0, s>>>(A, T->ke, B, m);
    SHRK_CUDA(cudaGetLastError());
  }
  SHRK_TRY(dft(B, m, T, +1.0, Wa, Wt, g.fam_fft, s));
  InterpArgs ia{d_q, nq, B, m, g.lo, g.dx, 1.0 / (double)m, epi};
  {
    LaunchScope ls(g.fam_interp, s);
    interp_kernel<N><<<blocks_for(nq, 256), 256, 0, s>>>(ia);
    SHRK_CUDA(cudaGetLastError());
  }
  return SHRK_OK;
}

shrk_status run_grid_order(const double* d_q, int64_t nq, const double* d_src, int64_t ns,
                           double eta, const GridPlan& g, const Epilogue& epi, cudaStream_t s,
                           const double* dens_in = nullptr, double* dens_out = nullptr) {
  // the first-source table and the run lists index sources with 32-bit ints
  if (ns > (int64_t)INT32_MAX) {
    set_error("fft grid methods: at most 2^31 - 1 sources per call");
    return SHRK_EINVAL;
  }
  switch (g.order) {
    case 2: return run_grid<2>(d_q, nq, d_src, ns, eta, g, epi, s, dens_in, dens_out);
    case 4: return run_grid<4>(d_q, nq, d_src, ns, eta, g, epi, s, dens_in, dens_out);
    case 6: return run_grid<6>(d_q, nq, d_src, ns, eta, g, epi, s, dens_in, dens_out);
    case 8: return run_grid<8>(d_q, nq, d_src, ns, eta, g, epi, s, dens_in, dens_out);
    default:
      set_error("fft5: the stencil order must be 2, 4, 6 or 8 nodes");
      return SHRK_EINVAL;
  }
}

}  // namespace

// nufft.rs:106-126 grid_size_for_range.
size_t nufft_grid_size(double raw_range, double eta) {
  double pad = std::max(NUFFT_PAD_ETA_MULT * eta, NUFFT_PAD_RANGE_FRAC * raw_range);
  double range = raw_range + 2.0 * pad;
  size_t max_grid = std::max(std::max(NUFFT_MAX_GRID, NUFFT_MIN_GRID), (size_t)2);
  double target = NUFFT_RESOLUTION * range / eta;
  target = std::isfinite(target) ? std::min(target, (double)max_grid) : (double)max_grid;
  return std::min(next_pow2(std::max((size_t)std::ceil(target), NUFFT_MIN_GRID)), max_grid);
}

// fft5.rs:339-361: pad = max(pad_eta_mult eta, pad_range_frac raw_range),
// m = next_pow2(min(max(ceil(8 range/eta), 8p), 2^20)), at least 2.
size_t fft5_grid_size(double lo_raw, double hi_raw, size_t p, double eta, double pad_eta_mult,
                      double pad_range_frac) {
  const double raw_range = hi_raw - lo_raw;
  const double pad = std::max(pad_eta_mult * eta, pad_range_frac * raw_range);
  const double lo = lo_raw - pad, hi = hi_raw + pad;
  const double range = hi - lo;
  size_t min_grid = sat_usize(std::ceil(8.0 * range / eta));
  const size_t p8 = p > SIZE_MAX / 8 ? SIZE_MAX : 8 * p;
  min_grid = std::min(std::max(min_grid, p8), FFT5_MAX_AUTO_GRID);
  return std::max(next_pow2(min_grid), (size_t)2);
}

// fft5.rs:339-361 with the NUFFT options (m fixed by the policy).
void nufft_geometry(double lo_raw, double hi_raw, double eta, int64_t* m, double* lo,
                    double* dx) {
  const double raw_range = hi_raw - lo_raw;
  *m = (int64_t)std::max(nufft_grid_size(raw_range, eta), (size_t)2);
  const double pad = std::max(NUFFT_PAD_ETA_MULT * eta, NUFFT_PAD_RANGE_FRAC * raw_range);
  *lo = lo_raw - pad;
  const double hi = hi_raw + pad;
  *dx = (hi - *lo) / (double)*m;
}

namespace {
GridPlan nufft_plan(int64_t m, double lo, double dx) {
  return GridPlan{4, m, lo, dx, "nufft_splat", "nufft_fft", "nufft_spectral", "nufft_interp"};
}
}  // namespace

shrk_status nufft_points(const double* d_q, int64_t nq, const double* d_src, int64_t ns,
                         double lo_raw, double hi_raw, double eta, const Epilogue& epi,
                         cudaStream_t s) {
  if (nq <= 0 || ns <= 0) return SHRK_OK;
  int64_t m = 0;
  double lo = 0.0, dx = 0.0;
  nufft_geometry(lo_raw, hi_raw, eta, &m, &lo, &dx);
  return run_grid_order(d_q, nq, d_src, ns, eta, nufft_plan(m, lo, dx), epi, s);
}

shrk_status nufft_density(const double* d_sorted_src, int64_t ns, int64_t m, double lo, double dx,
                          double* d_density, cudaStream_t s) {
  return run_grid_order(nullptr, 0, d_sorted_src, ns, 0.0, nufft_plan(m, lo, dx), Epilogue{}, s,
                        nullptr, d_density);
}

shrk_status nufft_eval(const double* d_density, int64_t m, double lo, double dx, double eta,
                       const double* d_q, int64_t nq, const Epilogue& epi, cudaStream_t s) {
  if (nq <= 0) return SHRK_OK;
  return run_grid_order(d_q, nq, nullptr, 0, eta, nufft_plan(m, lo, dx), epi, s, d_density,
                        nullptr);
}

shrk_status fft5_points(const double* d_q, int64_t nq, const double* d_src, int64_t ns,
                        double lo_raw, double hi_raw, double eta, const Fft5Opts& o,
                        const Epilogue& epi, cudaStream_t s) {
  if (nq <= 0 || ns <= 0) return SHRK_OK;
  const size_t m = o.m_override ? std::max(o.m_override, (size_t)2)
                                : fft5_grid_size(lo_raw, hi_raw, (size_t)ns, eta, o.pad_eta_mult,
                                                 o.pad_range_frac);
  if (m > (size_t)FFT_MAX_M || ((m & (m - 1)) != 0 && m > (size_t)FFT_MAX_M / 2)) {
    set_error("fft5: the grid size must be at most 2^22, or 2^21 when it is not a power of "
              "two (got " + std::to_string(m) + ")");
    return SHRK_ENOTIMPL;
  }
  const double raw_range = hi_raw - lo_raw;
  const double pad = std::max(o.pad_eta_mult * eta, o.pad_range_frac * raw_range);
  const double lo = lo_raw - pad, hi = hi_raw + pad;
  const double range = hi - lo;
  GridPlan g{o.order, (int64_t)m, lo, range / (double)m, "fft5_splat", "fft5_fft",
             "fft5_spectral", "fft5_interp"};
  return run_grid_order(d_q, nq, d_src, ns, eta, g, epi, s);
}

}  // namespace shrk
