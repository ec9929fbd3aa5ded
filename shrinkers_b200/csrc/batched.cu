// Batched exact transform of many spectra of uneven size in one persistent
// launch (no reference counterpart: it replaces a host loop of
// compute_all_stieltjes calls, src/stieltjes/mod.rs:601-790, one per
// spectrum).
//
// Spectrum s is ev[off_s .. off_s + p_s), evaluated at its own points with
// its own eta_s and scaled by 1/p_s.  The host splits every spectrum into
// (target tile x source split) work items -- tile = 256*R targets, split =
// SL sources, with (R, SL) taken per p-bucket from an autotuned table -- and
// sorts the items by cost, largest first.  A persistent grid (2 CTAs per SM)
// pulls items from a device counter, sums each with the same item body as
// the single-transform kernel (pair_item.cuh) into a per-split partial slab,
// and a per-spectrum kernel reduces the slabs in a fixed order (results do
// not depend on which CTA took which item).  The whole sequence (counter
// reset, block bounds, persistent kernel, reduction) is captured once per
// plan in a CUDA graph and replayed while the plan and buffers repeat.
#include "common.cuh"
#include "internal.h"
#include "pair_item.cuh"
#include "pairs.cuh"

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <iterator>
#include <mutex>
#include <string>
#include <vector>

namespace shrk {
namespace {

constexpr int NB = 8;            // p-buckets: [2^8, 2^9), ..., [2^15, inf)
constexpr int B_CTAS = 2;        // persistent CTAs per SM
constexpr int TUNE_R[] = {2, 4};
constexpr int TUNE_SL[] = {1024, 2048, 4096, 8192};

struct SpecDesc {
  int64_t off;         // first value of the spectrum
  int64_t p;
  int64_t part_base;   // first partial of split 0 (slab k at part_base + k*p)
  int64_t block_base;  // first SUB-block bound
  int split_len;       // SL (multiple of PAIR_CH)
  int R;               // targets per thread (2 or 4)
};

struct BItem {
  int spec, tile, split, pad;
};

struct BatchArgs {
  const double* ev;
  const double* eta;
  const SpecDesc* spec;
  const BItem* items;
  int n_items;
  int* counter;
  const double2* bounds;
  double* part_re;
  double* part_im;
  double near_k;
  int* err;
};

// (min, max) of every SUB-block of every spectrum; one CTA per spectrum.
__global__ void batched_bounds_kernel(const double* __restrict__ ev,
                                      const SpecDesc* __restrict__ spec,
                                      double2* __restrict__ bounds) {
  const SpecDesc d = spec[blockIdx.x];
  const int64_t nb = (d.p + SUB - 1) / SUB;
  for (int64_t b = threadIdx.x; b < nb; b += blockDim.x) {
    const int64_t b0 = b * SUB, b1 = min(d.p, b0 + SUB);
    double mn = INFINITY, mx = -INFINITY;
    for (int64_t i = b0; i < b1; ++i) {
      const double v = ev[d.off + i];
      mn = fmin(mn, v);
      mx = fmax(mx, v);
    }
    bounds[d.block_base + b] = make_double2(mn, mx);
  }
}

template <bool MIXED>
__global__ void __launch_bounds__(PAIR_NT, B_CTAS) batched_kernel(const BatchArgs a) {
  __shared__ PairStage st;
  __shared__ int s_item;
  pair_stage_init(st);
  uint32_t phase = 0u, pending = 0u;
  for (;;) {
    if (threadIdx.x == 0) s_item = atomicAdd(a.counter, 1);
    __syncthreads();
    const int i = s_item;
    __syncthreads();
    if (i >= a.n_items) return;
    const BItem w = a.items[i];
    const SpecDesc d = a.spec[w.spec];
    PairItem it;
    it.tgt = a.ev + d.off;
    it.nt = d.p;
    it.src = it.tgt;
    it.s0 = (int64_t)w.split * d.split_len;
    it.s1 = min(d.p, it.s0 + d.split_len);
    it.tile0 = (int64_t)w.tile * PAIR_NT * d.R;
    it.eta = a.eta[w.spec];
    it.near_dist = fmax(a.near_k * it.eta, 1e-9);
    it.bounds = a.bounds + d.block_base;
    it.out_re = a.part_re + d.part_base + (int64_t)w.split * d.p;
    it.out_im = a.part_im + d.part_base + (int64_t)w.split * d.p;
    it.err = a.err;
    it.use_tma = ((uintptr_t)(it.src + it.s0) & 15u) == 0;
    it.wait_cycles = WAIT_CYCLES_DEFAULT;
    const bool ok = d.R == 4 ? pair_item<MIXED, 4>(it, st, phase, pending)
                             : pair_item<MIXED, 2>(it, st, phase, pending);
    if (!ok) return;
  }
}

// Fixed-order sum of each spectrum's split slabs, scaled by 1/p_s.
__global__ void batched_reduce_kernel(const SpecDesc* __restrict__ spec,
                                      const double* __restrict__ part_re,
                                      const double* __restrict__ part_im,
                                      double* __restrict__ out_re, double* __restrict__ out_im) {
  const SpecDesc d = spec[blockIdx.x];
  const int n_splits = (int)((d.p + d.split_len - 1) / d.split_len);
  const double scale = 1.0 / (double)d.p;
  for (int64_t t = threadIdx.x; t < d.p; t += blockDim.x) {
    double re = 0.0, im = 0.0;
    for (int k = 0; k < n_splits; ++k) {
      re += part_re[d.part_base + (int64_t)k * d.p + t];
      im += part_im[d.part_base + (int64_t)k * d.p + t];
    }
    out_re[d.off + t] = re * scale;
    out_im[d.off + t] = im * scale;
  }
}

// Evenly spaced synthetic spectra for the autotuner: n spectra of p values
// in (0, 3), eta = 1/sqrt(p).
__global__ void tune_fill_kernel(double* ev, int64_t total, int64_t p, double* eta, int n) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < total) ev[i] = 3.0 * ((double)(i % p) + 0.5) / (double)p;
  if (i < n) eta[i] = 1.0 / sqrt((double)p);
}

// ------------------------------------------------------------- host --
struct Tune {
  int R[NB];
  int SL[NB];
  bool tuned = false;
  int version = 0;
};
constexpr int kMaxDev = 64;
constexpr int64_t kMaxSpectrum = 1LL << 24;
Tune g_tune[kMaxDev][2];
std::mutex g_tune_mu[kMaxDev];  // guards g_tune[dev] (and its autotuning run)

struct Plan {
  std::vector<SpecDesc> spec;
  std::vector<BItem> items;
  int64_t part_total = 0;
  int64_t block_total = 0;
};

int bucket_of(int64_t p) {
  int b = 63 - __builtin_clzll((unsigned long long)p);
  return std::min(std::max(b, 8), 15) - 8;
}

// The table the autotuner chose on a B200 (one run, per precision), used
// until a call tunes or installs another: (R, SL) per p-bucket.
constexpr int kDefaultR[2][NB] = {{2, 4, 2, 4, 4, 4, 4, 4}, {2, 4, 2, 4, 2, 2, 2, 2}};
constexpr int kDefaultSL[2][NB] = {{1024, 1024, 2048, 2048, 1024, 2048, 8192, 8192},
                                   {1024, 1024, 2048, 4096, 4096, 2048, 4096, 8192}};

void default_tune(Tune& t, int precision) {
  const int q = precision == SHRK_PREC_MIXED ? 1 : 0;
  for (int b = 0; b < NB; ++b) {
    t.R[b] = kDefaultR[q][b];
    t.SL[b] = kDefaultSL[q][b];
  }
}

// Items and slab layout.  R_force / SL_force > 0 override the table.
void build_plan(const int64_t* off, int64_t n, const Tune& t, int R_force, int SL_force,
                Plan& pl) {
  pl.spec.resize(n);
  pl.items.clear();
  pl.part_total = 0;
  pl.block_total = 0;
  std::vector<int64_t> cost;
  for (int64_t s = 0; s < n; ++s) {
    const int64_t p = off[s + 1] - off[s];
    const int b = bucket_of(p);
    SpecDesc& d = pl.spec[s];
    d.off = off[s];
    d.p = p;
    d.R = R_force > 0 ? R_force : t.R[b];
    d.split_len = SL_force > 0 ? SL_force : t.SL[b];
    d.part_base = pl.part_total;
    d.block_base = pl.block_total;
    const int64_t tt = (int64_t)PAIR_NT * d.R;
    const int64_t n_tiles = (p + tt - 1) / tt;
    const int64_t n_splits = (p + d.split_len - 1) / d.split_len;
    pl.part_total += n_splits * p;
    pl.block_total += (p + SUB - 1) / SUB;
    for (int64_t ti = 0; ti < n_tiles; ++ti)
      for (int64_t k = 0; k < n_splits; ++k) {
        pl.items.push_back({(int)s, (int)ti, (int)k, 0});
        // A tile costs its full width whatever its fill (idle slots still run).
        cost.push_back(tt * std::min<int64_t>(d.split_len, p - k * d.split_len));
      }
  }
  // Largest items first: the persistent grid then finishes with small ones.
  std::vector<int> order(pl.items.size());
  for (size_t i = 0; i < order.size(); ++i) order[i] = (int)i;
  std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return cost[x] > cost[y]; });
  std::vector<BItem> sorted(pl.items.size());
  for (size_t i = 0; i < order.size(); ++i) sorted[i] = pl.items[order[i]];
  pl.items.swap(sorted);
}

// Sizes that fix the scratch layout of a plan.
struct PlanShape {
  size_t n_spec = 0, n_items = 0;
  int64_t part_total = 0, block_total = 0;
};

PlanShape shape_of(const Plan& pl) {
  PlanShape sh;
  sh.n_spec = pl.spec.size();
  sh.n_items = pl.items.size();
  sh.part_total = pl.part_total;
  sh.block_total = pl.block_total;
  return sh;
}

struct DevBuffers {
  SpecDesc* spec;
  BItem* items;
  int* counter;
  double2* bounds;
  double* part_re;
  double* part_im;
};

// Scratch slots of the batched path: 12 descriptors, 13 items + counter,
// 14 partial slabs, 22 block bounds, 23 autotuner inputs.
shrk_status get_buffers(const PlanShape& sh, DevBuffers& b) {
  void* p = nullptr;
  SHRK_TRY(scratch_get(12, sizeof(SpecDesc) * sh.n_spec, &p));
  b.spec = (SpecDesc*)p;
  const size_t item_bytes = (sizeof(BItem) * sh.n_items + 255) / 256 * 256;
  SHRK_TRY(scratch_get(13, item_bytes + 256, &p));
  b.items = (BItem*)p;
  b.counter = (int*)((char*)p + item_bytes);
  SHRK_TRY(scratch_get(14, sizeof(double) * 2 * (size_t)sh.part_total, &p));
  b.part_re = (double*)p;
  b.part_im = (double*)p + sh.part_total;
  SHRK_TRY(scratch_get(22, sizeof(double2) * (size_t)std::max<int64_t>(sh.block_total, 1), &p));
  b.bounds = (double2*)p;
  return SHRK_OK;
}

shrk_status upload_plan(const Plan& pl, const DevBuffers& b, cudaStream_t s) {
  SHRK_CUDA(cudaMemcpyAsync(b.spec, pl.spec.data(), sizeof(SpecDesc) * pl.spec.size(),
                            cudaMemcpyHostToDevice, s));
  SHRK_CUDA(cudaMemcpyAsync(b.items, pl.items.data(), sizeof(BItem) * pl.items.size(),
                            cudaMemcpyHostToDevice, s));
  // The host vectors may be reused as soon as this call returns.
  SHRK_CUDA(cudaStreamSynchronize(s));
  return SHRK_OK;
}

// The kernels of one batched transform (no library timing: also used while
// the stream is being captured into a graph).
shrk_status enqueue(const Plan& pl, const DevBuffers& b, const double* d_ev, const double* d_eta,
                    int precision, double* d_re, double* d_im, cudaStream_t s) {
  const int n = (int)pl.spec.size();
  const bool mixed = precision == SHRK_PREC_MIXED;
  SHRK_CUDA(cudaMemsetAsync(b.counter, 0, sizeof(int), s));
  if (mixed) {
    batched_bounds_kernel<<<n, 128, 0, s>>>(d_ev, b.spec, b.bounds);
    SHRK_CUDA(cudaGetLastError());
  }
  BatchArgs a;
  a.ev = d_ev;
  a.eta = d_eta;
  a.spec = b.spec;
  a.items = b.items;
  a.n_items = (int)pl.items.size();
  a.counter = b.counter;
  a.bounds = b.bounds;
  a.part_re = b.part_re;
  a.part_im = b.part_im;
  a.near_k = mixed_near_k();
  a.err = device_error_word();
  const int grid = (int)std::min<int64_t>((int64_t)pl.items.size(), (int64_t)sm_count() * B_CTAS);
  if (mixed) batched_kernel<true><<<grid, PAIR_NT, 0, s>>>(a);
  else batched_kernel<false><<<grid, PAIR_NT, 0, s>>>(a);
  SHRK_CUDA(cudaGetLastError());
  batched_reduce_kernel<<<n, 256, 0, s>>>(b.spec, b.part_re, b.part_im, d_re, d_im);
  SHRK_CUDA(cudaGetLastError());
  return SHRK_OK;
}

int kernels_per_call(int precision) { return precision == SHRK_PREC_MIXED ? 3 : 2; }

// One cached graph per call context (it reads that context's scratch slots):
// the last plan.
struct GraphCache {
  bool valid = false;
  std::vector<int64_t> offsets;
  int precision = -1;
  int tune_version = -1;
  const void* ptrs[10] = {};
  PlanShape shape;
  cudaGraphExec_t exec = nullptr;
  ~GraphCache() {
    if (exec) cudaGraphExecDestroy(exec);
  }
};

int current_device() {
  int d = 0;
  cudaGetDevice(&d);
  return d;
}

// Times one forced (R, SL) configuration on the synthetic batch (ms).
shrk_status time_config(const Plan& pl, const double* d_ev, const double* d_eta, int precision,
                        double* d_re, double* d_im, cudaStream_t s, float* ms) {
  DevBuffers b;
  SHRK_TRY(get_buffers(shape_of(pl), b));
  SHRK_TRY(upload_plan(pl, b, s));
  SHRK_TRY(enqueue(pl, b, d_ev, d_eta, precision, d_re, d_im, s));  // warm-up
  cudaEvent_t e0, e1;
  SHRK_CUDA(cudaEventCreate(&e0));
  SHRK_CUDA(cudaEventCreate(&e1));
  SHRK_CUDA(cudaEventRecord(e0, s));
  shrk_status st = enqueue(pl, b, d_ev, d_eta, precision, d_re, d_im, s);
  SHRK_CUDA(cudaEventRecord(e1, s));
  SHRK_CUDA(cudaEventSynchronize(e1));
  SHRK_CUDA(cudaEventElapsedTime(ms, e0, e1));
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  add_launches(2 * kernels_per_call(precision));
  return st;
}

// Autotuner: for each p-bucket, a synthetic batch of evenly spaced spectra
// (p = 1.5 * 2^b, about 4M targets and at most 5e9 pairs) is timed for every
// (R, SL) candidate; the fastest is kept.
shrk_status autotune(int precision, Tune& t, cudaStream_t s) {
  default_tune(t, precision);
  for (int b = 0; b < NB; ++b) {
    const int64_t p = 3LL << (b + 7);
    const int64_t n = std::max<int64_t>(1, std::min<int64_t>((1LL << 22) / p,
                                                             (int64_t)5e9 / (p * p)));
    const int64_t total = n * p;
    void* buf = nullptr;
    SHRK_TRY(scratch_get(23, sizeof(double) * (3 * (size_t)total + (size_t)n), &buf));
    double* ev = (double*)buf;
    double* re = ev + total;
    double* im = re + total;
    double* eta = im + total;
    tune_fill_kernel<<<(unsigned)((total + 255) / 256), 256, 0, s>>>(ev, total, p, eta, (int)n);
    SHRK_CUDA(cudaGetLastError());
    add_launches(1);
    std::vector<int64_t> off(n + 1);
    for (int64_t i = 0; i <= n; ++i) off[i] = i * p;
    float best = INFINITY;
    for (int R : TUNE_R) {
      for (int SL : TUNE_SL) {
        if (SL > TUNE_SL[0] && SL / 2 >= p) continue;  // one split already
        Plan pl;
        build_plan(off.data(), n, t, R, SL, pl);
        float ms = 0.f;
        SHRK_TRY(time_config(pl, ev, eta, precision, re, im, s, &ms));
        if (ms < best) {
          best = ms;
          t.R[b] = R;
          t.SL[b] = SL;
        }
      }
    }
  }
  t.tuned = true;
  t.version += 1;
  return SHRK_OK;
}

}  // namespace

shrk_status batched_set_tune(int precision, const int* table) {
  const int dev = current_device();
  if (dev < 0 || dev >= kMaxDev) {
    set_error("device ordinal out of range");
    return SHRK_EINVAL;
  }
  for (int b = 0; b < NB; ++b) {
    const int R = table[2 * b], SL = table[2 * b + 1];
    const bool r_ok = std::find(std::begin(TUNE_R), std::end(TUNE_R), R) != std::end(TUNE_R);
    const bool s_ok = std::find(std::begin(TUNE_SL), std::end(TUNE_SL), SL) != std::end(TUNE_SL);
    if (!r_ok || !s_ok) {
      set_error("batched tuning table: R must be 2 or 4 and SL one of 1024, 2048, 4096, 8192 "
                "(bucket " + std::to_string(b) + ")");
      return SHRK_EINVAL;
    }
  }
  std::lock_guard<std::mutex> lk(g_tune_mu[dev]);
  Tune& t = g_tune[dev][precision];
  for (int b = 0; b < NB; ++b) {
    t.R[b] = table[2 * b];
    t.SL[b] = table[2 * b + 1];
  }
  t.tuned = true;
  t.version += 1;
  return SHRK_OK;
}

shrk_status batched_tune(int precision, bool force, int* table, cudaStream_t s) {
  const int dev = current_device();
  if (dev < 0 || dev >= kMaxDev) {
    set_error("device ordinal out of range");
    return SHRK_EINVAL;
  }
  std::lock_guard<std::mutex> lk(g_tune_mu[dev]);
  Tune& t = g_tune[dev][precision];
  if (force || !t.tuned) SHRK_TRY(autotune(precision, t, s));
  if (table)
    for (int b = 0; b < NB; ++b) {
      table[2 * b] = t.R[b];
      table[2 * b + 1] = t.SL[b];
    }
  return SHRK_OK;
}

shrk_status batched(const double* d_ev, const int64_t* d_offsets, const int64_t* h_offsets,
                    int64_t n, const double* d_eta, int precision, double* d_re, double* d_im,
                    cudaStream_t s) {
  if (n <= 0) return SHRK_OK;
  std::vector<int64_t> off;
  if (!h_offsets) {
    // Device-pointer entry: the plan is built on the host.
    off.resize(n + 1);
    std::vector<double> eta(n);
    SHRK_CUDA(cudaMemcpyAsync(off.data(), d_offsets, sizeof(int64_t) * (n + 1),
                              cudaMemcpyDeviceToHost, s));
    SHRK_CUDA(cudaMemcpyAsync(eta.data(), d_eta, sizeof(double) * n, cudaMemcpyDeviceToHost, s));
    SHRK_CUDA(cudaStreamSynchronize(s));
    if (off[0] != 0) {
      set_error("offsets[0] must be 0");
      return SHRK_EINVAL;
    }
    for (int64_t i = 0; i < n; ++i) {
      if (off[i + 1] <= off[i]) {
        set_error("every spectrum must be non-empty");
        return SHRK_EINVAL;
      }
      if (!(std::isfinite(eta[i]) && eta[i] > 0.0)) {
        set_error("eta must be a positive finite number");
        return SHRK_EINVAL;
      }
    }
    h_offsets = off.data();
  }
  for (int64_t i = 0; i < n; ++i)
    if (h_offsets[i + 1] - h_offsets[i] > kMaxSpectrum) {
      set_error("a spectrum of the batch has more than 16777216 eigenvalues; use "
                "shrk_stieltjes_all for it");
      return SHRK_EINVAL;
    }
  const int dev = current_device();
  if (dev < 0 || dev >= kMaxDev) {
    set_error("device ordinal out of range");
    return SHRK_EINVAL;
  }
  Tune t;
  {
    std::lock_guard<std::mutex> lk(g_tune_mu[dev]);
    Tune& tt = g_tune[dev][precision];
    if (!tt.tuned) {
      // The B200 table by default; SHRK_BATCHED_AUTOTUNE=1 tunes on this
      // device at the first call instead (plans, and so the split summation
      // order, then depend on timing).
      const char* env = std::getenv("SHRK_BATCHED_AUTOTUNE");
      if (env && std::strcmp(env, "1") == 0) {
        SHRK_TRY(autotune(precision, tt, s));
      } else {
        default_tune(tt, precision);
        tt.tuned = true;
      }
    }
    t = tt;
  }

  // Replay the cached graph when the plan (offsets, precision, tuning) and
  // every buffer it references are unchanged.
  GraphCache& gc = ctx_state<GraphCache>(EXT_BATCHED_GRAPH);
  DevBuffers b;
  if (gc.valid && gc.precision == precision && gc.tune_version == t.version &&
      (int64_t)gc.offsets.size() == n + 1 &&
      std::memcmp(gc.offsets.data(), h_offsets, sizeof(int64_t) * (n + 1)) == 0) {
    SHRK_TRY(get_buffers(gc.shape, b));
    const void* ptrs[10] = {d_ev, d_eta, d_re, d_im, b.spec, b.items, b.part_re, b.bounds,
                            device_error_word(), (const void*)s};
    if (std::memcmp(gc.ptrs, ptrs, sizeof(ptrs)) == 0) {
      LaunchScope ls("batched", s);
      add_launches(kernels_per_call(precision) - 1);
      SHRK_CUDA(cudaGraphLaunch(gc.exec, s));
      return SHRK_OK;
    }
  }
  Plan pl;
  build_plan(h_offsets, n, t, 0, 0, pl);
  if (pl.items.size() > (size_t)INT32_MAX / 2) {
    set_error("the batch has too many work items");
    return SHRK_EINVAL;
  }
  SHRK_TRY(get_buffers(shape_of(pl), b));
  const void* ptrs[10] = {d_ev, d_eta, d_re, d_im, b.spec, b.items, b.part_re, b.bounds,
                          device_error_word(), (const void*)s};
  SHRK_TRY(upload_plan(pl, b, s));
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  SHRK_CUDA(cudaStreamIsCapturing(s, &cap));
  // The legacy default stream cannot be captured, and a stream the caller
  // is already capturing takes the kernels into the caller's graph.
  if (s == nullptr || cap != cudaStreamCaptureStatusNone) {
    LaunchScope ls("batched", s);
    add_launches(kernels_per_call(precision) - 1);
    return enqueue(pl, b, d_ev, d_eta, precision, d_re, d_im, s);
  }
  if (gc.exec) {
    cudaGraphExecDestroy(gc.exec);
    gc.exec = nullptr;
  }
  gc.valid = false;
  cudaGraph_t graph = nullptr;
  SHRK_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
  const shrk_status est = enqueue(pl, b, d_ev, d_eta, precision, d_re, d_im, s);
  const cudaError_t ce = cudaStreamEndCapture(s, &graph);
  if (est != SHRK_OK) {
    if (graph) cudaGraphDestroy(graph);
    return est;
  }
  if (ce != cudaSuccess) return cuda_fail(ce, "cudaStreamEndCapture(batched)");
  const cudaError_t ie = cudaGraphInstantiate(&gc.exec, graph, 0);
  cudaGraphDestroy(graph);
  if (ie != cudaSuccess) return cuda_fail(ie, "cudaGraphInstantiate(batched)");
  gc.offsets.assign(h_offsets, h_offsets + n + 1);
  gc.shape = shape_of(pl);
  gc.precision = precision;
  gc.tune_version = t.version;
  std::memcpy(gc.ptrs, ptrs, sizeof(ptrs));
  gc.valid = true;
  LaunchScope ls("batched", s);
  add_launches(kernels_per_call(precision) - 1);
  SHRK_CUDA(cudaGraphLaunch(gc.exec, s));
  return SHRK_OK;
}

}  // namespace shrk
