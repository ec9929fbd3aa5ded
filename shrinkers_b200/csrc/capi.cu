// C ABI of libshrinkers_b200 (include/shrinkers_b200.h): argument checks,
// method policy, per-device state, host<->device staging, and the host-side
// pieces of the estimators (sort, BEMA, inverse BBP) that the reference also
// runs on the host.  All heavy arithmetic runs in the kernels of exact.cu,
// fftgrid.cu, chebcode.cu and batched.cu; there is no CPU fallback.
#include "common.cuh"
#include "internal.h"
#include "../../include/shrinkers_b200_diag.h"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <limits>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

namespace shrk {

// ------------------------------------------------------------ errors --
static thread_local std::string t_last_error;

void set_error(const std::string& msg) { t_last_error = msg; }

shrk_status cuda_fail(cudaError_t e, const char* what) {
  set_error(std::string("CUDA error in ") + what + ": " + cudaGetErrorString(e));
  if (e == cudaErrorMemoryAllocation) return SHRK_ENOMEM;
  return SHRK_ECUDA;
}

static shrk_status einval(const std::string& msg) {
  set_error(msg);
  return SHRK_EINVAL;
}

// ---------------------------------------------------------- contexts --
// A context holds what one stream of calls needs: the scratch slots, the
// device error word and the modules' per-context caches (FFT tables, the
// batched path's CUDA graph, the matrix path's handles).  Calls on one
// context are serialised by its mutex (they share the scratch); calls on
// different contexts run concurrently.  Host-pointer entry points use one
// context per host thread and device, with a stream of its own; `_dev`
// entry points use one context per (device, stream) they are given, so calls
// on different streams never share scratch.
constexpr int kExtSlots = 8;

struct Context {
  std::recursive_mutex mu;
  int dev = 0;
  int sms = 0;
  cudaStream_t stream = nullptr;  // the stream of a host-thread context (owned)
  bool host = false;
  bool in_use = true;             // host-thread contexts: false once their thread exited
  uintptr_t key = 0;              // `_dev` contexts: the stream handle
  Scratch slots[64];
  int* err = nullptr;
  void* ext[kExtSlots] = {};
  void (*ext_del[kExtSlots])(void*) = {};
  // Host-pointer calls: pinned staging of their host<->device copies (grow-
  // only; sized at call entry from the previous call's needs) and the
  // device->host copies waiting for the call's one synchronisation.
  char* stage = nullptr;
  size_t stage_bytes = 0, stage_used = 0, stage_want = 0;
  bool stage_busy = false;  // copies from/to the stage may still be in flight
  struct PendingCopy { void* dst; size_t off, bytes; };
  std::vector<PendingCopy> pending;
  // source_hint of the running host-pointer call
  const double* hint_dev = nullptr;
  int64_t hint_n = 0;
  bool hint_sorted = false;
  double hint_first = 0.0, hint_last = 0.0, hint_min = 0.0, hint_max = 0.0;
};

static std::mutex g_ctx_mu;  // guards the registries below, not the contexts
static std::map<std::pair<int, uintptr_t>, Context*> g_stream_ctx;
static std::vector<Context*> g_host_ctx;
static thread_local Context* t_cur = nullptr;  // the context of the running call

// The calling thread's host contexts; on thread exit they become free for
// the next thread that needs one on that device (no CUDA call at exit).
struct ThreadContexts {
  std::map<int, Context*> by_dev;
  ~ThreadContexts() {
    std::lock_guard<std::mutex> lk(g_ctx_mu);
    for (auto& kv : by_dev) kv.second->in_use = false;
  }
};
static thread_local ThreadContexts t_host;

static shrk_status init_context(Context* c, int dev, bool host) {
  c->dev = dev;
  c->host = host;
  SHRK_CUDA(cudaDeviceGetAttribute(&c->sms, cudaDevAttrMultiProcessorCount, dev));
  if (host) SHRK_CUDA(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
  SHRK_CUDA(cudaMalloc(&c->err, sizeof(int)));
  SHRK_CUDA(cudaMemset(c->err, 0, sizeof(int)));
  return SHRK_OK;
}

static shrk_status host_context(Context** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return cuda_fail(e, "cudaGetDevice");
  auto it = t_host.by_dev.find(dev);
  if (it != t_host.by_dev.end()) {
    *out = it->second;
    return SHRK_OK;
  }
  Context* c = nullptr;
  {
    std::lock_guard<std::mutex> lk(g_ctx_mu);
    for (Context* x : g_host_ctx)
      if (!x->in_use && x->dev == dev) {
        x->in_use = true;
        c = x;
        break;
      }
  }
  if (!c) {
    std::unique_ptr<Context> n(new Context());
    SHRK_TRY(init_context(n.get(), dev, true));
    c = n.release();
    std::lock_guard<std::mutex> lk(g_ctx_mu);
    g_host_ctx.push_back(c);
  }
  t_host.by_dev[dev] = c;
  *out = c;
  return SHRK_OK;
}

static shrk_status stream_context(const void* stream, Context** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return cuda_fail(e, "cudaGetDevice");
  const auto key = std::make_pair(dev, (uintptr_t)stream);
  {
    std::lock_guard<std::mutex> lk(g_ctx_mu);
    auto it = g_stream_ctx.find(key);
    if (it != g_stream_ctx.end()) {
      *out = it->second;
      return SHRK_OK;
    }
  }
  std::unique_ptr<Context> n(new Context());
  n->key = (uintptr_t)stream;
  SHRK_TRY(init_context(n.get(), dev, false));
  std::lock_guard<std::mutex> lk(g_ctx_mu);
  auto ins = g_stream_ctx.emplace(key, n.get());
  if (ins.second) {
    *out = n.release();
  } else {  // another thread registered it first
    cudaFree(n->err);
    *out = ins.first->second;
  }
  return SHRK_OK;
}

// Frees everything a context holds on the device (its mutex held).
static void release_context_memory(Context* c) {
  for (auto& sl : c->slots) {
    if (sl.ptr) cudaFree(sl.ptr);
    sl.ptr = nullptr;
    sl.bytes = 0;
  }
  for (int k = 0; k < kExtSlots; ++k) {
    if (c->ext[k] && c->ext_del[k]) c->ext_del[k](c->ext[k]);
    c->ext[k] = nullptr;
    c->ext_del[k] = nullptr;
  }
}

shrk_status scratch_get(int slot, size_t bytes, void** out) {
  Scratch& s = t_cur->slots[slot];
  if (s.bytes < bytes) {
    if (s.ptr) {
      cudaError_t e = cudaFree(s.ptr);
      if (e != cudaSuccess) return cuda_fail(e, "cudaFree(scratch)");
    }
    s.ptr = nullptr;
    s.bytes = 0;
    size_t want = std::max<size_t>(bytes, 256);
    cudaError_t e = cudaMalloc(&s.ptr, want);
    if (e != cudaSuccess) return cuda_fail(e, "cudaMalloc(scratch)");
    s.bytes = want;
  }
  *out = s.ptr;
  return SHRK_OK;
}

void* ctx_ext(int k, void* (*make)(), void (*del)(void*)) {
  Context* c = t_cur;
  if (!c->ext[k]) {
    c->ext[k] = make();
    c->ext_del[k] = del;
  }
  return c->ext[k];
}

void set_source_hint(const double* d_src, const double* h_src, int64_t n) {
  Context* c = t_cur;
  // Up to 16 384 values the host scan (~1 ns a value) costs less than the
  // device check's launch and read-back; above, the device checks.
  constexpr int64_t kHostScanMax = 16384;
  if (!c || n <= 0 || n > kHostScanMax) return;
  bool sorted = true;
  double mn = h_src[0], mx = h_src[0];
  for (int64_t i = 1; i < n; ++i) {
    if (!(h_src[i - 1] <= h_src[i])) sorted = false;
    mn = std::min(mn, h_src[i]);
    mx = std::max(mx, h_src[i]);
  }
  c->hint_dev = d_src;
  c->hint_n = n;
  c->hint_sorted = sorted;
  c->hint_first = h_src[0];
  c->hint_last = h_src[n - 1];
  c->hint_min = mn;
  c->hint_max = mx;
}

bool source_hint(const double* d_src, int64_t n, bool* sorted, double* first, double* last,
                 double* lo, double* hi) {
  Context* c = t_cur;
  if (!c || c->hint_dev != d_src || c->hint_n != n || !d_src) return false;
  *sorted = c->hint_sorted;
  *first = c->hint_first;
  *last = c->hint_last;
  if (lo) *lo = c->hint_min;
  if (hi) *hi = c->hint_max;
  return true;
}

int* device_error_word() { return t_cur->err; }
int sm_count() { return t_cur ? t_cur->sms : 148; }
cudaStream_t library_stream() { return t_cur->stream; }

static shrk_status check_error_word(Context* c, cudaStream_t s) {
  int h = 0;
  char* st = (c->host && s == c->stream && c->stage && c->stage_used + 256 <= c->stage_bytes)
                 ? c->stage + c->stage_used
                 : nullptr;
  SHRK_CUDA(cudaMemcpyAsync(st ? (void*)st : (void*)&h, c->err, sizeof(int),
                            cudaMemcpyDeviceToHost, s));
  SHRK_CUDA(cudaStreamSynchronize(s));
  c->stage_busy = false;
  if (st) std::memcpy(&h, st, sizeof(int));
  for (const auto& q : c->pending) std::memcpy(q.dst, c->stage + q.off, q.bytes);
  c->pending.clear();
  if (h != DEV_ERR_NONE) {
    SHRK_CUDA(cudaMemsetAsync(c->err, 0, sizeof(int), s));
    SHRK_CUDA(cudaStreamSynchronize(s));
    if (h == DEV_ERR_TIMEOUT) {
      set_error("a bounded device-side wait gave up (timeout)");
      return SHRK_ETIMEOUT;
    }
    set_error("a device-side self-check failed (code " + std::to_string(h) + ")");
    return SHRK_ECUDA;
  }
  return SHRK_OK;
}

shrk_status check_device_error(cudaStream_t s) { return check_error_word(t_cur, s); }

// ------------------------------------------------------------ timing --
static std::atomic<int64_t> g_launches{0};
static std::atomic<bool> g_timing{false};
static std::mutex g_timing_mu;  // guards g_timed
struct TimedLaunch { std::string family; cudaEvent_t a, b; };
static std::vector<TimedLaunch> g_timed;

void add_launches(int64_t n) { g_launches.fetch_add(n); }

LaunchScope::LaunchScope(const char* fam, cudaStream_t s) : family(fam), stream(s) {
  g_launches.fetch_add(1);
  if (g_timing) {
    cudaEventCreate(&start);
    cudaEventCreate(&stop);
    cudaEventRecord(start, s);
  }
}
LaunchScope::~LaunchScope() {
  if (start) {
    cudaEventRecord(stop, stream);
    std::lock_guard<std::mutex> lk(g_timing_mu);
    g_timed.push_back({family, start, stop});
  }
}

// ----------------------------------------------------------- helpers --
static bool is_auto(int m) {
  return m == SHRK_M_AUTO || m == SHRK_M_SPEED_AUTO || m == SHRK_M_ACCURACY_AUTO;
}
static bool is_exact_family(int m) {
  return m == SHRK_M_NAIVE || m == SHRK_M_AUTOVEC || m == SHRK_M_BLOCKED ||
         m == SHRK_M_BLOCKED_AUTOVEC || m == SHRK_M_BLOCKED_TILED ||
         m == SHRK_M_BLOCKED_WINDOWED || m == SHRK_M_BLOCKED_HYBRID;
}
static bool is_cheb(int m) {
  return m == SHRK_M_CHEBCODE || m == SHRK_M_CHEBCODE_FAST || m == SHRK_M_CHEBCODE_XTREME ||
         m == SHRK_M_CHEBCODE_BALANCED;
}

static shrk_status check_common(size_t p, double eta, int method, int precision) {
  if (p == 0) return einval("eigenvalues must be non-empty");
  if (!(std::isfinite(eta) && eta > 0.0)) return einval("eta must be a positive finite number");
  if (method < 0 || method > SHRK_M_ACCURACY_AUTO) return einval("unknown method id");
  if (precision != SHRK_PREC_F64 && precision != SHRK_PREC_MIXED)
    return einval("unknown precision id");
  return SHRK_OK;
}

static shrk_status check_cutoff(double cutoff) {
  if (std::isnan(cutoff)) return SHRK_OK;
  if (!(std::isfinite(cutoff) && cutoff > 0.0))
    return einval("cutoff ratio must be a positive finite number");
  return SHRK_OK;
}

static shrk_status not_impl(int m) {
  set_error(std::string("method '") + shrk_method_name(m) +
            "' has no GPU implementation in shrinkers_b200 (no CPU fallback)");
  return SHRK_ENOTIMPL;
}

// Host<->device copies of the host-pointer entry points.  Small ones (at
// most 1 MiB) are staged through the context's pinned buffer: an upload is a
// host memcpy into the stage plus an asynchronous copy; a download is an
// asynchronous copy into the stage that check_device_error completes (one
// synchronisation per call, shared with the error-word read).  Larger copies,
// and small ones that do not fit the stage (it grows before the next call),
// go direct.
static char* stage_take(Context* c, size_t bytes, size_t* off) {
  // Large copies go direct: the DMA engine reads pinned user memory at full
  // speed and the driver stages pageable memory itself; an extra host copy
  // only pays for small, latency-bound transfers.
  constexpr size_t kStageCopyMax = (size_t)1 << 20;
  if (bytes > kStageCopyMax) return nullptr;
  const size_t al = (bytes + 255) & ~(size_t)255;
  c->stage_want += al;
  if (!c->stage || c->stage_used + al > c->stage_bytes) return nullptr;
  *off = c->stage_used;
  c->stage_used += al;
  c->stage_busy = true;
  return c->stage + *off;
}

static shrk_status h2d(void* dst, const void* src, size_t bytes, cudaStream_t s) {
  Context* c = t_cur;
  size_t off = 0;
  char* st = (c && c->host && s == c->stream) ? stage_take(c, bytes, &off) : nullptr;
  if (st) {
    std::memcpy(st, src, bytes);
    SHRK_CUDA(cudaMemcpyAsync(dst, st, bytes, cudaMemcpyHostToDevice, s));
  } else {
    SHRK_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, s));
  }
  return SHRK_OK;
}

static shrk_status d2h(void* dst, const void* src, size_t bytes, cudaStream_t s) {
  Context* c = t_cur;
  size_t off = 0;
  char* st = (c && c->host && s == c->stream) ? stage_take(c, bytes, &off) : nullptr;
  if (st) {
    SHRK_CUDA(cudaMemcpyAsync(st, src, bytes, cudaMemcpyDeviceToHost, s));
    c->pending.push_back({dst, off, bytes});
  } else {
    SHRK_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, s));
  }
  return SHRK_OK;
}

// At the entry of a host-pointer call: settle what an earlier call that
// returned early may have left in flight, and size the stage.
static shrk_status stage_begin(Context* c) {
  if (c->stage_busy) {
    SHRK_CUDA(cudaStreamSynchronize(c->stream));
    c->stage_busy = false;
  }
  c->pending.clear();
  constexpr size_t kStageMax = (size_t)8 << 20;
  const size_t want = std::min(std::max(c->stage_want, (size_t)1 << 16), kStageMax);
  if (want > c->stage_bytes) {
    if (c->stage) cudaFreeHost(c->stage);
    c->stage = nullptr;
    c->stage_bytes = 0;
    const size_t grow = std::min(std::max(want, 2 * c->stage_bytes), kStageMax);
    if (cudaMallocHost((void**)&c->stage, grow) == cudaSuccess) c->stage_bytes = grow;
    else cudaGetLastError();  // no pinned memory: the copies go direct
  }
  c->stage_used = 0;
  c->stage_want = 0;
  return SHRK_OK;
}

// Scratch slot map: 0 split partials, 1 block bounds, 2 adjoint partials,
// 3 input spectrum, 4/5 outputs, 6 query points, 7 raw sums (2 arrays),
// 8 sorted copy of the sources, 9/10 hybrid temporaries, 11 FFT grids,
// 12/13/14/22/23 batched path (its cached graph reads 12, 13, 14 and 22, so
// no other path may write them), 15 probe sink, 16..21 treecode,
// 24 FFT-grid stencil weights, 25..31 (see the kernel files), 32..38 the
// matrix front-end (matrix.cu), 39..45 the dyadic FMM (fmm.cu).

static bool is_fft5_family(int m) {
  return m == SHRK_M_FFT5 || m == SHRK_M_FFT3 || m == SHRK_M_FFT2;
}

// Raw (or scaled) sums of `method` at targets d_tgt against d_src, written
// through `epi`.  The method must already be resolved.  all_points: the
// targets are the sources (compute_all_stieltjes, mod.rs:601-790), else
// arbitrary query points (compute_stieltjes_at_points, mod.rs:394-494).
// A shard of a multi-GPU call passes the size of the whole call's query set
// (nq_total, for the policies that depend on it) and, for all points, where
// its targets start in the spectrum (tgt_offset).
static shrk_status sums_dispatch(const double* d_tgt, int64_t nt, const double* d_src,
                                 int64_t ns, double eta, int method,
                                 int precision, double cutoff, const Epilogue& epi,
                                 cudaStream_t s, bool all_points, int64_t nq_total = -1,
                                 int64_t tgt_offset = 0) {
  if (nq_total < 0) nq_total = nt;
  const bool cut = !std::isnan(cutoff);
  // mod.rs:265-287: at query points, every grid method without a points
  // path of its own takes the exact per-point sum.
  if (!all_points && (method == SHRK_M_ADAPTIVE || method == SHRK_M_DST ||
                      method == SHRK_M_TREECODE || method == SHRK_M_EWALD ||
                      method == SHRK_M_HODLR))
    return exact_pair_sums(d_tgt, nt, d_src, ns, eta, precision, epi, s);
  if (is_fft5_family(method) || method == SHRK_M_ADAPTIVE || method == SHRK_M_DST) {
    const double* ds = nullptr;
    double first = 0.0, last = 0.0;
    SHRK_TRY(sorted_sources(d_src, ns, &ds, &first, &last, s));
    const Fft5Opts opts;  // fft5.rs:237-249 defaults (heptic)
    if (is_fft5_family(method))  // mod.rs:634-641 / 447-453: one kernel, three names
      return fft5_points(d_tgt, nt, ds, ns, first, last, eta, opts, epi, s);
    // adaptive.rs:43-68, mod.rs:672-690: fft5 real part; imaginary part
    // windowed (adaptive: ratio 10 by default; dst: the caller's ratio, or the
    // exact sums without one).
    void* raw = nullptr;
    SHRK_TRY(scratch_get(7, sizeof(double) * 2 * nt, &raw));
    double* rre = (double*)raw;
    double* rim = rre + nt;
    void* tmp = nullptr;
    SHRK_TRY(scratch_get(9, sizeof(double) * nt, &tmp));
    Epilogue e1;
    e1.mode = EPI_SUMS;
    e1.scale = 1.0;
    e1.out_re = rre;
    e1.out_im = (double*)tmp;
    SHRK_TRY(fft5_points(d_tgt, nt, ds, ns, first, last, eta, opts, e1, s));
    const double ratio = (method == SHRK_M_ADAPTIVE && !cut) ? 10.0 : cutoff;
    if (std::isnan(ratio)) {
      Epilogue e2 = e1;  // real part into the scratch, imaginary part kept
      e2.out_re = (double*)tmp;
      e2.out_im = rim;
      SHRK_TRY(exact_pair_sums(d_tgt, nt, d_src, ns, eta, precision, e2, s));
    } else {
      SHRK_TRY(windowed_sums(d_tgt, nt, ds, ns, eta, ratio * eta, 1.0, (double*)tmp, rim, s));
    }
    return apply_epilogue(d_tgt, rre, rim, nt, epi, s);
  }
  if (is_exact_family(method)) {
    const bool windowed_re = cut && (method == SHRK_M_BLOCKED || method == SHRK_M_BLOCKED_TILED ||
                                     method == SHRK_M_BLOCKED_WINDOWED ||
                                     method == SHRK_M_BLOCKED_AUTOVEC);
    const bool windowed_im = windowed_re || (cut && method == SHRK_M_BLOCKED_HYBRID);
    if (!windowed_re && !windowed_im)
      return exact_pair_sums(d_tgt, nt, d_src, ns, eta, precision, epi, s);
    void* raw = nullptr;
    SHRK_TRY(scratch_get(7, sizeof(double) * 2 * nt, &raw));
    double* rre = (double*)raw;
    double* rim = rre + nt;
    if (windowed_re) {
      SHRK_TRY(windowed_sums(d_tgt, nt, d_src, ns, eta, cutoff * eta, 1.0, rre, rim, s));
    } else {  // hybrid: exact real part, windowed imaginary part
      void* tmp = nullptr;
      SHRK_TRY(scratch_get(9, sizeof(double) * nt, &tmp));
      Epilogue e1;
      e1.mode = EPI_SUMS;
      e1.scale = 1.0;
      e1.out_re = rre;
      e1.out_im = (double*)tmp;
      SHRK_TRY(exact_pair_sums(d_tgt, nt, d_src, ns, eta, precision, e1, s));
      void* tmp2 = nullptr;
      SHRK_TRY(scratch_get(10, sizeof(double) * nt, &tmp2));
      SHRK_TRY(windowed_sums(d_tgt, nt, d_src, ns, eta, cutoff * eta, 1.0, (double*)tmp2, rim, s));
    }
    return apply_epilogue(d_tgt, rre, rim, nt, epi, s);
  }
  if (all_points && method == SHRK_M_TREECODE) {
    // StieltjesMethod::TreeCode ("fmm", mod.rs:646-655: a multipole treecode,
    // theta 0.5, order 6, accuracy pinned at 1e-3, treecode.rs:357-393): the
    // dyadic Chebyshev FMM of fmm.cu, order 16, M2L on the tensor cores
    // (TF32 x3, ~1e-6 of |S|).  fmm_all writes S/p in the caller's order.
    // A shard evaluates every point and keeps its slice.
    void* raw = nullptr;
    SHRK_TRY(scratch_get(7, sizeof(double) * 2 * ns, &raw));
    double* rre = (double*)raw;
    double* rim = rre + ns;
    SHRK_TRY(fmm_all(d_src, ns, eta, 16, 1, rre, rim, s));
    Epilogue e2 = epi;
    e2.scale = epi.scale * (double)ns;  // the values are already S/p
    return apply_epilogue(d_tgt, rre + tgt_offset, rim + tgt_offset, nt, e2, s);
  }
  if (method == SHRK_M_NUFFT || is_cheb(method)) {
    const double* ds = nullptr;
    double first = 0.0, last = 0.0;
    SHRK_TRY(sorted_sources(d_src, ns, &ds, &first, &last, s));
    if (method == SHRK_M_NUFFT) {
      SHRK_TRY(nufft_points(d_tgt, nt, ds, ns, first, last, eta, epi, s));
    } else {
      ChebParams prm;
      cheb_preset(method, &prm);
      // At arbitrary query points the leaf capacity is relaxed by the grid
      // rule (mod.rs:475-489).
      if (!all_points) prm.leaf_cap = (int)grid_leaf_cap(prm.n, ns, nq_total, prm.leaf_cap);
      SHRK_TRY(chebcode_points(d_tgt, nt, ds, ns, eta, prm, epi, s));
    }
    return SHRK_OK;
  }
  return not_impl(method);
}

static int resolve(int method, int parallelism, size_t p) {
  return shrk_resolve_auto_method(method, parallelism == SHRK_PAR_PARALLEL ? 1 : 0, p);
}

// ------------------------------------------------ host estimators -- //
// detection.rs:75-83
static double mp_median_factor(double gamma) {
  double g = std::min(std::max(gamma, 0.0), 1.0);
  return 0.999995823 - 0.333211332 * g - 0.0106766617 * g * g - 0.000758816762 * g * g * g -
         0.00256753402 * g * g * g * g;
}
// estimation.rs:37-39
static double bbp_threshold(double gamma, double sigma2) {
  double s = 1.0 + std::sqrt(gamma);
  return sigma2 * (s * s);
}
// estimation.rs:48-56
static double inverse_bbp(double lh, double gamma, double sigma2) {
  double x = lh / sigma2;
  double a = x + 1.0 - gamma;
  double disc = a * a - 4.0 * x;
  if (disc <= 0.0) return bbp_threshold(gamma, sigma2);
  double ell = ((x + 1.0 - gamma) + std::sqrt(disc)) / 2.0;
  return ell * sigma2;
}

struct SpikeSplit {
  size_t k = 0;
  double edge = 0.0, sigma2 = 0.0;
  std::vector<size_t> idx;
  std::vector<double> sorted, spikes, spike_sample, bulk;
};

// detection.rs:134-153 (median 111-121, scan_above 49-63) on a sorted copy.
static void bema(const double* sorted, size_t p, double gamma, double margin, SpikeSplit& out) {
  out.idx.clear();
  if (p == 0) return;
  double med = (p % 2 == 0) ? (sorted[p / 2 - 1] + sorted[p / 2]) / 2.0 : sorted[p / 2];
  double sigma2 = med / mp_median_factor(gamma);
  double edge = bbp_threshold(gamma, sigma2);
  double thr = edge * std::max(margin, 1.0);
  for (size_t i = p; i-- > 0;) {
    if (sorted[i] > thr) out.idx.push_back(i);
    else break;
  }
  std::reverse(out.idx.begin(), out.idx.end());
  out.k = out.idx.size();
  out.edge = edge;
  out.sigma2 = sigma2;
}

// spiked/mod.rs:54-91 detect_debias_split (spikes returned descending).
static void detect_debias_split(const double* ev, size_t p, double gamma, double margin,
                                SpikeSplit& s) {
  s.sorted.assign(ev, ev + p);
  // spectra usually arrive sorted: an O(p) check skips the O(p log p) sort
  // (equal doubles are indistinguishable, so either way gives the same array)
  if (!std::is_sorted(s.sorted.begin(), s.sorted.end()))
    std::stable_sort(s.sorted.begin(), s.sorted.end());
  bema(s.sorted.data(), p, gamma, margin, s);
  s.spikes.clear();
  s.spike_sample.clear();
  for (size_t i : s.idx) {
    s.spike_sample.push_back(s.sorted[i]);
    s.spikes.push_back(inverse_bbp(s.sorted[i], gamma, s.sigma2));
  }
  std::reverse(s.spikes.begin(), s.spikes.end());
  std::reverse(s.spike_sample.begin(), s.spike_sample.end());
  s.bulk.clear();
  size_t q = 0;
  for (size_t i = 0; i < p; ++i) {
    if (q < s.idx.size() && s.idx[q] == i) { ++q; continue; }
    s.bulk.push_back(s.sorted[i]);
  }
}

// Ledoit-Wolf xi on the device for host ev (estimation.rs:75-90).
static shrk_status lw_device(const double* ev, size_t p, double c, int method, int precision,
                             int parallelism, double eta, double* xi) {
  cudaStream_t s = t_cur->stream;
  int m = resolve(method, parallelism, p);
  if (std::isnan(eta)) eta = 0.4 / std::sqrt((double)p);  // mod.rs:150-153
  void* dev = nullptr;
  SHRK_TRY(scratch_get(3, sizeof(double) * p, &dev));
  void* out = nullptr;
  SHRK_TRY(scratch_get(4, sizeof(double) * p, &out));
  SHRK_TRY(h2d(dev, ev, sizeof(double) * p, s));
  set_source_hint((const double*)dev, ev, (int64_t)p);
  Epilogue epi;
  epi.mode = EPI_LW;
  epi.scale = 1.0 / (double)p;
  epi.c = c;
  epi.out_re = (double*)out;
  SHRK_TRY(sums_dispatch((const double*)dev, (int64_t)p, (const double*)dev, (int64_t)p, eta,
                         m, precision, NAN, epi, s, true));
  SHRK_TRY(d2h(xi, out, sizeof(double) * p, s));
  return check_device_error(s);
}

// deconvolution/mod.rs:116-259 with the inversion fused into the epilogue.
static shrk_status deconv_device(const double* ev, size_t p, double c, size_t n_points, double eta,
                                 double lmin, double lmax, int method, int precision,
                                 int parallelism, double cutoff, double* out7) {
  if (p == 0) return SHRK_OK;
  cudaStream_t s = t_cur->stream;
  double eta_val = std::isnan(eta) ? 0.1 / std::sqrt((double)p) : eta;
  double mn = INFINITY, mx = -INFINITY;
  for (size_t i = 0; i < p; ++i) {
    mn = std::min(mn, ev[i]);
    mx = std::max(mx, ev[i]);
  }
  double range = (mx - mn) > 0.0 ? mx - mn : 1.0;
  double margin = 0.2 * range;
  double lo = std::isnan(lmin) ? std::max(mn - margin, 0.0) : lmin;
  double hi = std::isnan(lmax) ? mx + margin : lmax;
  double step = n_points > 1 ? (hi - lo) / ((double)n_points - 1.0) : 0.0;
  double* grid = out7;
  for (size_t k = 0; k < n_points; ++k) grid[k] = lo + step * (double)k;
  // config.rs:507-516 resolve_auto_at_points (parallelism Auto -> Sequential)
  const bool par = parallelism == SHRK_PAR_PARALLEL;
  int m = method;
  if (is_auto(m)) m = shrk_grid_appropriate(shrk_resolve_auto_method(m, par, p), p, n_points);
  void* dev = nullptr;
  SHRK_TRY(scratch_get(3, sizeof(double) * p, &dev));
  void* dq = nullptr;
  SHRK_TRY(scratch_get(6, sizeof(double) * n_points, &dq));
  void* out = nullptr;
  SHRK_TRY(scratch_get(4, sizeof(double) * 6 * n_points, &out));
  SHRK_TRY(h2d(dev, ev, sizeof(double) * p, s));
  set_source_hint((const double*)dev, ev, (int64_t)p);
  SHRK_TRY(h2d(dq, grid, sizeof(double) * n_points, s));
  Epilogue epi;
  epi.mode = EPI_MP;
  epi.scale = 1.0 / (double)p;
  epi.c = c;
  epi.eta = eta_val;
  for (int i = 0; i < 6; ++i) epi.out[i] = (double*)out + i * n_points;
  SHRK_TRY(sums_dispatch((const double*)dq, (int64_t)n_points, (const double*)dev, (int64_t)p,
                         eta_val, m, precision, cutoff, epi, s, false));
  SHRK_TRY(d2h(out7 + n_points, out, sizeof(double) * 6 * n_points, s));
  return check_device_error(s);
}

// Selects and locks the context of a call for its lifetime: Guard() the
// calling thread's host context (host-pointer entry points), Guard(stream)
// the context of (current device, stream) (`_dev` entry points).  Nested
// calls on the same context are allowed (the mutex is recursive); the
// previous context is restored on exit.
struct Guard {
  Context* prev = t_cur;
  Context* ctx = nullptr;
  shrk_status st;
  std::unique_lock<std::recursive_mutex> lk;
  Guard() { st = host_context(&ctx); enter(); }
  explicit Guard(const void* stream) { st = stream_context(stream, &ctx); enter(); }
  ~Guard() { t_cur = prev; }
  Guard(const Guard&) = delete;
  Guard& operator=(const Guard&) = delete;

 private:
  void enter() {
    if (st != SHRK_OK) return;
    lk = std::unique_lock<std::recursive_mutex>(ctx->mu);
    t_cur = ctx;
    ctx->hint_dev = nullptr;  // a hint never outlives the call that set it
    // the outermost host-pointer call on this context owns the stage
    if (ctx->host && prev != ctx) st = stage_begin(ctx);
  }
};

// lib_enter / lib_exit: the host context of the calling thread, as a stack
// of (previous context, entered context) pairs.
static thread_local std::vector<std::pair<Context*, Context*>> t_lib_stack;

shrk_status lib_enter(cudaStream_t* stream) {
  Context* c = nullptr;
  shrk_status st = host_context(&c);
  if (st != SHRK_OK) c = nullptr;
  t_lib_stack.emplace_back(t_cur, c);
  *stream = nullptr;
  if (!c) return st;
  c->mu.lock();
  t_cur = c;
  *stream = c->stream;
  return SHRK_OK;
}

void lib_exit() {
  if (t_lib_stack.empty()) return;
  const auto top = t_lib_stack.back();
  t_lib_stack.pop_back();
  if (top.second) top.second->mu.unlock();
  t_cur = top.first;
}

}  // namespace shrk

using namespace shrk;

// ===================================================================== ABI

extern "C" {

size_t shrk_last_error(char* buf, size_t len) {
  const std::string& e = t_last_error;
  if (buf && len) {
    size_t n = std::min(len - 1, e.size());
    std::memcpy(buf, e.data(), n);
    buf[n] = '\0';
  }
  return e.size();
}

const char* shrk_version(void) { return "0.1.0"; }

int shrk_device_count(void) {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return n;
}

// config.rs:92-118
const char* shrk_method_name(int m) {
  static const char* names[] = {
      "naive", "autovec", "blocked", "blocked_autovec", "blocked_tiled", "blocked_windowed",
      "blocked_hybrid", "adaptive", "fft5", "fft3", "fft2", "nufft", "fmm", "chebcode",
      "chebcode_fast", "chebcode_xtreme", "chebcode_balanced", "ewald", "dst", "auto", "hodlr",
      "speed_auto", "accuracy_auto"};
  if (m < 0 || m > SHRK_M_ACCURACY_AUTO) return "?";
  return names[m];
}

// python.rs:321-350
shrk_status shrk_parse_method(const char* name, int* out) {
  static const struct { const char* n; int m; } tab[] = {
      {"naive", SHRK_M_NAIVE}, {"autovec", SHRK_M_AUTOVEC}, {"blocked", SHRK_M_BLOCKED},
      {"blocked_autovec", SHRK_M_BLOCKED_AUTOVEC}, {"blocked_tiled", SHRK_M_BLOCKED_TILED},
      {"blocked_windowed", SHRK_M_BLOCKED_WINDOWED}, {"blocked_hybrid", SHRK_M_BLOCKED_HYBRID},
      {"adaptive", SHRK_M_ADAPTIVE}, {"fft5", SHRK_M_FFT5}, {"fft3", SHRK_M_FFT3},
      {"fft2", SHRK_M_FFT2}, {"nufft", SHRK_M_NUFFT}, {"fft_fast", SHRK_M_NUFFT},
      {"fmm", SHRK_M_TREECODE}, {"treecode", SHRK_M_TREECODE}, {"chebcode", SHRK_M_CHEBCODE},
      {"chebyshev", SHRK_M_CHEBCODE}, {"chebcode_fast", SHRK_M_CHEBCODE_FAST},
      {"chebf", SHRK_M_CHEBCODE_FAST}, {"chebcode_xtreme", SHRK_M_CHEBCODE_XTREME},
      {"chebx", SHRK_M_CHEBCODE_XTREME}, {"chebcode_balanced", SHRK_M_CHEBCODE_BALANCED},
      {"chebb", SHRK_M_CHEBCODE_BALANCED}, {"ewald", SHRK_M_EWALD}, {"dst", SHRK_M_DST},
      {"auto", SHRK_M_AUTO}, {"hodlr", SHRK_M_HODLR}, {"speed_auto", SHRK_M_SPEED_AUTO},
      {"speed", SHRK_M_SPEED_AUTO}, {"accuracy_auto", SHRK_M_ACCURACY_AUTO},
      {"accuracy", SHRK_M_ACCURACY_AUTO}};
  if (!name || !out) return einval("null argument");
  for (auto& e : tab)
    if (std::strcmp(e.n, name) == 0) {
      *out = e.m;
      return SHRK_OK;
    }
  return einval(std::string("unknown method '") + name + "'");
}

// config.rs:543-555 + pareto_autogen.rs:22-86
int shrk_resolve_auto_method(int m, int parallel, size_t p) {
  struct Bin { size_t p_max; int ss, sp, as, ap; };
  static const Bin bins[] = {
      {1000, SHRK_M_CHEBCODE_FAST, SHRK_M_CHEBCODE_FAST, SHRK_M_BLOCKED_TILED, SHRK_M_BLOCKED},
      {2000, SHRK_M_CHEBCODE_FAST, SHRK_M_CHEBCODE_FAST, SHRK_M_BLOCKED_TILED, SHRK_M_AUTOVEC},
      {5000, SHRK_M_CHEBCODE_FAST, SHRK_M_CHEBCODE_FAST, SHRK_M_BLOCKED_TILED, SHRK_M_AUTOVEC},
      {10000, SHRK_M_CHEBCODE_FAST, SHRK_M_CHEBCODE_FAST, SHRK_M_BLOCKED, SHRK_M_BLOCKED_TILED},
      {20000, SHRK_M_CHEBCODE_FAST, SHRK_M_CHEBCODE_FAST, SHRK_M_BLOCKED, SHRK_M_BLOCKED},
      {50000, SHRK_M_CHEBCODE_FAST, SHRK_M_CHEBCODE_FAST, SHRK_M_BLOCKED_TILED, SHRK_M_BLOCKED},
      {SIZE_MAX, SHRK_M_NUFFT, SHRK_M_NUFFT, SHRK_M_BLOCKED_TILED, SHRK_M_BLOCKED},
  };
  if (!is_auto(m)) return m;
  const Bin* b = &bins[6];
  for (const Bin& x : bins)
    if (p <= x.p_max) { b = &x; break; }
  if (m != SHRK_M_ACCURACY_AUTO) return parallel ? b->sp : b->ss;
  return parallel ? b->ap : b->as;
}

// config.rs:565-585
int shrk_grid_appropriate(int m, size_t p, size_t nq) {
  if (nq > SIZE_MAX / 4 || nq * 4 >= p) return m;
  if (m == SHRK_M_NUFFT && p >= 300000) return m;
  switch (m) {
    case SHRK_M_FFT5: case SHRK_M_FFT3: case SHRK_M_FFT2: case SHRK_M_NUFFT:
    case SHRK_M_ADAPTIVE: case SHRK_M_DST:
      return SHRK_M_CHEBCODE_FAST;
    default:
      return m;
  }
}

double shrk_mixed_near_k(void) { return mixed_near_k(); }

shrk_status shrk_stieltjes_all_dev(const double* d_ev, size_t p, double eta, int method,
                                   int precision, double cutoff, int parallelism, double* d_re,
                                   double* d_im, void* stream) {
  SHRK_TRY(check_common(p, eta, method, precision));
  SHRK_TRY(check_cutoff(cutoff));
  Guard g(stream);
  SHRK_TRY(g.st);
  cudaStream_t s = (cudaStream_t)stream;  // null = the legacy default stream
  int m = resolve(method, parallelism, p);
  Epilogue epi;
  epi.mode = EPI_SUMS;
  epi.scale = 1.0 / (double)p;
  epi.out_re = d_re;
  epi.out_im = d_im;
  return sums_dispatch(d_ev, (int64_t)p, d_ev, (int64_t)p, eta, m, precision, cutoff,
                       epi, s, true);
}

shrk_status shrk_stieltjes_shard_dev(const double* d_tgt, size_t nt, size_t nq_total,
                                     int all_points, const double* d_ev, size_t p, double eta,
                                     int method, int precision, double cutoff, int parallelism,
                                     double* d_re, double* d_im, void* stream) {
  SHRK_TRY(check_common(p, eta, method, precision));
  SHRK_TRY(check_cutoff(cutoff));
  if (nq_total < nt) {
    set_error("shard: nq_total must be at least nt");
    return SHRK_EINVAL;
  }
  int64_t offset = 0;
  if (all_points) {
    // the targets must be a slice of the spectrum (compared as addresses)
    const uintptr_t t = (uintptr_t)d_tgt, e = (uintptr_t)d_ev;
    const bool inside = t >= e && (t - e) % sizeof(double) == 0 && nt <= p &&
                        (t - e) / sizeof(double) <= (uintptr_t)(p - nt);
    if (!inside || nq_total != p) {
      set_error("shard: all-points targets must be a slice of the spectrum, nq_total = p");
      return SHRK_EINVAL;
    }
    offset = (int64_t)((t - e) / sizeof(double));
  }
  if (nt == 0) return SHRK_OK;
  Guard g(stream);
  SHRK_TRY(g.st);
  cudaStream_t s = (cudaStream_t)stream;
  const bool par = parallelism == SHRK_PAR_PARALLEL;
  int m = method;
  if (all_points) m = resolve(method, parallelism, p);
  else if (is_auto(m)) m = shrk_grid_appropriate(shrk_resolve_auto_method(m, par, p), p, nq_total);
  Epilogue epi;
  epi.mode = EPI_SUMS;
  epi.scale = all_points ? 1.0 / (double)p : 1.0;
  epi.out_re = d_re;
  epi.out_im = d_im;
  return sums_dispatch(d_tgt, (int64_t)nt, d_ev, (int64_t)p, eta, m, precision, cutoff, epi, s,
                       all_points != 0, (int64_t)nq_total, offset);
}

shrk_status shrk_stieltjes_all(const double* ev, size_t p, double eta, int method, int precision,
                               double cutoff, int parallelism, double* out_re, double* out_im) {
  SHRK_TRY(check_common(p, eta, method, precision));
  SHRK_TRY(check_cutoff(cutoff));
  Guard g;
  SHRK_TRY(g.st);
  cudaStream_t s = t_cur->stream;
  int m = resolve(method, parallelism, p);
  void* dev = nullptr;
  SHRK_TRY(scratch_get(3, sizeof(double) * p, &dev));
  void* out = nullptr;
  SHRK_TRY(scratch_get(4, sizeof(double) * 2 * p, &out));
  SHRK_TRY(h2d(dev, ev, sizeof(double) * p, s));
  set_source_hint((const double*)dev, ev, (int64_t)p);
  Epilogue epi;
  epi.mode = EPI_SUMS;
  epi.scale = 1.0 / (double)p;
  epi.out_re = (double*)out;
  epi.out_im = (double*)out + p;
  SHRK_TRY(sums_dispatch((const double*)dev, (int64_t)p, (const double*)dev, (int64_t)p, eta,
                         m, precision, cutoff, epi, s, true));
  SHRK_TRY(d2h(out_re, out, sizeof(double) * p, s));
  SHRK_TRY(d2h(out_im, (double*)out + p, sizeof(double) * p, s));
  return check_device_error(s);
}

shrk_status shrk_stieltjes_all_f32(const float* ev, size_t p, float eta, int method,
                                   double cutoff, float* out_re, float* out_im) {
  if (p == 0) return einval("eigenvalues must be non-empty");
  if (!(std::isfinite(eta) && eta > 0.0f)) return einval("eta must be a positive finite number");
  SHRK_TRY(check_cutoff(cutoff));
  // mod.rs:818-847: Blocked/BlockedTiled/Auto without a cutoff run the f32
  // kernel; every other combination runs the f64 path and rounds.
  if (!(method == SHRK_M_BLOCKED || method == SHRK_M_BLOCKED_TILED || method == SHRK_M_AUTO) ||
      !std::isnan(cutoff)) {
    std::vector<double> e64(ev, ev + p), r(p), i(p);
    // Parallelism::Sequential (mod.rs:836-845)
    SHRK_TRY(shrk_stieltjes_all(e64.data(), p, (double)eta, method, SHRK_PREC_F64, cutoff,
                                SHRK_PAR_SEQUENTIAL, r.data(), i.data()));
    for (size_t k = 0; k < p; ++k) {
      out_re[k] = (float)r[k];
      out_im[k] = (float)i[k];
    }
    return SHRK_OK;
  }
  Guard g;
  SHRK_TRY(g.st);
  cudaStream_t s = t_cur->stream;
  void* dev = nullptr;
  SHRK_TRY(scratch_get(3, sizeof(float) * p, &dev));
  void* out = nullptr;
  SHRK_TRY(scratch_get(4, sizeof(float) * 2 * p, &out));
  SHRK_TRY(h2d(dev, ev, sizeof(float) * p, s));
  SHRK_TRY(all_f32((const float*)dev, (int64_t)p, eta, (float*)out, (float*)out + p, s));
  SHRK_TRY(d2h(out_re, out, sizeof(float) * p, s));
  SHRK_TRY(d2h(out_im, (float*)out + p, sizeof(float) * p, s));
  return check_device_error(s);
}

shrk_status shrk_stieltjes_at_points_dev(const double* d_q, size_t nq, const double* d_ev, size_t p,
                                         double eta, int method, int precision, double cutoff,
                                         int parallelism, double* d_re, double* d_im,
                                         void* stream) {
  SHRK_TRY(check_common(p, eta, method, precision));
  SHRK_TRY(check_cutoff(cutoff));
  if (nq == 0) return SHRK_OK;
  Guard g(stream);
  SHRK_TRY(g.st);
  cudaStream_t s = (cudaStream_t)stream;  // null = the legacy default stream
  const bool par = parallelism == SHRK_PAR_PARALLEL;
  int m = method;
  if (is_auto(m)) m = shrk_grid_appropriate(shrk_resolve_auto_method(m, par, p), p, nq);
  Epilogue epi;
  epi.mode = EPI_SUMS;
  epi.scale = 1.0;
  epi.out_re = d_re;
  epi.out_im = d_im;
  return sums_dispatch(d_q, (int64_t)nq, d_ev, (int64_t)p, eta, m, precision, cutoff,
                       epi, s, false);
}

shrk_status shrk_stieltjes_at_points(const double* q, size_t nq, const double* ev, size_t p,
                                     double eta, int method, int precision, double cutoff,
                                     int parallelism, double* raw_re, double* raw_im) {
  SHRK_TRY(check_common(p, eta, method, precision));
  SHRK_TRY(check_cutoff(cutoff));
  if (nq == 0) return SHRK_OK;
  Guard g;
  SHRK_TRY(g.st);
  cudaStream_t s = t_cur->stream;
  const bool par = parallelism == SHRK_PAR_PARALLEL;
  int m = method;
  if (is_auto(m)) m = shrk_grid_appropriate(shrk_resolve_auto_method(m, par, p), p, nq);
  void* dev = nullptr;
  SHRK_TRY(scratch_get(3, sizeof(double) * p, &dev));
  void* dq = nullptr;
  SHRK_TRY(scratch_get(6, sizeof(double) * nq, &dq));
  void* out = nullptr;
  SHRK_TRY(scratch_get(4, sizeof(double) * 2 * nq, &out));
  SHRK_TRY(h2d(dev, ev, sizeof(double) * p, s));
  set_source_hint((const double*)dev, ev, (int64_t)p);
  SHRK_TRY(h2d(dq, q, sizeof(double) * nq, s));
  Epilogue epi;
  epi.mode = EPI_SUMS;
  epi.scale = 1.0;
  epi.out_re = (double*)out;
  epi.out_im = (double*)out + nq;
  SHRK_TRY(sums_dispatch((const double*)dq, (int64_t)nq, (const double*)dev, (int64_t)p, eta,
                         m, precision, cutoff, epi, s, false));
  SHRK_TRY(d2h(raw_re, out, sizeof(double) * nq, s));
  SHRK_TRY(d2h(raw_im, (double*)out + nq, sizeof(double) * nq, s));
  return check_device_error(s);
}

shrk_status shrk_stieltjes_with_deriv(const double* ev, size_t p, double eta, double* re,
                                      double* im, double* dre, double* dim) {
  SHRK_TRY(check_common(p, eta, SHRK_M_BLOCKED, SHRK_PREC_F64));
  Guard g;
  SHRK_TRY(g.st);
  cudaStream_t s = t_cur->stream;
  void* dev = nullptr;
  SHRK_TRY(scratch_get(3, sizeof(double) * p, &dev));
  void* out = nullptr;
  SHRK_TRY(scratch_get(4, sizeof(double) * 4 * p, &out));
  SHRK_TRY(h2d(dev, ev, sizeof(double) * p, s));
  set_source_hint((const double*)dev, ev, (int64_t)p);
  double* o = (double*)out;
  SHRK_TRY(with_deriv((const double*)dev, (int64_t)p, eta, o, o + p, o + 2 * p, o + 3 * p, s));
  SHRK_TRY(d2h(re, o, sizeof(double) * p, s));
  SHRK_TRY(d2h(im, o + p, sizeof(double) * p, s));
  SHRK_TRY(d2h(dre, o + 2 * p, sizeof(double) * p, s));
  SHRK_TRY(d2h(dim, o + 3 * p, sizeof(double) * p, s));
  return check_device_error(s);
}

shrk_status shrk_stieltjes_batched_dev(const double* d_ev, const int64_t* d_offsets,
                                       size_t n_spectra, const double* d_eta, int precision,
                                       double* d_re, double* d_im, void* stream) {
  if (n_spectra == 0) return SHRK_OK;
  if (precision != SHRK_PREC_F64 && precision != SHRK_PREC_MIXED)
    return einval("unknown precision id");
  Guard g(stream);
  SHRK_TRY(g.st);
  cudaStream_t s = (cudaStream_t)stream;  // null = the legacy default stream
  return batched(d_ev, d_offsets, nullptr, (int64_t)n_spectra, d_eta, precision, d_re, d_im, s);
}

shrk_status shrk_stieltjes_batched(const double* ev, const int64_t* offsets, size_t n_spectra,
                                   const double* eta, int precision, double* out_re,
                                   double* out_im) {
  if (n_spectra == 0) return SHRK_OK;
  if (offsets[0] != 0) return einval("offsets[0] must be 0");
  for (size_t i = 0; i < n_spectra; ++i) {
    if (offsets[i + 1] <= offsets[i]) return einval("every spectrum must be non-empty");
    if (!(std::isfinite(eta[i]) && eta[i] > 0.0))
      return einval("eta must be a positive finite number");
  }
  if (precision != SHRK_PREC_F64 && precision != SHRK_PREC_MIXED)
    return einval("unknown precision id");
  const size_t total = (size_t)offsets[n_spectra];
  Guard g;
  SHRK_TRY(g.st);
  cudaStream_t s = t_cur->stream;
  void* dev = nullptr;
  SHRK_TRY(scratch_get(3, sizeof(double) * total, &dev));
  void* out = nullptr;
  SHRK_TRY(scratch_get(4, sizeof(double) * 2 * total, &out));
  void* doff = nullptr;
  SHRK_TRY(scratch_get(6, sizeof(int64_t) * (n_spectra + 1) + sizeof(double) * n_spectra, &doff));
  double* deta = (double*)((int64_t*)doff + n_spectra + 1);
  SHRK_TRY(h2d(dev, ev, sizeof(double) * total, s));
  SHRK_TRY(h2d(doff, offsets, sizeof(int64_t) * (n_spectra + 1), s));
  SHRK_TRY(h2d(deta, eta, sizeof(double) * n_spectra, s));
  SHRK_TRY(batched((const double*)dev, (const int64_t*)doff, offsets, (int64_t)n_spectra, deta,
                   precision, (double*)out, (double*)out + total, s));
  SHRK_TRY(d2h(out_re, out, sizeof(double) * total, s));
  SHRK_TRY(d2h(out_im, (double*)out + total, sizeof(double) * total, s));
  return check_device_error(s);
}

shrk_status shrk_batched_autotune(int precision, int force, int32_t* table) {
  if (precision != SHRK_PREC_F64 && precision != SHRK_PREC_MIXED)
    return einval("unknown precision id");
  Guard g;
  SHRK_TRY(g.st);
  int t[16];
  SHRK_TRY(batched_tune(precision, force != 0, t, t_cur->stream));
  if (table)
    for (int i = 0; i < 16; ++i) table[i] = t[i];
  return check_device_error(t_cur->stream);
}

shrk_status shrk_batched_set_tune(int precision, const int32_t* table) {
  if (precision != SHRK_PREC_F64 && precision != SHRK_PREC_MIXED)
    return einval("unknown precision id");
  if (!table) return einval("null table");
  int t[16];
  for (int i = 0; i < 16; ++i) t[i] = table[i];
  return batched_set_tune(precision, t);
}

shrk_status shrk_stieltjes_adjoint_dev(const double* d_ev, size_t p, double eta,
                                       const double* d_gre, const double* d_gim, int precision,
                                       double* d_grad, void* stream) {
  SHRK_TRY(check_common(p, eta, SHRK_M_BLOCKED, precision));
  Guard g(stream);
  SHRK_TRY(g.st);
  cudaStream_t s = (cudaStream_t)stream;  // null = the legacy default stream
  return adjoint(d_ev, (int64_t)p, eta, d_gre, d_gim, precision, d_grad, s);
}

static shrk_status check_cheb_method(int method, ChebParams* prm) {
  if (!is_cheb(method) || !cheb_preset(method, prm))
    return einval("the treecode adjoint takes a ChebCode method (chebcode, chebcode_fast, "
                  "chebcode_xtreme, chebcode_balanced)");
  return SHRK_OK;
}

shrk_status shrk_chebcode_evaluate_many_dev(const double* d_ev, size_t p, const double* d_etas,
                                            size_t n_eta, int method, double* d_re, double* d_im,
                                            void* stream) {
  if (p == 0) return einval("eigenvalues must be non-empty");
  if (n_eta == 0) return SHRK_OK;
  ChebParams prm;
  SHRK_TRY(check_cheb_method(method, &prm));
  Guard g(stream);
  SHRK_TRY(g.st);
  return chebcode_evaluate_many(d_ev, (int64_t)p, d_etas, (int64_t)n_eta, prm, d_re, d_im,
                                (cudaStream_t)stream);
}

shrk_status shrk_chebcode_evaluate_many(const double* ev, size_t p, const double* etas,
                                        size_t n_eta, int method, double* out_re,
                                        double* out_im) {
  if (p == 0) return einval("eigenvalues must be non-empty");
  if (n_eta == 0) return SHRK_OK;
  for (size_t k = 0; k < n_eta; ++k)
    if (!(std::isfinite(etas[k]) && etas[k] > 0.0))
      return einval("eta must be a positive finite number");
  ChebParams prm;
  SHRK_TRY(check_cheb_method(method, &prm));
  Guard g;
  SHRK_TRY(g.st);
  cudaStream_t s = t_cur->stream;
  void* dev = nullptr;
  SHRK_TRY(scratch_get(3, sizeof(double) * (p + n_eta), &dev));
  void* out = nullptr;
  SHRK_TRY(scratch_get(4, sizeof(double) * 2 * p * n_eta, &out));
  double* d = (double*)dev;
  SHRK_TRY(h2d(d, ev, sizeof(double) * p, s));
  set_source_hint(d, ev, (int64_t)p);
  SHRK_TRY(h2d(d + p, etas, sizeof(double) * n_eta, s));
  double* o = (double*)out;
  SHRK_TRY(chebcode_evaluate_many(d, (int64_t)p, d + p, (int64_t)n_eta, prm, o, o + p * n_eta,
                                  s));
  SHRK_TRY(d2h(out_re, o, sizeof(double) * p * n_eta, s));
  SHRK_TRY(d2h(out_im, o + p * n_eta, sizeof(double) * p * n_eta, s));
  return check_device_error(s);
}

shrk_status shrk_stieltjes_adjoint_treecode_dev(const double* d_ev, size_t p, double eta,
                                                const double* d_gre, const double* d_gim,
                                                int method, double* d_grad, void* stream) {
  SHRK_TRY(check_common(p, eta, SHRK_M_BLOCKED, SHRK_PREC_F64));
  ChebParams prm;
  SHRK_TRY(check_cheb_method(method, &prm));
  Guard g(stream);
  SHRK_TRY(g.st);
  cudaStream_t s = (cudaStream_t)stream;  // null = the legacy default stream
  return chebcode_adjoint(d_ev, (int64_t)p, eta, d_gre, d_gim, prm, d_grad, s);
}

shrk_status shrk_stieltjes_adjoint_treecode(const double* ev, size_t p, double eta,
                                            const double* g_re, const double* g_im, int method,
                                            double* grad) {
  SHRK_TRY(check_common(p, eta, SHRK_M_BLOCKED, SHRK_PREC_F64));
  ChebParams prm;
  SHRK_TRY(check_cheb_method(method, &prm));
  Guard g;
  SHRK_TRY(g.st);
  cudaStream_t s = t_cur->stream;
  void* dev = nullptr;
  SHRK_TRY(scratch_get(3, sizeof(double) * 3 * p, &dev));
  void* out = nullptr;
  SHRK_TRY(scratch_get(4, sizeof(double) * p, &out));
  double* d = (double*)dev;
  SHRK_TRY(h2d(d, ev, sizeof(double) * p, s));
  set_source_hint(d, ev, (int64_t)p);
  SHRK_TRY(h2d(d + p, g_re, sizeof(double) * p, s));
  SHRK_TRY(h2d(d + 2 * p, g_im, sizeof(double) * p, s));
  SHRK_TRY(chebcode_adjoint(d, (int64_t)p, eta, d + p, d + 2 * p, prm, (double*)out, s));
  SHRK_TRY(d2h(grad, out, sizeof(double) * p, s));
  return check_device_error(s);
}

shrk_status shrk_stieltjes_adjoint(const double* ev, size_t p, double eta, const double* g_re,
                                   const double* g_im, int precision, double* grad) {
  SHRK_TRY(check_common(p, eta, SHRK_M_BLOCKED, precision));
  Guard g;
  SHRK_TRY(g.st);
  cudaStream_t s = t_cur->stream;
  void* dev = nullptr;
  SHRK_TRY(scratch_get(3, sizeof(double) * 3 * p, &dev));
  void* out = nullptr;
  SHRK_TRY(scratch_get(4, sizeof(double) * p, &out));
  double* d = (double*)dev;
  SHRK_TRY(h2d(d, ev, sizeof(double) * p, s));
  set_source_hint(d, ev, (int64_t)p);
  SHRK_TRY(h2d(d + p, g_re, sizeof(double) * p, s));
  SHRK_TRY(h2d(d + 2 * p, g_im, sizeof(double) * p, s));
  SHRK_TRY(adjoint(d, (int64_t)p, eta, d + p, d + 2 * p, precision, (double*)out, s));
  SHRK_TRY(d2h(grad, out, sizeof(double) * p, s));
  return check_device_error(s);
}

// ------------------------------------------------------- consumers --
double shrk_shrinkage_factor(double li, double c, double mr, double mi) {
  double tr = c * li * mr, ti = c * li * mi;
  double dr = 1.0 - c + tr, di = ti;
  double n2 = dr * dr + di * di;
  return n2 > 0.0 ? li / n2 : li;
}
double shrk_inverse_bbp(double lh, double gamma, double sigma2) {
  return inverse_bbp(lh, gamma, sigma2);
}
double shrk_bbp_threshold(double gamma, double sigma2) { return bbp_threshold(gamma, sigma2); }
double shrk_mp_median_factor(double gamma) { return mp_median_factor(gamma); }

shrk_status shrk_detect_spikes_bema(const double* sorted, size_t p, double gamma, double margin,
                                    size_t* k, int64_t* idx, double* edge, double* sigma2) {
  SpikeSplit s;
  bema(sorted, p, gamma, margin, s);
  *k = s.k;
  for (size_t i = 0; i < s.k; ++i) idx[i] = (int64_t)s.idx[i];
  *edge = s.edge;
  *sigma2 = s.sigma2;
  return SHRK_OK;
}

shrk_status shrk_ledoit_wolf_shrinkage(const double* ev, size_t p, double c, int method,
                                       int precision, int parallelism, double eta, double* xi) {
  if (p == 0) return SHRK_OK;
  if (!std::isnan(eta)) SHRK_TRY(check_common(p, eta, method, precision));
  Guard g;
  SHRK_TRY(g.st);
  return lw_device(ev, p, c, method, precision, parallelism, eta, xi);
}

static shrk_status check_fmm(size_t p, double eta, int order) {
  if (p == 0) return einval("eigenvalues must be non-empty");
  if (p > (size_t)INT32_MAX) return einval("fmm: at most 2^31 - 1 eigenvalues");
  if (!(std::isfinite(eta) && eta > 0.0)) return einval("eta must be a positive finite number");
  if (order < 4 || order > 16) return einval("fmm: the expansion order must be in [4, 16]");
  return SHRK_OK;
}

shrk_status shrk_stieltjes_fmm_dev(const double* d_ev, size_t p, double eta, int order, int m2l,
                                   double* d_re, double* d_im, void* stream) {
  SHRK_TRY(check_fmm(p, eta, order));
  if (m2l != 0 && m2l != 1) return einval("fmm: m2l must be 0 (FP64) or 1 (tensor cores, TF32 x3)");
  Guard g(stream);
  SHRK_TRY(g.st);
  return fmm_all(d_ev, (int64_t)p, eta, order, m2l, d_re, d_im, (cudaStream_t)stream);
}

shrk_status shrk_stieltjes_fmm(const double* ev, size_t p, double eta, int order, int m2l,
                               double* out_re, double* out_im) {
  SHRK_TRY(check_fmm(p, eta, order));
  if (m2l != 0 && m2l != 1) return einval("fmm: m2l must be 0 (FP64) or 1 (tensor cores, TF32 x3)");
  Guard g;
  SHRK_TRY(g.st);
  cudaStream_t s = t_cur->stream;
  void* dev = nullptr;
  SHRK_TRY(scratch_get(3, sizeof(double) * p, &dev));
  void* out = nullptr;
  SHRK_TRY(scratch_get(4, sizeof(double) * 2 * p, &out));
  SHRK_TRY(h2d(dev, ev, sizeof(double) * p, s));
  set_source_hint((const double*)dev, ev, (int64_t)p);
  SHRK_TRY(fmm_all((const double*)dev, (int64_t)p, eta, order, m2l, (double*)out,
                   (double*)out + p, s));
  SHRK_TRY(d2h(out_re, out, sizeof(double) * p, s));
  SHRK_TRY(d2h(out_im, (double*)out + p, sizeof(double) * p, s));
  return check_device_error(s);
}

shrk_status shrk_stieltjes_scaled_ray_dev(const double* d_ev, size_t p, double scale,
                                          double* d_re, double* d_im, void* stream) {
  if (p == 0) return einval("eigenvalues must be non-empty");
  if (!(std::isfinite(scale) && scale > 0.0))
    return einval("scale must be a positive finite number");
  Guard g(stream);
  SHRK_TRY(g.st);
  return scaled_ray_sums(d_ev, (int64_t)p, scale, d_re, d_im, (cudaStream_t)stream);
}

shrk_status shrk_stieltjes_scaled_ray(const double* ev, size_t p, double scale, double* raw_re,
                                      double* raw_im) {
  if (p == 0) return einval("eigenvalues must be non-empty");
  if (!(std::isfinite(scale) && scale > 0.0))
    return einval("scale must be a positive finite number");
  Guard g;
  SHRK_TRY(g.st);
  cudaStream_t s = t_cur->stream;
  void* dev = nullptr;
  SHRK_TRY(scratch_get(3, sizeof(double) * p, &dev));
  void* out = nullptr;
  SHRK_TRY(scratch_get(4, sizeof(double) * 2 * p, &out));
  SHRK_TRY(h2d(dev, ev, sizeof(double) * p, s));
  set_source_hint((const double*)dev, ev, (int64_t)p);
  SHRK_TRY(scaled_ray_sums((const double*)dev, (int64_t)p, scale, (double*)out,
                           (double*)out + p, s));
  SHRK_TRY(d2h(raw_re, out, sizeof(double) * p, s));
  SHRK_TRY(d2h(raw_im, (double*)out + p, sizeof(double) * p, s));
  return check_device_error(s);
}

static shrk_status check_fft5_opts(size_t p, double eta, int order, double pad_eta_mult,
                                   double pad_range_frac) {
  if (p == 0) return einval("eigenvalues must be non-empty");
  if (!(std::isfinite(eta) && eta > 0.0)) return einval("eta must be a positive finite number");
  if (order != 2 && order != 4 && order != 6 && order != 8)
    return einval("order must be 2, 4, 6 or 8 stencil nodes");
  if (!std::isfinite(pad_eta_mult) || !std::isfinite(pad_range_frac))
    return einval("padding multipliers must be finite");
  return SHRK_OK;
}

shrk_status shrk_stieltjes_fft5_with_options_dev(const double* d_ev, size_t p, double eta,
                                                 int order, size_t m_override,
                                                 double pad_eta_mult, double pad_range_frac,
                                                 double* d_re, double* d_im, void* stream) {
  SHRK_TRY(check_fft5_opts(p, eta, order, pad_eta_mult, pad_range_frac));
  Guard g(stream);
  SHRK_TRY(g.st);
  cudaStream_t s = (cudaStream_t)stream;
  const double* ds = nullptr;
  double first = 0.0, last = 0.0;
  SHRK_TRY(sorted_sources(d_ev, (int64_t)p, &ds, &first, &last, s));
  Fft5Opts o;
  o.order = order;
  o.m_override = m_override;
  o.pad_eta_mult = pad_eta_mult;
  o.pad_range_frac = pad_range_frac;
  Epilogue epi;
  epi.mode = EPI_SUMS;
  epi.scale = 1.0;
  epi.out_re = d_re;
  epi.out_im = d_im;
  return fft5_points(d_ev, (int64_t)p, ds, (int64_t)p, first, last, eta, o, epi, s);
}

shrk_status shrk_stieltjes_fft5_with_options(const double* ev, size_t p, double eta, int order,
                                             size_t m_override, double pad_eta_mult,
                                             double pad_range_frac, double* raw_re,
                                             double* raw_im) {
  SHRK_TRY(check_fft5_opts(p, eta, order, pad_eta_mult, pad_range_frac));
  Guard g;
  SHRK_TRY(g.st);
  cudaStream_t s = t_cur->stream;
  void* dev = nullptr;
  SHRK_TRY(scratch_get(3, sizeof(double) * p, &dev));
  void* out = nullptr;
  SHRK_TRY(scratch_get(4, sizeof(double) * 2 * p, &out));
  SHRK_TRY(h2d(dev, ev, sizeof(double) * p, s));
  set_source_hint((const double*)dev, ev, (int64_t)p);
  const double* ds = nullptr;
  double first = 0.0, last = 0.0;
  SHRK_TRY(sorted_sources((const double*)dev, (int64_t)p, &ds, &first, &last, s));
  Fft5Opts o;
  o.order = order;
  o.m_override = m_override;
  o.pad_eta_mult = pad_eta_mult;
  o.pad_range_frac = pad_range_frac;
  Epilogue epi;
  epi.mode = EPI_SUMS;
  epi.scale = 1.0;
  epi.out_re = (double*)out;
  epi.out_im = (double*)out + p;
  SHRK_TRY(fft5_points((const double*)dev, (int64_t)p, ds, (int64_t)p, first, last, eta, o, epi,
                       s));
  SHRK_TRY(d2h(raw_re, out, sizeof(double) * p, s));
  SHRK_TRY(d2h(raw_im, (double*)out + p, sizeof(double) * p, s));
  return check_device_error(s);
}

// ------------------------------------------------ NUFFT stages apart --
// The point-sharded NUFFT over several GPUs: every rank splats its shard of
// the sources onto the common grid, the densities are summed (one all-reduce
// of m <= 65 536 doubles), and every rank evaluates its shard of the queries.

static shrk_status check_grid(int64_t m, double lo, double dx) {
  if (m < 2 || m > (int64_t)1 << 22 || ((m & (m - 1)) != 0 && m > (int64_t)1 << 21)) {
    set_error("grid: m must lie in [2, 2^22] (at most 2^21 when not a power of two)");
    return SHRK_EINVAL;
  }
  if (!std::isfinite(lo) || !std::isfinite(dx) || dx == 0.0) {
    set_error("grid: lo and dx must be finite and dx non-zero");
    return SHRK_EINVAL;
  }
  return SHRK_OK;
}

shrk_status shrk_nufft_grid(double first, double last, double eta, int64_t* m, double* lo,
                            double* dx) {
  if (!std::isfinite(first) || !std::isfinite(last)) {
    set_error("nufft_grid: first and last must be finite");
    return SHRK_EINVAL;
  }
  if (!(std::isfinite(eta) && eta > 0.0)) {
    set_error("eta must be a positive finite number");
    return SHRK_EINVAL;
  }
  if (!m || !lo || !dx) {
    set_error("nufft_grid: null output pointer");
    return SHRK_EINVAL;
  }
  nufft_geometry(first, last, eta, m, lo, dx);
  return SHRK_OK;
}

shrk_status shrk_nufft_density_dev(const double* d_src, size_t ns, int64_t m, double lo,
                                   double dx, double* d_density, void* stream) {
  SHRK_TRY(check_grid(m, lo, dx));
  if (ns > (size_t)INT32_MAX) {
    set_error("nufft_density: at most 2^31 - 1 sources per call");
    return SHRK_EINVAL;
  }
  Guard g(stream);
  SHRK_TRY(g.st);
  cudaStream_t s = (cudaStream_t)stream;
  const double* ds = d_src;
  if (ns > 0) {
    double first = 0.0, last = 0.0;
    SHRK_TRY(sorted_sources(d_src, (int64_t)ns, &ds, &first, &last, s));
  }
  return nufft_density(ds, (int64_t)ns, m, lo, dx, d_density, s);
}

shrk_status shrk_nufft_eval_dev(const double* d_density, int64_t m, double lo, double dx,
                                double eta, const double* d_q, size_t nq, double* d_re,
                                double* d_im, void* stream) {
  SHRK_TRY(check_grid(m, lo, dx));
  if (!(std::isfinite(eta) && eta > 0.0)) {
    set_error("eta must be a positive finite number");
    return SHRK_EINVAL;
  }
  if (nq == 0) return SHRK_OK;
  Guard g(stream);
  SHRK_TRY(g.st);
  cudaStream_t s = (cudaStream_t)stream;
  Epilogue epi;
  epi.mode = EPI_SUMS;
  epi.scale = 1.0;
  epi.out_re = d_re;
  epi.out_im = d_im;
  return nufft_eval(d_density, m, lo, dx, eta, d_q, (int64_t)nq, epi, s);
}

// inverse.rs safe_reciprocal: 1/x, or the largest double for x <= 0 or
// non-finite.
static double safe_reciprocal(double x) {
  return (x > 0.0 && std::isfinite(x)) ? 1.0 / x : std::numeric_limits<double>::max();
}

shrk_status shrk_inverse_nonlinear_shrinkage(const double* ev, size_t p, double c, int method,
                                             double* precision_ev, double* covariance_ev,
                                             double* smoothing, double* theta_out,
                                             double* htheta_out) {
  *smoothing = 0.0;
  if (p == 0) return SHRK_OK;
  if (!(std::isfinite(c) && c > 0.0 && c <= 1.0))
    return einval("concentration ratio c must be in (0, 1]");
  if (method < 0 || method > 2)
    return einval("unknown inverse shrinkage method (expected 0 qis, 1 lis or 2 gis)");
  for (size_t i = 0; i < p; ++i)
    if (!(std::isfinite(ev[i]) && ev[i] > 0.0))
      return einval("eigenvalues must be strictly positive for inverse shrinkage (found " +
                    std::to_string(ev[i]) + ")");
  // Ledoit-Wolf bandwidth (inverse.rs:170), then theta + i Htheta = ev_i m(z_i)
  // on the ray z_i = ev_i (1 + i h) from the GPU.
  const double p_f = (double)p, inv_p = 1.0 / p_f;
  const double h = std::pow(std::min(c * c, 1.0 / (c * c)), 0.35) / std::pow(p_f, 0.35);
  *smoothing = h;
  std::vector<double> re(p), im(p);
  SHRK_TRY(shrk_stieltjes_scaled_ray(ev, p, h, re.data(), im.data()));
  // inverse.rs:183-259, in the reference's evaluation order.
  std::vector<double> theta(p), htheta(p), inv_lambda(p), delta(p), omega(p);
  double min_inv = INFINITY, trace = 0.0;
  for (size_t i = 0; i < p; ++i) {
    theta[i] = ev[i] * re[i] * inv_p;
    htheta[i] = ev[i] * im[i] * inv_p;
    inv_lambda[i] = 1.0 / ev[i];
    min_inv = std::min(min_inv, inv_lambda[i]);
    trace += ev[i];
  }
  const double omc = 1.0 - c;
  for (size_t i = 0; i < p; ++i) {
    const double x = inv_lambda[i], th = theta[i];
    const double amp2 = theta[i] * theta[i] + htheta[i] * htheta[i];
    const double denom = omc * omc * x + 2.0 * c * omc * x * th + c * c * x * amp2;
    delta[i] = (denom > 0.0 && std::isfinite(denom)) ? 1.0 / denom : ev[i];
    const double lis = omc * x + 2.0 * c * x * th;
    omega[i] = lis > min_inv ? lis : min_inv;
  }
  if (method == 0) {  // QIS: trace-preserving rescale of the covariance
    double sum = 0.0;
    for (size_t i = 0; i < p; ++i) sum += delta[i];
    const double scale = (sum > 0.0 && std::isfinite(sum)) ? trace / sum : 1.0;
    for (size_t i = 0; i < p; ++i) {
      covariance_ev[i] = delta[i] * scale;
      precision_ev[i] = safe_reciprocal(covariance_ev[i]);
    }
  } else if (method == 1) {  // LIS
    for (size_t i = 0; i < p; ++i) {
      covariance_ev[i] = safe_reciprocal(omega[i]);
      precision_ev[i] = omega[i];
    }
  } else {  // GIS: geometric mean of the QIS and LIS covariance estimates
    for (size_t i = 0; i < p; ++i) {
      const double ratio = omega[i] / delta[i];
      precision_ev[i] = (ratio > 0.0 && std::isfinite(ratio)) ? std::sqrt(ratio)
                                                              : safe_reciprocal(ev[i]);
      covariance_ev[i] = safe_reciprocal(precision_ev[i]);
    }
  }
  if (theta_out) std::copy(theta.begin(), theta.end(), theta_out);
  if (htheta_out) std::copy(htheta.begin(), htheta.end(), htheta_out);
  return SHRK_OK;
}

shrk_status shrk_rie_shrinkage(const double* ev, size_t p, double c, int method, int precision,
                               int parallelism, double* xi) {
  if (p == 0) return SHRK_OK;
  {
    Guard g;
    SHRK_TRY(g.st);
    SHRK_TRY(lw_device(ev, p, c, method, precision, parallelism, NAN, xi));
  }
  double tr = 0.0, sh = 0.0;
  for (size_t i = 0; i < p; ++i) tr += ev[i];
  for (size_t i = 0; i < p; ++i) sh += xi[i];
  double scale = sh > 0.0 ? tr / sh : 1.0;  // shrinkage.rs:37-44
  for (size_t i = 0; i < p; ++i) xi[i] *= scale;
  return SHRK_OK;
}

shrk_status shrk_spectral_deconvolution(const double* ev, size_t p, double c, size_t n_points,
                                        double eta, double lmin, double lmax, int method,
                                        int precision, int parallelism, double cutoff,
                                        double* out7) {
  SHRK_TRY(check_cutoff(cutoff));
  if (p == 0 || n_points == 0) return SHRK_OK;
  Guard g;
  SHRK_TRY(g.st);
  return deconv_device(ev, p, c, n_points, eta, lmin, lmax, method, precision, parallelism, cutoff,
                       out7);
}

shrk_status shrk_estimate_population_eigenvalues(const double* ev, size_t p, double c,
                                                 double margin, int precision, size_t* k,
                                                 double* spikes, double* spike_sample,
                                                 double* bulk_edge, double* sigma2,
                                                 double* bulk_population, double* bulk_sample) {
  *k = 0;
  *bulk_edge = 0.0;
  *sigma2 = 0.0;
  if (p == 0) return SHRK_OK;
  SpikeSplit sp;
  detect_debias_split(ev, p, c, margin, sp);
  *k = sp.k;
  *bulk_edge = sp.edge;
  *sigma2 = sp.sigma2;
  std::copy(sp.spikes.begin(), sp.spikes.end(), spikes);
  std::copy(sp.spike_sample.begin(), sp.spike_sample.end(), spike_sample);
  std::copy(sp.bulk.begin(), sp.bulk.end(), bulk_sample);
  if (sp.bulk.empty()) return SHRK_OK;
  Guard g;
  SHRK_TRY(g.st);
  // RmtConfig::new(c): Blocked, Sequential, eta = 0.4/sqrt(p_bulk)
  return lw_device(sp.bulk.data(), sp.bulk.size(), c, SHRK_M_BLOCKED, precision,
                   SHRK_PAR_SEQUENTIAL, NAN, bulk_population);
}

shrk_status shrk_deconvolve_spiked(const double* ev, size_t p, double c, size_t n_points,
                                   double eta, double margin, int method, int precision,
                                   int parallelism, double cutoff, size_t* k, double* spikes,
                                   double* spike_sample, double* bulk_edge, double* sigma2,
                                   double* out7) {
  SHRK_TRY(check_cutoff(cutoff));
  *k = 0;
  *bulk_edge = 0.0;
  *sigma2 = 0.0;
  if (p == 0) return SHRK_OK;
  SpikeSplit sp;
  detect_debias_split(ev, p, c, margin, sp);
  *k = sp.k;
  *bulk_edge = sp.edge;
  *sigma2 = sp.sigma2;
  std::copy(sp.spikes.begin(), sp.spikes.end(), spikes);
  std::copy(sp.spike_sample.begin(), sp.spike_sample.end(), spike_sample);
  if (sp.bulk.empty()) return SHRK_OK;
  Guard g;
  SHRK_TRY(g.st);
  return deconv_device(sp.bulk.data(), sp.bulk.size(), c, n_points, eta, NAN, NAN, method,
                       precision, parallelism, cutoff, out7);
}

// --------------------------------------------------------- streams --
shrk_status shrk_stream_check(void* stream) {
  Guard g(stream);
  SHRK_TRY(g.st);
  return check_error_word(g.ctx, (cudaStream_t)stream);
}

shrk_status shrk_stream_release(void* stream) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return cuda_fail(e, "cudaGetDevice");
  Context* c = nullptr;
  {
    std::lock_guard<std::mutex> lk(g_ctx_mu);
    auto it = g_stream_ctx.find(std::make_pair(dev, (uintptr_t)stream));
    if (it == g_stream_ctx.end()) return SHRK_OK;
    c = it->second;
    g_stream_ctx.erase(it);
  }
  // No call can enter the context any more; wait for the one that may run.
  std::lock_guard<std::recursive_mutex> lk(c->mu);
  e = cudaStreamSynchronize((cudaStream_t)stream);
  release_context_memory(c);
  if (c->err) cudaFree(c->err);
  c->err = nullptr;
  if (e != cudaSuccess) return cuda_fail(e, "cudaStreamSynchronize(release)");
  return SHRK_OK;
}

// ------------------------------------------------------- profiling --
void shrk_timing_enable(int on) { g_timing = on != 0; }

void shrk_timing_reset(void) {
  std::lock_guard<std::mutex> lk(g_timing_mu);
  for (auto& t : g_timed) {
    cudaEventDestroy(t.a);
    cudaEventDestroy(t.b);
  }
  g_timed.clear();
  g_launches.store(0);
}

shrk_status shrk_timing_read(const char* name, int64_t* launches, double* total_ms) {
  std::lock_guard<std::mutex> lk(g_timing_mu);
  int64_t n = 0;
  double ms = 0.0;
  for (auto& t : g_timed) {
    if (name && t.family != name) continue;
    float f = 0.0f;
    cudaError_t e = cudaEventSynchronize(t.b);
    if (e == cudaSuccess) e = cudaEventElapsedTime(&f, t.a, t.b);
    if (e != cudaSuccess) return cuda_fail(e, "cudaEventElapsedTime");
    ++n;
    ms += f;
  }
  *launches = n;
  *total_ms = ms;
  return SHRK_OK;
}

int64_t shrk_launch_count(void) { return g_launches.load(); }

shrk_status shrk_measure_pipe_rates(double* fp32, double* fp64) {
  Guard g;
  SHRK_TRY(g.st);
  return measure_pipe_rates(fp32, fp64);
}

shrk_status shrk_measure_rcp_bias(double* uniform_mean, double* log_mean) {
  Guard g;
  SHRK_TRY(g.st);
  if (!uniform_mean || !log_mean) return einval("null output pointer");
  return measure_rcp_bias(uniform_mean, log_mean);
}

long long shrk_diag_set_wait_limit(long long cycles) { return set_wait_cycles(cycles); }

shrk_status shrk_diag_dgemm(int ta, int tb, int64_t m, int64_t n, int64_t k, double alpha,
                            const double* d_a, int64_t lda, const double* d_b, int64_t ldb,
                            double beta, double* d_c, int64_t ldc, void* stream) {
  if (m < 0 || n < 0 || k < 0 || !d_c || (k > 0 && (!d_a || !d_b))) {
    set_error("dgemm: invalid arguments");
    return SHRK_EINVAL;
  }
  if (lda < (ta ? k : m) || ldb < (tb ? n : k) || ldc < m || lda < 1 || ldb < 1 || ldc < 1) {
    set_error("dgemm: leading dimensions too small");
    return SHRK_EINVAL;
  }
  Guard g(stream);
  SHRK_TRY(g.st);
  return dgemm(ta != 0, tb != 0, m, n, k, alpha, d_a, lda, d_b, ldb, beta, d_c, ldc,
               (cudaStream_t)stream);
}

}  // extern "C"
