// TEST INFRASTRUCTURE ONLY (see oracle.h): exact O(p^2) family, dispatchers,
// value+derivative, double-double truth and the FP64 direct-sum adjoint.
//
// Every function cites the reference file:line whose arithmetic it restates
// (paths inside the shrinkers crate).
#include "oracle.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>
#include <omp.h>

namespace orc {

// ---------------------------------------------------------------- policy --

bool is_auto(int m) { return m == AUTO || m == SPEED_AUTO || m == ACCURACY_AUTO; }

// pareto_autogen.rs:22-86 (bins and lookup), config.rs:543-555.
int resolve_auto_method(int m, bool parallel, size_t p) {
  struct Bin { size_t p_max; int ss, sp, as, ap; };
  static const Bin bins[] = {
      {1000, CHEBCODE_FAST, CHEBCODE_FAST, BLOCKED_TILED, BLOCKED},
      {2000, CHEBCODE_FAST, CHEBCODE_FAST, BLOCKED_TILED, AUTOVEC},
      {5000, CHEBCODE_FAST, CHEBCODE_FAST, BLOCKED_TILED, AUTOVEC},
      {10000, CHEBCODE_FAST, CHEBCODE_FAST, BLOCKED, BLOCKED_TILED},
      {20000, CHEBCODE_FAST, CHEBCODE_FAST, BLOCKED, BLOCKED},
      {50000, CHEBCODE_FAST, CHEBCODE_FAST, BLOCKED_TILED, BLOCKED},
      {SIZE_MAX, NUFFT, NUFFT, BLOCKED_TILED, BLOCKED},
  };
  if (m != AUTO && m != SPEED_AUTO && m != ACCURACY_AUTO) return m;
  const bool speed = (m != ACCURACY_AUTO);
  const Bin* b = &bins[6];
  for (const Bin& x : bins) {
    if (p <= x.p_max) { b = &x; break; }
  }
  if (speed) return parallel ? b->sp : b->ss;
  return parallel ? b->ap : b->as;
}

// config.rs:565-585.
int grid_appropriate(int m, size_t p, size_t nq) {
  // nq.saturating_mul(4) >= p
  if (nq > SIZE_MAX / 4 || nq * 4 >= p) return m;
  if (m == NUFFT && p >= 300000) return m;
  switch (m) {
    case FFT5: case FFT3: case FFT2: case NUFFT: case ADAPTIVE: case DST:
      return CHEBCODE_FAST;
    default:
      return m;
  }
}

// mod.rs:541-543.
bool is_sorted_ascending(const double* v, size_t n) {
  for (size_t i = 1; i < n; ++i)
    if (!(v[i - 1] <= v[i])) return false;
  return true;
}

// ------------------------------------------------------- per-point sums --

// naive.rs:15-25 with term.rs:26-31 (plain products, IEEE divide).
void naive_sum(double x, const double* ev, size_t p, double eta, double* re, double* im) {
  double sr = 0.0, si = 0.0;
  for (size_t j = 0; j < p; ++j) {
    double diff = x - ev[j];
    double denom = diff * diff + eta * eta;
    double inv = 1.0 / denom;
    sr += diff * inv;
    si += eta * inv;
  }
  *re = sr;
  *im = si;
}

// autovec.rs:19-30 with the hoisted term term.rs:40-45 (fused denominator).
void autovec_sum(double x, const double* ev, size_t p, double eta, double* re, double* im) {
  const double eta_sq = eta * eta;
  double sr = 0.0, sinv = 0.0;
  for (size_t j = 0; j < p; ++j) {
    double diff = x - ev[j];
    double denom = std::fma(diff, diff, eta_sq);
    double inv = 1.0 / denom;
    sr += diff * inv;
    sinv += inv;
  }
  *re = sr;
  *im = eta * sinv;
}

static size_t partition_lt(const double* v, size_t n, double x) {  // first v[i] >= x
  return (size_t)(std::lower_bound(v, v + n, x) - v);
}
static size_t partition_le(const double* v, size_t n, double x) {  // first v[i] > x
  return (size_t)(std::upper_bound(v, v + n, x) - v);
}

// cacheblock.rs:124-151 (cutoff = NaN means None -> autovec).
void sum_cutoff(double x, const double* ev, size_t p, double eta, double cutoff, double* re,
                double* im) {
  if (std::isnan(cutoff)) {
    autovec_sum(x, ev, p, eta, re, im);
    return;
  }
  const double eta_sq = eta * eta;
  const double window = cutoff * eta;
  size_t lo = partition_lt(ev, p, x - window);
  size_t hi = partition_le(ev, p, x + window);
  double sr = 0.0, sinv = 0.0;
  for (size_t j = lo; j < hi; ++j) {
    double diff = x - ev[j];
    double denom = std::fma(diff, diff, eta_sq);
    double inv = 1.0 / denom;
    sr += diff * inv;
    sinv += inv;
  }
  *re = sr;
  *im = eta * sinv;
}

// cacheblock.rs:531-546.
static void sum_windowed(double x, const double* ev, size_t p, double eta, double cut, double* re,
                         double* im) {
  const double eta_sq = eta * eta;
  const double window = cut * eta;
  size_t lo = partition_lt(ev, p, x - window);
  size_t hi = partition_le(ev, p, x + window);
  double sr = 0.0, si = 0.0;
  for (size_t j = lo; j < hi; ++j) {
    double diff = x - ev[j];
    double denom = std::fma(diff, diff, eta_sq);
    double inv = 1.0 / denom;
    sr = std::fma(diff, inv, sr);
    si = std::fma(eta, inv, si);
  }
  *re = sr;
  *im = si;
}

// ------------------------------------------------------ symmetric sweep --

// cacheblock.rs:841-954 (SoA sink 738-771; the AoS sink 773-818 performs the
// same operations in the same order).  Raw sums.
void symmetric_sweep(const double* evs, size_t p, double eta, double* R, double* I) {
  const double eta_sq = eta * eta;
  const double diag = 1.0 / eta;
  for (size_t k = 0; k < p; ++k) { R[k] = 0.0; I[k] = diag; }
  size_t t0 = 0;
  while (t0 < p) {
    size_t t1 = std::min(t0 + 4, p);
    double rr[4] = {0, 0, 0, 0}, ri[4] = {0, 0, 0, 0};
    for (size_t i = t0; i < t1; ++i) {
      double li = evs[i];
      size_t ii = i - t0;
      for (size_t j = i + 1; j < t1; ++j) {
        double d = li - evs[j];
        double inv = 1.0 / std::fma(d, d, eta_sq);
        rr[ii] = std::fma(d, inv, rr[ii]);
        ri[ii] = std::fma(eta, inv, ri[ii]);
        R[j] -= d * inv;
        I[j] += eta * inv;
      }
    }
    size_t j0 = t1;
    while (j0 + 4 <= p) {
      double l[4] = {evs[j0], evs[j0 + 1], evs[j0 + 2], evs[j0 + 3]};
      double cr[4] = {0, 0, 0, 0}, ci[4] = {0, 0, 0, 0};
      for (size_t i = t0; i < t1; ++i) {
        double li = evs[i];
        size_t ii = i - t0;
        for (int q = 0; q < 4; ++q) {
          double d = li - l[q];
          double inv = 1.0 / std::fma(d, d, eta_sq);
          rr[ii] = std::fma(d, inv, rr[ii]);
          ri[ii] = std::fma(eta, inv, ri[ii]);
          cr[q] = std::fma(-d, inv, cr[q]);
          ci[q] = std::fma(eta, inv, ci[q]);
        }
      }
      for (int q = 0; q < 4; ++q) {
        R[j0 + q] += cr[q];
        I[j0 + q] += ci[q];
      }
      j0 += 4;
    }
    while (j0 < p) {
      double lj = evs[j0];
      for (size_t i = t0; i < t1; ++i) {
        double d = evs[i] - lj;
        double inv = 1.0 / std::fma(d, d, eta_sq);
        rr[i - t0] = std::fma(d, inv, rr[i - t0]);
        ri[i - t0] = std::fma(eta, inv, ri[i - t0]);
        R[j0] -= d * inv;
        I[j0] += eta * inv;
      }
      j0 += 1;
    }
    for (size_t i = t0; i < t1; ++i) {
      R[i] += rr[i - t0];
      I[i] += ri[i - t0];
    }
    t0 = t1;
  }
}

// ------------------------------------------------------- tiled kernels --

// cacheblock.rs:1286-1424 tiled_one_block_no_cutoff.  Per target the
// accumulation order is: source quads in ascending order (lj0..lj3 inside a
// quad), then the 1-3 trailing sources; identical for the 4x-unrolled rows
// and the remainder rows, so one loop per target restates it exactly.
static void tiled_one_target(double t, const double* ev, size_t p, double eta, double eta_sq,
                             double* r, double* i) {
  double orr = *r, oi = *i;
  for (size_t j = 0; j < p; ++j) {
    double d = t - ev[j];
    double inv = 1.0 / std::fma(d, d, eta_sq);
    orr = std::fma(d, inv, orr);
    oi = std::fma(eta, inv, oi);
  }
  *r = orr;
  *i = oi;
}

void tiled_one_target_pub(double t, const double* ev, size_t p, double eta, double eta_sq,
                          double* r, double* i) {
  tiled_one_target(t, ev, p, eta, eta_sq, r, i);
}

// cacheblock.rs:1286-1424 with the reference's loop shape as well as its
// order: a block of TILED_BS targets (cacheblock.rs:1433) advances together
// over each quad of sources, four sources per target per step.  Each target
// still meets its sources in ascending order, so the sums are those of
// tiled_one_target bit for bit; the block's 32 accumulation chains and their
// divisions are independent, which is where the reference's speed comes
// from (the compiler vectorises the target loop when the ISA has FMA).
// Positions past nb repeat the first target and are discarded.
static const size_t TILED_BS = 32;

static void tiled_block(const double* t, size_t nb, const double* ev, size_t p, double eta,
                        double eta_sq, double* re, double* im) {
  double x[TILED_BS], ar[TILED_BS], ai[TILED_BS];
  for (size_t k = 0; k < TILED_BS; ++k) {
    x[k] = t[k < nb ? k : 0];
    ar[k] = 0.0;
    ai[k] = 0.0;
  }
  size_t j = 0;
  for (; j + 4 <= p; j += 4) {
    const double l0 = ev[j], l1 = ev[j + 1], l2 = ev[j + 2], l3 = ev[j + 3];
    for (size_t k = 0; k < TILED_BS; ++k) {
      double r = ar[k], i = ai[k];
      const double d0 = x[k] - l0;
      const double v0 = 1.0 / std::fma(d0, d0, eta_sq);
      r = std::fma(d0, v0, r);
      i = std::fma(eta, v0, i);
      const double d1 = x[k] - l1;
      const double v1 = 1.0 / std::fma(d1, d1, eta_sq);
      r = std::fma(d1, v1, r);
      i = std::fma(eta, v1, i);
      const double d2 = x[k] - l2;
      const double v2 = 1.0 / std::fma(d2, d2, eta_sq);
      r = std::fma(d2, v2, r);
      i = std::fma(eta, v2, i);
      const double d3 = x[k] - l3;
      const double v3 = 1.0 / std::fma(d3, d3, eta_sq);
      r = std::fma(d3, v3, r);
      i = std::fma(eta, v3, i);
      ar[k] = r;
      ai[k] = i;
    }
  }
  for (; j < p; ++j) {  // cacheblock.rs:1406-1423, the 1-3 trailing sources
    const double lj = ev[j];
    for (size_t k = 0; k < TILED_BS; ++k) {
      const double d = x[k] - lj;
      const double v = 1.0 / std::fma(d, d, eta_sq);
      ar[k] = std::fma(d, v, ar[k]);
      ai[k] = std::fma(eta, v, ai[k]);
    }
  }
  for (size_t k = 0; k < nb; ++k) {
    re[k] = ar[k];
    im[k] = ai[k];
  }
}

// cacheblock.rs:1454-1513 over blocks of TILED_BS targets on every host
// thread (raw sums at `targets`).
void tiled_blocks_parallel(const double* targets, size_t nt, const double* ev, size_t p,
                           double eta, double* re, double* im) {
  const double eta_sq = eta * eta;
  const long nblk = (long)((nt + TILED_BS - 1) / TILED_BS);
#pragma omp parallel for schedule(dynamic, 1)
  for (long b = 0; b < nblk; ++b) {
    const size_t t0 = (size_t)b * TILED_BS;
    const size_t nb = std::min(TILED_BS, nt - t0);
    tiled_block(targets + t0, nb, ev, p, eta, eta_sq, re + t0, im + t0);
  }
}

// cacheblock.rs:1255-1278 tiled_span_no_cutoff (bs only groups targets).
void tiled_span_no_cutoff(const double* targets, size_t nt, const double* ev, size_t p,
                          size_t /*bs*/, double eta, double* re, double* im) {
  const double eta_sq = eta * eta;
  for (size_t k = 0; k < nt; ++k) {
    re[k] = 0.0;
    im[k] = 0.0;
    tiled_one_target(targets[k], ev, p, eta, eta_sq, &re[k], &im[k]);
  }
}

// cacheblock.rs:1454-1513: disjoint target spans over all host threads.
// Same sums as tiled_one_target per target, taken in the block loop shape.
void tiled_parallel(const double* ev, size_t p, double eta, double* re, double* im) {
  tiled_blocks_parallel(ev, p, ev, p, eta, re, im);
}

// cacheblock.rs:167-224 + at_points_inner_loop 236-437.  Per query the
// accumulation runs over the sources in ascending order (pairs of sources,
// then the odd last one): re via fused mul_add, im as a plain sum of inv,
// scaled by eta at the end.  `cutoff` NaN = None.
void blocked_at_points(const double* q, size_t nq, const double* ev, size_t p, double eta,
                       double cutoff, double* re, double* im) {
  const double eta_sq = eta * eta;
  const bool cut_on = !std::isnan(cutoff);
  const double cut = cut_on ? cutoff * eta : INFINITY;
  for (size_t i = 0; i < nq; ++i) {
    double r = 0.0, s = 0.0;
    const double qi = q[i];
    for (size_t j = 0; j < p; ++j) {
      double d = qi - ev[j];
      double a = d < 0.0 ? -d : d;
      if (!cut_on || a <= cut) {
        double inv = 1.0 / std::fma(d, d, eta_sq);
        r = std::fma(d, inv, r);
        s += inv;
      }
    }
    re[i] = r;
    im[i] = s * eta;
  }
}

// cacheblock.rs:452-529 (lambda_j-outer window sweep).
void windowed(const double* ev, size_t p, double eta, double cut, double* R, double* I) {
  const double eta_sq = eta * eta;
  const double window = cut * eta;
  for (size_t k = 0; k < p; ++k) { R[k] = 0.0; I[k] = 0.0; }
  for (size_t jj = 0; jj < p; ++jj) {
    double lj = ev[jj];
    size_t lo = partition_lt(ev, p, lj - window);
    size_t hi = partition_le(ev, p, lj + window);
    for (size_t i = lo; i < hi; ++i) {
      double d = ev[i] - lj;
      double inv = 1.0 / std::fma(d, d, eta_sq);
      R[i] = std::fma(d, inv, R[i]);
      I[i] = std::fma(eta, inv, I[i]);
    }
  }
}

// cacheblock.rs:550-577.
void windowed_parallel(const double* ev, size_t p, double eta, double cut, double* R, double* I) {
#pragma omp parallel for schedule(dynamic, 64)
  for (long k = 0; k < (long)p; ++k) sum_windowed(ev[k], ev, p, eta, cut, &R[k], &I[k]);
}

// ----------------------------------------------------------- dispatch --

static const size_t PAR_TILED_MIN_P = 2000;  // mod.rs:518
static const size_t RAYON_MIN_P = 512;       // mod.rs:525

// mod.rs:562-594 dispatch_exact_blocked (raw sums).
static void dispatch_exact_blocked(const double* ev, size_t p, double eta, double cutoff,
                                   bool parallel, double* re, double* im) {
  if (!std::isnan(cutoff)) {
    if (parallel) windowed_parallel(ev, p, eta, cutoff, re, im);
    else windowed(ev, p, eta, cutoff, re, im);
    return;
  }
  if (parallel && p < RAYON_MIN_P) { symmetric_sweep(ev, p, eta, re, im); return; }
  if (parallel && p >= PAR_TILED_MIN_P) { tiled_parallel(ev, p, eta, re, im); return; }
  if (parallel) {  // compute_all_stieltjes_blocked_parallel, cacheblock.rs:80-96
#pragma omp parallel for schedule(dynamic, 16)
    for (long k = 0; k < (long)p; ++k) sum_cutoff(ev[k], ev, p, eta, NAN, &re[k], &im[k]);
    return;
  }
  symmetric_sweep(ev, p, eta, re, im);
}

// mod.rs:601-790 (exact family, ChebCode presets and NUFFT).  Scaled by 1/p.
int compute_all(const double* ev, size_t p, double eta, int method, double cutoff, bool parallel,
                double* re, double* im) {
  if (p == 0) return 0;
  const double inv_p = 1.0 / (double)p;
  method = resolve_auto_method(method, parallel, p);
  switch (method) {
    case BLOCKED:
    case BLOCKED_TILED:
      dispatch_exact_blocked(ev, p, eta, cutoff, parallel, re, im);
      break;
    case BLOCKED_WINDOWED:
      if (std::isnan(cutoff)) {
        // windowed kernels fall back to the exact blocked path without a
        // cutoff (cacheblock.rs:462-464, 557-559)
        if (parallel) {
#pragma omp parallel for schedule(dynamic, 16)
          for (long k = 0; k < (long)p; ++k) sum_cutoff(ev[k], ev, p, eta, NAN, &re[k], &im[k]);
        } else {
          symmetric_sweep(ev, p, eta, re, im);
        }
      } else if (parallel) {
        windowed_parallel(ev, p, eta, cutoff, re, im);
      } else {
        windowed(ev, p, eta, cutoff, re, im);
      }
      break;
    case BLOCKED_HYBRID: {  // mod.rs:738-757
      std::vector<double> r2(p), i2(p);
      if (parallel) {
#pragma omp parallel for schedule(dynamic, 16)
        for (long k = 0; k < (long)p; ++k) sum_cutoff(ev[k], ev, p, eta, NAN, &re[k], &i2[k]);
      } else {
        symmetric_sweep(ev, p, eta, re, i2.data());
      }
      if (std::isnan(cutoff)) symmetric_sweep(ev, p, eta, r2.data(), im);
      else windowed(ev, p, eta, cutoff, r2.data(), im);
      break;
    }
    case NAIVE:
    case AUTOVEC:
#pragma omp parallel for schedule(dynamic, 16) if (parallel)
      for (long k = 0; k < (long)p; ++k) {
        if (method == NAIVE) naive_sum(ev[k], ev, p, eta, &re[k], &im[k]);
        else autovec_sum(ev[k], ev, p, eta, &re[k], &im[k]);
      }
      break;
    case CHEBCODE:
    case CHEBCODE_FAST:
    case CHEBCODE_XTREME:
    case CHEBCODE_BALANCED: {
      ChebPreset pr;
      cheb_preset(method, &pr);
      chebcode_points(ev, p, ev, p, eta, pr.theta, pr.n, pr.leaf_cap, pr.f32, parallel, re, im);
      break;
    }
    case NUFFT:
      nufft_points(ev, p, ev, p, eta, parallel, re, im);
      break;
    case FFT5:
    case FFT3:
    case FFT2:  // mod.rs:634-641: one dual-convolution kernel for all three names
      if (fft5_points(ev, p, ev, p, eta, 8, 0, 1000.0, 0.75, re, im)) return 4;
      break;
    case ADAPTIVE:
    case DST: {
      // adaptive.rs:43-68 / mod.rs:672-690: fft5 real part, windowed
      // imaginary part (adaptive: ratio 10 by default; dst: the caller's
      // cutoff, the exact blocked sums without one).
      std::vector<double> tmp(p);
      if (fft5_points(ev, p, ev, p, eta, 8, 0, 1000.0, 0.75, re, tmp.data())) return 4;
      double cut = cutoff;
      if (method == ADAPTIVE && std::isnan(cut)) cut = 10.0;
      if (std::isnan(cut)) symmetric_sweep(ev, p, eta, tmp.data(), im);
      else windowed(ev, p, eta, cut, tmp.data(), im);
      break;
    }
    default:
      return 4;
  }
  for (size_t k = 0; k < p; ++k) {
    re[k] *= inv_p;
    im[k] *= inv_p;
  }
  return 0;
}

// mod.rs:394-494 (raw sums).
int compute_at_points(const double* q, size_t nq, const double* ev, size_t p, double eta,
                      int method, double cutoff, bool parallel, double* re, double* im) {
  if (is_auto(method)) {
    int r = resolve_auto_method(method, parallel, p);
    method = grid_appropriate(r, p, nq);
  }
  switch (method) {
    case BLOCKED: case BLOCKED_TILED: case BLOCKED_WINDOWED: case BLOCKED_HYBRID:
      if (parallel) {
#pragma omp parallel for schedule(dynamic, 16)
        for (long k = 0; k < (long)nq; ++k) sum_cutoff(q[k], ev, p, eta, cutoff, &re[k], &im[k]);
      } else {
        blocked_at_points(q, nq, ev, p, eta, cutoff, re, im);
      }
      return 0;
    case NUFFT:
      nufft_points(q, nq, ev, p, eta, parallel, re, im);
      return 0;
    case CHEBCODE: case CHEBCODE_FAST: case CHEBCODE_XTREME: case CHEBCODE_BALANCED: {
      ChebPreset pr;
      cheb_preset(method, &pr);
      size_t leaf = grid_leaf_cap(pr.n, p, nq, pr.leaf_cap);
      chebcode_points(q, nq, ev, p, eta, pr.theta, pr.n, (int)leaf, pr.f32, parallel, re, im);
      return 0;
    }
    case NAIVE:
#pragma omp parallel for schedule(dynamic, 16) if (parallel)
      for (long k = 0; k < (long)nq; ++k) naive_sum(q[k], ev, p, eta, &re[k], &im[k]);
      return 0;
    case FFT5: case FFT3: case FFT2:  // mod.rs:447-453
      return fft5_points(q, nq, ev, p, eta, 8, 0, 1000.0, 0.75, re, im);
    case AUTOVEC:
    // mod.rs:265-287: the remaining grid methods evaluate single points with
    // the autovec sum.
    case ADAPTIVE: case DST: case TREECODE: case EWALD: case HODLR:
#pragma omp parallel for schedule(dynamic, 16) if (parallel)
      for (long k = 0; k < (long)nq; ++k) autovec_sum(q[k], ev, p, eta, &re[k], &im[k]);
      return 0;
    default:
      return 4;
  }
}

}  // namespace orc

// ================================================================ C ABI ==
using namespace orc;

extern "C" {

int orc_resolve_auto_method(int m, int parallel, size_t p) { return resolve_auto_method(m, parallel != 0, p); }
int orc_grid_appropriate(int m, size_t p, size_t nq) { return grid_appropriate(m, p, nq); }

// term.rs:26-31
void orc_term(double li, double lj, double eta, double* re, double* im) {
  double diff = li - lj;
  double denom = diff * diff + eta * eta;
  double inv = 1.0 / denom;
  *re = diff * inv;
  *im = eta * inv;
}
// term.rs:40-45
void orc_term_hoisted(double li, double lj, double eta, double* re, double* inv_out) {
  double diff = li - lj;
  double denom = std::fma(diff, diff, eta * eta);
  double inv = 1.0 / denom;
  *re = diff * inv;
  *inv_out = inv;
}

void orc_naive_sum(double x, const double* ev, size_t p, double eta, double* re, double* im) {
  naive_sum(x, ev, p, eta, re, im);
}
void orc_autovec_sum(double x, const double* ev, size_t p, double eta, double* re, double* im) {
  autovec_sum(x, ev, p, eta, re, im);
}
void orc_symmetric_sweep(const double* ev, size_t p, double eta, double* re, double* im) {
  symmetric_sweep(ev, p, eta, re, im);
}
void orc_tiled_full_square(const double* ev, size_t p, double eta, double* re, double* im) {
  tiled_parallel(ev, p, eta, re, im);
}
void orc_blocked_at_points(const double* q, size_t nq, const double* ev, size_t p, double eta,
                           double cutoff, double* re, double* im) {
  blocked_at_points(q, nq, ev, p, eta, cutoff, re, im);
}
int orc_compute_all(const double* ev, size_t p, double eta, int method, double cutoff,
                    int parallel, double* re, double* im) {
  return compute_all(ev, p, eta, method, cutoff, parallel != 0, re, im);
}
int orc_compute_at_points(const double* q, size_t nq, const double* ev, size_t p, double eta,
                          int method, double cutoff, int parallel, double* re, double* im) {
  return compute_at_points(q, nq, ev, p, eta, method, cutoff, parallel != 0, re, im);
}

// cacheblock.rs:1525-1572 + mod.rs:805-848: f32 full-square tiled kernel,
// scaled by 1/p in f32.  Per target: sources in order, fused f32 mul_add.
void orc_all_f32(const float* ev, size_t p, float eta, float* re, float* im) {
  const float eta_sq = eta * eta;
  const float inv_p = 1.0f / (float)p;
#pragma omp parallel for schedule(dynamic, 32)
  for (long k = 0; k < (long)p; ++k) {
    float r = 0.0f, s = 0.0f;
    float t = ev[k];
    for (size_t j = 0; j < p; ++j) {
      float d = t - ev[j];
      float inv = 1.0f / std::fmaf(d, d, eta_sq);
      r = std::fmaf(d, inv, r);
      s = std::fmaf(eta, inv, s);
    }
    re[k] = r * inv_p;
    im[k] = s * inv_p;
  }
}

// autovec.rs:38-77: raw value + derivative w.r.t. the query point.
void orc_with_deriv(const double* ev, size_t p, double eta, double* re, double* im, double* dre,
                    double* dim) {
  const double eta_sq = eta * eta;
#pragma omp parallel for schedule(dynamic, 16)
  for (long k = 0; k < (long)p; ++k) {
    double x = ev[k];
    double s_re = 0.0, s_inv = 0.0, d_re = 0.0, d_im = 0.0;
    for (size_t j = 0; j < p; ++j) {
      double d = x - ev[j];
      double den = d * d + eta_sq;
      double inv = 1.0 / den;
      s_re += d * inv;
      s_inv += inv;
      d_re -= (d * d - eta_sq) * inv * inv;
      d_im -= (2.0 * d * eta) * inv * inv;
    }
    re[k] = s_re;
    im[k] = eta * s_inv;
    dre[k] = d_re;
    dim[k] = d_im;
  }
}

// ----------------------------------------------- double-double "truth" --
// Error-free transformations (Knuth TwoSum, Dekker TwoProduct with Veltkamp
// splitting); used only to measure error statistics of the fast paths.
struct dd { double hi, lo; };
static inline dd two_sum(double a, double b) {
  double s = a + b, bb = s - a;
  return {s, (a - (s - bb)) + (b - bb)};
}
static inline void split(double a, double* h, double* l) {
  double t = 134217729.0 * a;
  *h = t - (t - a);
  *l = a - *h;
}
static inline dd two_prod(double a, double b) {
  double p = a * b, ah, al, bh, bl;
  split(a, &ah, &al);
  split(b, &bh, &bl);
  return {p, ((ah * bh - p) + ah * bl + al * bh) + al * bl};
}
static inline dd dd_add(dd a, dd b) {
  dd s = two_sum(a.hi, b.hi);
  dd t = two_sum(a.lo, b.lo);
  s.lo += t.hi;
  s = two_sum(s.hi, s.lo);
  s.lo += t.lo;
  return two_sum(s.hi, s.lo);
}
static inline dd dd_mul(dd a, dd b) {
  dd p = two_prod(a.hi, b.hi);
  p.lo += a.hi * b.lo + a.lo * b.hi;
  return two_sum(p.hi, p.lo);
}
static inline dd dd_div(dd a, dd b) {
  double q1 = a.hi / b.hi;
  dd r = dd_add(a, dd_mul({-q1, 0.0}, b));
  double q2 = r.hi / b.hi;
  r = dd_add(r, dd_mul({-q2, 0.0}, b));
  double q3 = r.hi / b.hi;
  dd q = two_sum(q1, q2);
  return dd_add(q, {q3, 0.0});
}

// Raw sums S(x) = sum_j 1/((x - ev_j) - i eta) in double-double, rounded.
void orc_truth_points(const double* q, size_t nq, const double* ev, size_t p, double eta,
                      double* re, double* im) {
  const dd eta2 = two_prod(eta, eta);
#pragma omp parallel for schedule(dynamic, 1)
  for (long k = 0; k < (long)nq; ++k) {
    dd sr = {0, 0}, si = {0, 0};
    for (size_t j = 0; j < p; ++j) {
      dd d = two_sum(q[k], -ev[j]);
      dd den = dd_add(dd_mul(d, d), eta2);
      dd inv = dd_div({1.0, 0.0}, den);
      sr = dd_add(sr, dd_mul(d, inv));
      si = dd_add(si, inv);
    }
    si = dd_mul(si, {eta, 0.0});
    re[k] = sr.hi + sr.lo;
    im[k] = si.hi + si.lo;
  }
}

// FP64 direct-sum gradient of L = sum_j (w_j Re m_j + v_j Im m_j) with
// m_j = (1/p) sum_i 1/(ev_i - z_j), z_j = ev_j + i eta (no reference
// counterpart; derived from d/dev_k of the definition):
//   dL/dev_k = (1/p) sum_j [ (w_k - w_j)(a^2 - eta^2) - (v_k + v_j) 2 a eta ] / (a^2 + eta^2)^2,
//   a = ev_k - ev_j  (the i = j terms cancel exactly).
void orc_adjoint_direct(const double* ev, size_t p, double eta, const double* w, const double* v,
                        const long* idx, size_t nidx, double* grad) {
  const double eta_sq = eta * eta, inv_p = 1.0 / (double)p;
#pragma omp parallel for schedule(dynamic, 1)
  for (long t = 0; t < (long)nidx; ++t) {
    long k = idx ? idx[t] : t;
    double acc = 0.0;
    for (size_t j = 0; j < p; ++j) {
      double a = ev[k] - ev[j];
      double den = a * a + eta_sq;
      double inv = 1.0 / den;
      double num = (w[k] - w[j]) * (a * a - eta_sq) - (v[k] + v[j]) * 2.0 * a * eta;
      acc += num * inv * inv;
    }
    grad[t] = acc * inv_p;
  }
}

int orc_num_threads(void) { return omp_get_max_threads(); }
void orc_set_num_threads(int n) { omp_set_num_threads(n); }

}  // extern "C"

extern "C" {
// The reference's parallel all-points route (cacheblock.rs:1454-1513) for a
// subset of targets: per target the same fused accumulation over all
// sources, spread over every host thread.  Raw sums.  Used to time a bounded
// sample of a large workload.
void orc_tiled_targets(const double* targets, size_t nt, const double* ev, size_t p, double eta,
                       double* re, double* im) {
  const double eta_sq = eta * eta;
#pragma omp parallel for schedule(dynamic, 4)
  for (long k = 0; k < (long)nt; ++k) {
    re[k] = 0.0;
    im[k] = 0.0;
    orc::tiled_one_target_pub(targets[k], ev, p, eta, eta_sq, &re[k], &im[k]);
  }
}

// The same sums in the reference's block loop shape (32 targets x source
// quads, cacheblock.rs:1286-1424), the fast form of the route for timing.
void orc_tiled_targets_blocked(const double* targets, size_t nt, const double* ev, size_t p,
                               double eta, double* re, double* im) {
  orc::tiled_blocks_parallel(targets, nt, ev, p, eta, re, im);
}
}
