// TEST INFRASTRUCTURE ONLY (see oracle.h): the FP64 consumers of the
// transform -- Ledoit-Wolf / RIE shrinkage (src/deconvolution/shrinkage.rs:
// 22-84, src/spiked/estimation.rs:75-90), El Karoui MP inversion
// (src/deconvolution/mod.rs:116-259), BEMA spike detection
// (src/spiked/detection.rs:49-153), inverse BBP (estimation.rs:37-56), the
// stage-1 split (src/spiked/mod.rs:54-91) and the two pipelines
// (src/deconvolution/population.rs:72-116, hybrid.rs:96-138).
#include "oracle.h"

#include <cfloat>

#include <algorithm>
#include <cmath>
#include <vector>

namespace orc {

// shrinkage.rs:22-34
static double shrinkage_factor(double li, double c, double mr, double mi) {
  double tr = c * li * mr, ti = c * li * mi;
  double dr = 1.0 - c + tr, di = ti;
  double n2 = dr * dr + di * di;
  return n2 > 0.0 ? li / n2 : li;
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
// detection.rs:75-83
static double mp_median_factor(double gamma) {
  double g = std::min(std::max(gamma, 0.0), 1.0);
  return 0.999995823 - 0.333211332 * g - 0.0106766617 * g * g - 0.000758816762 * g * g * g -
         0.00256753402 * g * g * g * g;
}
// detection.rs:111-121
static double median_sorted(const double* s, size_t n) {
  if (n == 0) return 0.0;
  if (n % 2 == 0) return (s[n / 2 - 1] + s[n / 2]) / 2.0;
  return s[n / 2];
}

struct Bema { size_t k; double edge, sigma2; std::vector<size_t> idx; };

// detection.rs:134-153 (+ estimate_bulk_noise 98-105, scan_above 49-63).
static Bema bema(const double* sorted, size_t p, double gamma, double margin) {
  Bema b{0, 0.0, 0.0, {}};
  if (p == 0) return b;
  double sigma2 = median_sorted(sorted, p) / mp_median_factor(gamma);
  double edge = bbp_threshold(gamma, sigma2);
  double threshold = edge * std::max(margin, 1.0);
  for (size_t i = p; i-- > 0;) {
    if (sorted[i] > threshold) b.idx.push_back(i);
    else break;
  }
  std::reverse(b.idx.begin(), b.idx.end());
  b.k = b.idx.size();
  b.edge = edge;
  b.sigma2 = sigma2;
  return b;
}

struct Split {
  Bema det;
  std::vector<double> sorted, spikes, spike_sample, bulk;
};

// spiked/mod.rs:54-91 detect_debias_split.
static Split split(const double* ev, size_t p, double gamma, double margin) {
  Split s;
  s.sorted.assign(ev, ev + p);
  std::stable_sort(s.sorted.begin(), s.sorted.end());
  s.det = bema(s.sorted.data(), p, gamma, margin);
  for (size_t i : s.det.idx) {
    s.spike_sample.push_back(s.sorted[i]);
    s.spikes.push_back(inverse_bbp(s.sorted[i], gamma, s.det.sigma2));
  }
  size_t q = 0;
  for (size_t i = 0; i < p; ++i) {
    if (q < s.det.idx.size() && s.det.idx[q] == i) { ++q; continue; }
    s.bulk.push_back(s.sorted[i]);
  }
  return s;
}

// mod.rs:192-211 + estimation.rs:75-90 (eta NaN -> 0.4/sqrt(p)).
static int ledoit_wolf(const double* ev, size_t p, double c, int method, bool parallel,
                       double eta, double* out) {
  if (p == 0) return 0;
  int m = resolve_auto_method(method, parallel, p);
  if (std::isnan(eta)) eta = 0.4 / std::sqrt((double)p);
  std::vector<double> re(p), im(p);
  int st = compute_all(ev, p, eta, m, NAN, parallel, re.data(), im.data());
  if (st) return st;
  for (size_t i = 0; i < p; ++i) out[i] = shrinkage_factor(ev[i], c, re[i], im[i]);
  return 0;
}

// deconvolution/mod.rs:116-259; seven outputs of n_points each.
static int spectral_deconvolution(const double* ev, size_t p, double c, size_t n_points,
                                  double eta, double lmin, double lmax, int method, bool parallel,
                                  double cutoff, double* grid, double* density, double* w_re,
                                  double* sr, double* si, double* pr, double* pi) {
  if (p == 0) return 0;
  double eta_val = std::isnan(eta) ? 0.1 / std::sqrt((double)p) : eta;
  double mn = INFINITY, mx = -INFINITY;
  for (size_t i = 0; i < p; ++i) { mn = std::min(mn, ev[i]); mx = std::max(mx, ev[i]); }
  double range = (mx - mn) > 0.0 ? mx - mn : 1.0;
  double margin = 0.2 * range;
  double lo = std::isnan(lmin) ? std::max(mn - margin, 0.0) : lmin;
  double hi = std::isnan(lmax) ? mx + margin : lmax;
  double step = n_points > 1 ? (hi - lo) / ((double)n_points - 1.0) : 0.0;
  for (size_t k = 0; k < n_points; ++k) grid[k] = lo + step * (double)k;
  // config.rs:507-516 resolve_auto_at_points
  int m = method;
  if (is_auto(m)) m = grid_appropriate(resolve_auto_method(m, parallel, p), p, n_points);
  std::vector<double> rr(n_points), ri(n_points);
  int st = compute_at_points(grid, n_points, ev, p, eta_val, m, cutoff, parallel, rr.data(),
                             ri.data());
  if (st) return st;
  const double inv_p = 1.0 / (double)p;
  for (size_t k = 0; k < n_points; ++k) {
    double zr = grid[k], zi = eta_val;
    double gr = -rr[k] * inv_p, gi = ri[k] * inv_p;
    double zgr = zr * gr - zi * gi, zgi = zr * gi + zi * gr;
    double ar = 1.0 - c - c * zgr, ai = -c * zgi;
    double an = ar * ar + ai * ai;
    double wr = an > 0.0 ? (zr * ar + zi * ai) / an : zr;
    double mr = ar * gr - ai * gi, mi = ar * gi + ai * gr;
    density[k] = mi / M_PI;
    w_re[k] = wr;
    sr[k] = gr;
    si[k] = gi;
    pr[k] = mr;
    pi[k] = mi;
  }
  return 0;
}

// mod.rs:304-319 compute_stieltjes_scaled_ray with RmtConfig::new(c)'s
// Blocked method and no cutoff: stieltjes_sum_for_one -> the autovec sum
// (mod.rs:244-262, cacheblock.rs:124-134) at z_i = lambda_i (1 + i scale);
// RAW sums.  The parallel route maps the same per-point sums.
void scaled_ray(const double* ev, size_t p, double scale, double* re, double* im) {
#pragma omp parallel for schedule(static)
  for (long i = 0; i < (long)p; ++i) {
    const double eta = scale * ev[i];
    autovec_sum(ev[i], ev, p, eta, &re[i], &im[i]);
  }
}

static double safe_reciprocal(double x) {  // inverse.rs safe_reciprocal
  return (x > 0.0 && std::isfinite(x)) ? 1.0 / x : DBL_MAX;
}

// deconvolution/inverse.rs:156-269 inverse_nonlinear_shrinkage.
// method: 0 QIS, 1 LIS, 2 GIS.
void inverse_shrinkage(const double* ev, size_t p, double c, int method, double* prec,
                       double* cov, double* theta, double* htheta, double* smoothing) {
  if (p == 0) {
    *smoothing = 0.0;
    return;
  }
  const double p_f = (double)p;
  const double inv_p = 1.0 / p_f;
  const double h = std::pow(std::min(c * c, 1.0 / (c * c)), 0.35) / std::pow(p_f, 0.35);
  *smoothing = h;
  std::vector<double> re(p), im(p), inv_lambda(p), delta(p), omega(p);
  scaled_ray(ev, p, h, re.data(), im.data());
  double min_inv = INFINITY, trace = 0.0;
  for (size_t i = 0; i < p; ++i) {
    const double li = ev[i];
    theta[i] = li * re[i] * inv_p;
    htheta[i] = li * im[i] * inv_p;
    const double x = 1.0 / li;
    inv_lambda[i] = x;
    min_inv = std::min(min_inv, x);
    trace += li;
  }
  const double omc = 1.0 - c;
  for (size_t i = 0; i < p; ++i) {
    const double x = inv_lambda[i];
    const double th = theta[i];
    const double amp2 = theta[i] * theta[i] + htheta[i] * htheta[i];
    const double denom = omc * omc * x + 2.0 * c * omc * x * th + c * c * x * amp2;
    delta[i] = (denom > 0.0 && std::isfinite(denom)) ? 1.0 / denom : ev[i];
    const double lis = omc * x + 2.0 * c * x * th;
    omega[i] = lis > min_inv ? lis : min_inv;
  }
  if (method == 0) {
    double sum = 0.0;
    for (size_t i = 0; i < p; ++i) sum += delta[i];
    const double scale = (sum > 0.0 && std::isfinite(sum)) ? trace / sum : 1.0;
    for (size_t i = 0; i < p; ++i) {
      cov[i] = delta[i] * scale;
      prec[i] = safe_reciprocal(cov[i]);
    }
  } else if (method == 1) {
    for (size_t i = 0; i < p; ++i) {
      cov[i] = safe_reciprocal(omega[i]);
      prec[i] = omega[i];
    }
  } else {
    for (size_t i = 0; i < p; ++i) {
      const double ratio = omega[i] / delta[i];
      prec[i] = (ratio > 0.0 && std::isfinite(ratio)) ? std::sqrt(ratio)
                                                      : safe_reciprocal(ev[i]);
      cov[i] = safe_reciprocal(prec[i]);
    }
  }
}

}  // namespace orc

using namespace orc;

extern "C" {

double orc_shrinkage_factor(double li, double c, double mr, double mi) {
  return shrinkage_factor(li, c, mr, mi);
}
double orc_inverse_bbp(double lh, double gamma, double sigma2) { return inverse_bbp(lh, gamma, sigma2); }
double orc_bbp_threshold(double gamma, double sigma2) { return bbp_threshold(gamma, sigma2); }
double orc_mp_median_factor(double g) { return mp_median_factor(g); }

// detection.rs:134-153 on an ascending spectrum; idx receives k indices.
size_t orc_bema(const double* sorted, size_t p, double gamma, double margin, int64_t* idx,
                double* edge, double* sigma2) {
  Bema b = bema(sorted, p, gamma, margin);
  for (size_t i = 0; i < b.k; ++i) idx[i] = (int64_t)b.idx[i];
  *edge = b.edge;
  *sigma2 = b.sigma2;
  return b.k;
}

int orc_ledoit_wolf(const double* ev, size_t p, double c, int method, int parallel, double eta,
                    double* out) {
  return ledoit_wolf(ev, p, c, method, parallel != 0, eta, out);
}

// shrinkage.rs:60-84 rie_shrinkage (trace-rescaled).
int orc_rie(const double* ev, size_t p, double c, int method, int parallel, double* out) {
  if (p == 0) return 0;
  int st = ledoit_wolf(ev, p, c, method, parallel != 0, NAN, out);
  if (st) return st;
  double tr = 0.0, sh = 0.0;
  for (size_t i = 0; i < p; ++i) tr += ev[i];
  for (size_t i = 0; i < p; ++i) sh += out[i];
  double scale = sh > 0.0 ? tr / sh : 1.0;
  for (size_t i = 0; i < p; ++i) out[i] *= scale;
  return 0;
}

int orc_spectral_deconvolution(const double* ev, size_t p, double c, size_t n_points, double eta,
                               double lmin, double lmax, int method, int parallel, double cutoff,
                               double* out7) {
  double* o = out7;
  size_t n = n_points;
  return spectral_deconvolution(ev, p, c, n, eta, lmin, lmax, method, parallel != 0, cutoff, o,
                                o + n, o + 2 * n, o + 3 * n, o + 4 * n, o + 5 * n, o + 6 * n);
}

// population.rs:72-116.  Outputs: k, spikes (desc), spike_sample (desc),
// edge, sigma2, bulk_population (len p-k), bulk_sample (len p-k).
int orc_estimate_population(const double* ev, size_t p, double c, double margin, size_t* k,
                            double* spikes, double* spike_sample, double* edge, double* sigma2,
                            double* bulk_pop, double* bulk_sample) {
  *k = 0; *edge = 0.0; *sigma2 = 0.0;
  if (p == 0) return 0;
  Split s = split(ev, p, c, margin);
  *k = s.det.k;
  *edge = s.det.edge;
  *sigma2 = s.det.sigma2;
  for (size_t i = 0; i < s.det.k; ++i) {
    spikes[i] = s.spikes[s.det.k - 1 - i];
    spike_sample[i] = s.spike_sample[s.det.k - 1 - i];
  }
  std::copy(s.bulk.begin(), s.bulk.end(), bulk_sample);
  // RmtConfig::new(c): Blocked, Sequential, eta = 0.4/sqrt(p_bulk)
  return ledoit_wolf(s.bulk.data(), s.bulk.size(), c, BLOCKED, false, NAN, bulk_pop);
}

// hybrid.rs:96-138.  out7 receives the bulk deconvolution (7 x n_points).
int orc_deconvolve_spiked(const double* ev, size_t p, double c, size_t n_points, double eta,
                          double margin, int method, int parallel, double cutoff, size_t* k,
                          double* spikes, double* spike_sample, double* edge, double* sigma2,
                          double* out7) {
  *k = 0; *edge = 0.0; *sigma2 = 0.0;
  if (p == 0) return 0;
  Split s = split(ev, p, c, margin);
  *k = s.det.k;
  *edge = s.det.edge;
  *sigma2 = s.det.sigma2;
  for (size_t i = 0; i < s.det.k; ++i) {
    spikes[i] = s.spikes[s.det.k - 1 - i];
    spike_sample[i] = s.spike_sample[s.det.k - 1 - i];
  }
  return orc_spectral_deconvolution(s.bulk.data(), s.bulk.size(), c, n_points, eta, NAN, NAN,
                                    method, parallel, cutoff, out7);
}

void orc_scaled_ray(const double* ev, size_t p, double scale, double* re, double* im) {
  scaled_ray(ev, p, scale, re, im);
}

void orc_inverse_shrinkage(const double* ev, size_t p, double c, int method, double* prec,
                           double* cov, double* theta, double* htheta, double* smoothing) {
  inverse_shrinkage(ev, p, c, method, prec, cov, theta, htheta, smoothing);
}

}  // extern "C"
