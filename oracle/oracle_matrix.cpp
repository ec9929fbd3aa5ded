// TEST INFRASTRUCTURE ONLY (see oracle.h): restatement of the matrix
// front-end of src/pipeline/mod.rs -- symmetric_eigh (Jacobi, 502-585),
// reconstruct_covariance (45-111), compute_d_bulk (114-129),
// clean_eigensystem (197-242), renormalize_to_unit_diagonal (331-341),
// reconstruct_from_eigenvalues (376-392), precision_from_eigensystem
// (409-464) -- and of compute_angular_overlaps
// (src/eigenvector_overlaps/overlaps.rs:26-46).  Matrices are row-major
// p x p; eigenvectors are the columns.
#include "oracle.h"

#include <algorithm>
#include <cmath>
#include <numeric>
#include <vector>

extern "C" {
int orc_rie(const double* ev, size_t p, double c, int method, int parallel, double* out);
double orc_mp_median_factor(double g);
void orc_inverse_shrinkage(const double* ev, size_t p, double c, int method, double* prec,
                           double* cov, double* theta, double* htheta, double* smoothing);
}

namespace orc {

// mod.rs:480-490: out[:, j] = in[:, idx[j]].
static void permute_columns(const double* in, size_t p, const size_t* idx, double* out) {
  for (size_t j = 0; j < p; ++j)
    for (size_t r = 0; r < p; ++r) out[r * p + j] = in[r * p + idx[j]];
}

// mod.rs:502-585: threshold Jacobi; eigenvalues ascending, eigenvectors as
// columns in the same order.
static void symmetric_eigh(const double* m, size_t p, double* evals, double* evecs) {
  std::vector<double> a(m, m + p * p), v(p * p, 0.0);
  for (size_t i = 0; i < p; ++i) v[i * p + i] = 1.0;
  const double eps = 1e-15;
  for (int sweep = 0; sweep < 100; ++sweep) {
    double max_off = 0.0;
    for (size_t i = 0; i < p; ++i)
      for (size_t j = i + 1; j < p; ++j) max_off = std::max(max_off, std::fabs(a[i * p + j]));
    if (max_off < eps) break;
    const double threshold = max_off * 0.1;
    for (size_t i = 0; i < p; ++i) {
      for (size_t j = i + 1; j < p; ++j) {
        const double aij = a[i * p + j];
        if (std::fabs(aij) < threshold) continue;
        const double diff = a[j * p + j] - a[i * p + i];
        const double theta = 0.5 * diff / aij;
        double t = 1.0 / (std::fabs(theta) + std::sqrt(1.0 + theta * theta));
        if (theta < 0.0) t = -t;
        const double c = 1.0 / std::sqrt(1.0 + t * t);
        const double s = t * c;
        const double tau = s / (1.0 + c);
        const double h = t * aij;
        a[i * p + i] -= h;
        a[j * p + j] += h;
        a[i * p + j] = 0.0;
        a[j * p + i] = 0.0;
        for (size_t k = 0; k < p; ++k) {
          if (k != i && k != j) {
            const double g = a[k * p + i], hh = a[k * p + j];
            a[k * p + i] = g - s * (hh + g * tau);
            a[k * p + j] = hh + s * (g - hh * tau);
            a[i * p + k] = a[k * p + i];
            a[j * p + k] = a[k * p + j];
          }
        }
        for (size_t k = 0; k < p; ++k) {
          const double g = v[k * p + i], hh = v[k * p + j];
          v[k * p + i] = g - s * (hh + g * tau);
          v[k * p + j] = hh + s * (g - hh * tau);
        }
      }
    }
  }
  std::vector<double> ev(p);
  for (size_t i = 0; i < p; ++i) ev[i] = a[i * p + i];
  std::vector<size_t> order(p);
  std::iota(order.begin(), order.end(), 0);
  std::sort(order.begin(), order.end(), [&](size_t x, size_t y) { return ev[x] < ev[y]; });
  for (size_t i = 0; i < p; ++i) evals[i] = ev[order[i]];
  permute_columns(v.data(), p, order.data(), evecs);
}

// overlaps.rs:26-46
static void angular_overlaps(const double* l, size_t p, double c, double sigma2, double* a2) {
  for (size_t i = 0; i < p; ++i) {
    a2[i] = 0.0;
    const double diff = l[i] - sigma2;
    if (diff > 1e-12) {
      const double num = 1.0 - (c * (sigma2 * sigma2)) / (diff * diff);
      const double den = 1.0 + (c * sigma2) / diff;
      if (num > 0.0) a2[i] = std::min(num / den, 1.0 - 1e-15);
    }
  }
}

// mod.rs:114-129
static double d_bulk(const double* l, const double* a2, size_t p) {
  double sum = 0.0;
  size_t count = 0;
  for (size_t i = 0; i < p; ++i)
    if (a2[i] == 0.0) {
      sum += l[i];
      ++count;
    }
  if (count > 0) return sum / (double)count;
  double mn = INFINITY;
  for (size_t i = 0; i < p; ++i) mn = std::min(mn, l[i]);
  return mn;
}

// mod.rs:45-111: Sigma = d_bulk I + sum over active t of scale_t v_t v_t^T.
static void reconstruct_covariance(const double* v, size_t p, const double* l, const double* a2,
                                   double* sigma) {
  const double db = d_bulk(l, a2, p);
  std::vector<size_t> act;
  std::vector<double> scales;
  for (size_t i = 0; i < p; ++i)
    if (a2[i] > 0.0) {
      act.push_back(i);
      scales.push_back(a2[i] * (l[i] - db));
    }
  const size_t k = act.size();
  std::fill(sigma, sigma + p * p, 0.0);
  if (k == 0) {
    for (size_t i = 0; i < p; ++i) sigma[i * p + i] = db;
    return;
  }
  std::vector<double> vp(p * k);
  for (size_t t = 0; t < k; ++t)
    for (size_t r = 0; r < p; ++r) vp[r * k + t] = v[r * p + act[t]];
  for (size_t r = 0; r < p; ++r) {
    double diag = db;
    for (size_t t = 0; t < k; ++t) {
      const double vr = vp[r * k + t];
      diag += scales[t] * vr * vr;
    }
    sigma[r * p + r] = diag;
    for (size_t c = r + 1; c < p; ++c) {
      double val = 0.0;
      for (size_t t = 0; t < k; ++t) val += scales[t] * vp[r * k + t] * vp[c * k + t];
      sigma[r * p + c] = val;
      sigma[c * p + r] = val;
    }
  }
}

// mod.rs:197-242 (sort descending, RIE with RmtConfig::new(c), sigma2 from
// the MP-median-corrected median, overlaps, reconstruction).
static int clean_eigensystem(const double* evecs, const double* evals, size_t p, double c,
                             double* sigma, double* sorted_evecs, double* l_rie, double* a2,
                             double* sigma2) {
  std::vector<size_t> idx(p);
  std::iota(idx.begin(), idx.end(), 0);
  std::sort(idx.begin(), idx.end(), [&](size_t x, size_t y) { return evals[y] < evals[x]; });
  std::vector<double> sorted(p);
  for (size_t i = 0; i < p; ++i) sorted[i] = evals[idx[i]];
  permute_columns(evecs, p, idx.data(), sorted_evecs);
  int st = orc_rie(sorted.data(), p, c, BLOCKED, 0, l_rie);
  if (st) return st;
  // detection.rs:97-117 estimate_bulk_noise (median of the descending list)
  const double med = (p % 2 == 0) ? (sorted[p / 2 - 1] + sorted[p / 2]) / 2.0 : sorted[p / 2];
  *sigma2 = med / orc_mp_median_factor(c);
  angular_overlaps(l_rie, p, c, *sigma2, a2);
  reconstruct_covariance(sorted_evecs, p, l_rie, a2, sigma);
  return 0;
}

// mod.rs:331-341
static void renormalize(const double* s, size_t p, double* out) {
  for (size_t i = 0; i < p; ++i)
    if (s[i * p + i] <= 0.0) {
      std::copy(s, s + p * p, out);
      return;
    }
  std::vector<double> sc(p);
  for (size_t i = 0; i < p; ++i) sc[i] = 1.0 / std::sqrt(s[i * p + i]);
  for (size_t i = 0; i < p; ++i)
    for (size_t j = 0; j < p; ++j) out[i * p + j] = s[i * p + j] * sc[i] * sc[j];
}

// mod.rs:376-392
static void reconstruct_from_eigenvalues(const double* v, size_t p, const double* d, double* out) {
  for (size_t r = 0; r < p; ++r)
    for (size_t c = r; c < p; ++c) {
      double x = 0.0;
      for (size_t t = 0; t < p; ++t) x += d[t] * v[r * p + t] * v[c * p + t];
      out[r * p + c] = x;
      out[c * p + r] = x;
    }
}

}  // namespace orc

using namespace orc;

extern "C" {

void orc_symmetric_eigh(const double* m, size_t p, double* evals, double* evecs) {
  symmetric_eigh(m, p, evals, evecs);
}

void orc_angular_overlaps(const double* l, size_t p, double c, double sigma2, double* a2) {
  angular_overlaps(l, p, c, sigma2, a2);
}

int orc_clean_eigensystem(const double* evecs, const double* evals, size_t p, double c,
                          double* sigma, double* sorted_evecs, double* l_rie, double* a2,
                          double* sigma2) {
  return clean_eigensystem(evecs, evals, p, c, sigma, sorted_evecs, l_rie, a2, sigma2);
}

// mod.rs:244-331 + python.rs:729-731: eigendecompose, clean, optionally
// renormalize to unit diagonal.
int orc_clean_matrix(const double* m, size_t p, double c, int renorm, double* sigma,
                     double* sorted_evecs, double* l_rie, double* a2, double* sigma2) {
  std::vector<double> ev(p), vec(p * p);
  symmetric_eigh(m, p, ev.data(), vec.data());
  int st = clean_eigensystem(vec.data(), ev.data(), p, c, sigma, sorted_evecs, l_rie, a2, sigma2);
  if (st || !renorm) return st;
  std::vector<double> tmp(sigma, sigma + p * p);
  renormalize(tmp.data(), p, sigma);
  return 0;
}

void orc_renormalize(const double* s, size_t p, double* out) { renormalize(s, p, out); }

// mod.rs:409-464 precision_from_eigensystem.
void orc_precision_from_eigensystem(const double* evecs, const double* evals, size_t p, double c,
                                    int method, double* prec, double* sorted_evecs,
                                    double* prec_ev, double* cov_ev, double* smoothing) {
  std::vector<size_t> idx(p);
  std::iota(idx.begin(), idx.end(), 0);
  std::sort(idx.begin(), idx.end(), [&](size_t x, size_t y) { return evals[y] < evals[x]; });
  std::vector<double> sorted(p), th(p), hth(p);
  for (size_t i = 0; i < p; ++i) sorted[i] = evals[idx[i]];
  permute_columns(evecs, p, idx.data(), sorted_evecs);
  orc_inverse_shrinkage(sorted.data(), p, c, method, prec_ev, cov_ev, th.data(), hth.data(),
                        smoothing);
  reconstruct_from_eigenvalues(sorted_evecs, p, prec_ev, prec);
}

// mod.rs:466-478 estimate_precision_matrix.
void orc_estimate_precision_matrix(const double* m, size_t p, double c, int method, double* prec,
                                   double* sorted_evecs, double* prec_ev, double* cov_ev,
                                   double* smoothing) {
  std::vector<double> ev(p), vec(p * p);
  symmetric_eigh(m, p, ev.data(), vec.data());
  orc_precision_from_eigensystem(vec.data(), ev.data(), p, c, method, prec, sorted_evecs, prec_ev,
                                 cov_ev, smoothing);
}

}  // extern "C"
