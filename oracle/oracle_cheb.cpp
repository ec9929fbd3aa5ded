// TEST INFRASTRUCTURE ONLY (see oracle.h): restatement of the Chebyshev
// treecode of src/stieltjes/chebcode.rs (build 242-572, traversals 607-828,
// presets 926-998, batch evaluation 1148-1277) and the grid leaf-cap rule
// of src/stieltjes/mod.rs:361-370.
#include "oracle.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

namespace orc {

static const int MAX_TREE_DEPTH = 48;     // chebcode.rs:95
static const float OUTSIDE_THETA2 = 1.69f;  // chebcode.rs:108

struct NodeF32 { float lo, hi, accept_hw; uint32_t lo_idx, hi_idx; int32_t right; };

struct Tree {
  std::vector<double> sorted, lo, hi, accept_hw, nodes, w;
  std::vector<size_t> lo_idx, hi_idx;
  std::vector<int32_t> right;
  std::vector<NodeF32> node_f32;
  std::vector<float> panel_f32;
  int n;
  double theta_sq;
};

// chebcode.rs:242-246
static std::vector<double> cheb_nodes_m1(int n) {
  std::vector<double> s(n);
  for (int j = 0; j < n; ++j) s[j] = std::cos((double)j * M_PI / (double)(n - 1));
  return s;
}
// chebcode.rs:250-261
static std::vector<double> bary_weights_m1(int n) {
  std::vector<double> l(n);
  for (int j = 0; j < n; ++j) {
    double sign = (j % 2 == 0) ? 1.0 : -1.0;
    l[j] = (j == 0 || j == n - 1) ? 0.5 * sign : sign;
  }
  return l;
}

// chebcode.rs:309-337 barycentric_row.
static void bary_row(double x, const double* t, const double* lam, double* w, double* v, int n,
                     double mass) {
  double s = 0.0;
  int hit = -1;
  for (int j = 0; j < n; ++j) {
    double d = x - t[j];
    if (d == 0.0) { hit = j; break; }
    double q = lam[j] / d;
    v[j] = q;
    s += q;
  }
  if (hit >= 0) { w[hit] += mass; return; }
  double m = mass * (1.0 / s);
  for (int j = 0; j < n; ++j) w[j] = std::fma(m, v[j], w[j]);
}

// chebcode.rs:347-388 build_topology (+ set_node_positions 268-278).
static int32_t build_topology(Tree& T, const std::vector<double>& sm1, size_t lo_idx,
                              size_t hi_idx, size_t leaf_cap, int depth) {
  int32_t idx = (int32_t)T.lo.size();
  size_t count = hi_idx - lo_idx;
  double lo = T.sorted[lo_idx], hi = T.sorted[hi_idx - 1];
  T.lo.push_back(lo);
  T.hi.push_back(hi);
  double hw = 0.5 * (hi - lo);
  T.accept_hw.push_back(hw * hw / T.theta_sq);
  T.lo_idx.push_back(lo_idx);
  T.hi_idx.push_back(hi_idx);
  double c = 0.5 * (lo + hi), l = 0.5 * (hi - lo);
  for (int j = 0; j < T.n; ++j) {
    T.nodes.push_back(c + l * sm1[j]);
    T.w.push_back(0.0);
  }
  T.right.push_back(-1);
  if (count <= leaf_cap || depth >= MAX_TREE_DEPTH) return idx;
  double mid = lo + 0.5 * (hi - lo);
  const double* b = T.sorted.data();
  size_t split = (size_t)(std::upper_bound(b + lo_idx, b + hi_idx, mid) - b);
  if (split == lo_idx || split == hi_idx) split = (lo_idx + hi_idx) / 2;
  build_topology(T, sm1, lo_idx, split, leaf_cap, depth + 1);
  int32_t ri = build_topology(T, sm1, split, hi_idx, leaf_cap, depth + 1);
  T.right[idx] = ri;
  return idx;
}

// chebcode.rs:509-572 FlatChebTree::build.
static void build_tree(Tree& T, const double* sorted, size_t p, int n, double theta,
                       size_t leaf_cap) {
  T.sorted.assign(sorted, sorted + p);
  T.n = n;
  T.theta_sq = theta * theta;
  std::vector<double> lam = bary_weights_m1(n), sm1 = cheb_nodes_m1(n);
  build_topology(T, sm1, 0, p, leaf_cap, 0);
  const size_t nn = T.lo.size();
  std::vector<double> v(n);
  // fill_leaves (401-460): leaves are independent; sequential order here.
  for (size_t i = 0; i < nn; ++i) {
    if (T.right[i] >= 0) continue;
    double* w = &T.w[i * n];
    for (int j = 0; j < n; ++j) w[j] = 0.0;
    for (size_t k = T.lo_idx[i]; k < T.hi_idx[i]; ++k)
      bary_row(T.sorted[k], &T.nodes[i * n], lam.data(), w, v.data(), n, 1.0);
  }
  // merge_all_weights (474-506): reverse pre-order sweep.
  for (size_t pi = nn; pi-- > 0;) {
    if (T.right[pi] < 0) continue;
    double* pw = &T.w[pi * n];
    for (int j = 0; j < n; ++j) pw[j] = 0.0;
    const double* t = &T.nodes[pi * n];
    int32_t kids[2] = {(int32_t)pi + 1, T.right[pi]};
    for (int32_t ci : kids) {
      for (int ti = 0; ti < n; ++ti) {
        double m = T.w[(size_t)ci * n + ti];
        if (m == 0.0) continue;
        bary_row(T.nodes[(size_t)ci * n + ti], t, lam.data(), pw, v.data(), n, m);
      }
    }
  }
  // f32 mirrors (551-570).
  T.node_f32.resize(nn);
  T.panel_f32.assign(nn * 2 * n, 0.0f);
  for (size_t i = 0; i < nn; ++i) {
    T.node_f32[i] = {(float)T.lo[i], (float)T.hi[i], (float)T.accept_hw[i], (uint32_t)T.lo_idx[i],
                     (uint32_t)T.hi_idx[i], T.right[i]};
    for (int j = 0; j < n; ++j) {
      T.panel_f32[i * 2 * n + j] = (float)T.nodes[i * n + j];
      T.panel_f32[i * 2 * n + n + j] = (float)T.w[i * n + j];
    }
  }
}

// Exact leaf sum with the two-lane F64x2 schedule of 620-649 (unfused lane
// fma, true-division recip, hsum = l0 + l1, scalar tail).
static inline void leaf_sum(const double* xs, size_t len, double x, double eta, double eta2,
                            double* lr_out, double* li_out) {
  double ar0 = 0, ar1 = 0, ai0 = 0, ai1 = 0;
  size_t k = 0;
  while (k + 2 <= len) {
    double d0 = x - xs[k], d1 = x - xs[k + 1];
    double inv0 = 1.0 / (eta2 + d0 * d0), inv1 = 1.0 / (eta2 + d1 * d1);
    ar0 = ar0 + d0 * inv0;
    ar1 = ar1 + d1 * inv1;
    ai0 = ai0 + inv0;
    ai1 = ai1 + inv1;
    k += 2;
  }
  double lr = ar0 + ar1, li = ai0 + ai1;
  while (k < len) {
    double d = x - xs[k];
    double inv = 1.0 / (d * d + eta2);
    lr += d * inv;
    li += inv;
    ++k;
  }
  (void)eta;
  *lr_out = lr;
  *li_out = li;
}

// chebcode.rs:607-711 contribution_f64.
static void contribution_f64(const Tree& T, double x, double eta, double* re_o, double* im_o) {
  const int n = T.n;
  int32_t stack[MAX_TREE_DEPTH + 2];
  int top = 0;
  stack[top++] = 0;
  double re = 0.0, im = 0.0;
  const double eta2 = eta * eta;
  while (top > 0) {
    int32_t node = stack[--top];
    size_t ni = (size_t)node;
    if (T.right[ni] < 0) {
      double lr, li;
      leaf_sum(&T.sorted[T.lo_idx[ni]], T.hi_idx[ni] - T.lo_idx[ni], x, eta, eta2, &lr, &li);
      re += lr;
      im += eta * li;
      continue;
    }
    double lo = T.lo[ni], hi = T.hi[ni];
    double cl = std::max(std::max(lo - x, x - hi), 0.0);
    double d_sq = std::fma(cl, cl, eta2);
    if (T.accept_hw[ni] < d_sq) {
      const double* ts = &T.nodes[ni * n];
      const double* ws = &T.w[ni * n];
      double a0 = 0, a1 = 0, b0 = 0, b1 = 0;
      int j = 0;
      while (j + 2 <= n) {
        double d0 = x - ts[j], d1 = x - ts[j + 1];
        double inv0 = 1.0 / (eta2 + d0 * d0), inv1 = 1.0 / (eta2 + d1 * d1);
        double q0 = ws[j] * inv0, q1 = ws[j + 1] * inv1;
        a0 = a0 + q0 * d0;
        a1 = a1 + q1 * d1;
        b0 = b0 + q0;
        b1 = b1 + q1;
        j += 2;
      }
      double fr = a0 + a1, fi = b0 + b1;
      while (j < n) {
        double dj = x - ts[j];
        double q = ws[j] / (dj * dj + eta2);
        fr += q * dj;
        fi += q;
        ++j;
      }
      re += fr;
      im += eta * fi;
    } else {
      int32_t r = T.right[ni];
      if (r >= 0) {
        stack[top++] = r;
        stack[top++] = node + 1;
      }
    }
  }
  *re_o = re;
  *im_o = im;
}

// chebcode.rs:722-828 contribution_fast32 (four-lane f32 far field).
static void contribution_fast32(const Tree& T, double lambda, double eta, double* re_o,
                                double* im_o) {
  const int n = T.n;
  int32_t stack[MAX_TREE_DEPTH + 2];
  int top = 0;
  stack[top++] = 0;
  const float x = (float)lambda, e32 = (float)eta, eta2 = e32 * e32;
  float fre[4] = {0, 0, 0, 0}, fim[4] = {0, 0, 0, 0};
  double leaf_re = 0.0, leaf_im = 0.0;
  const double eta2d = eta * eta;
  while (top > 0) {
    int32_t node = stack[--top];
    const NodeF32& nd = T.node_f32[(size_t)node];
    if (nd.right < 0) {
      double lr, li;
      leaf_sum(&T.sorted[nd.lo_idx], (size_t)(nd.hi_idx - nd.lo_idx), lambda, eta, eta2d, &lr,
               &li);
      leaf_re += lr;
      leaf_im += eta * li;
      continue;
    }
    float cl = std::max(std::max(nd.lo - x, x - nd.hi), 0.0f);
    float d_sq = std::fmaf(cl, cl, eta2);
    float outside = (cl == 0.0f) ? d_sq : OUTSIDE_THETA2 * d_sq;
    if (nd.accept_hw < outside) {
      const float* ts = &T.panel_f32[(size_t)node * 2 * n];
      const float* ws = ts + n;
      int j = 0;
      while (j + 4 <= n) {
        for (int l = 0; l < 4; ++l) {
          float d = x - ts[j + l];
          float inv = 1.0f / (eta2 + d * d);
          float q = ws[j + l] * inv;
          fre[l] = fre[l] + q * d;
          fim[l] = fim[l] + q;
        }
        j += 4;
      }
      if (j < n) {
        float dt[4] = {0, 0, 0, 0}, wt[4] = {0, 0, 0, 0};
        for (int k = 0; k < n - j; ++k) {
          dt[k] = x - ts[j + k];
          wt[k] = ws[j + k];
        }
        for (int l = 0; l < 4; ++l) {
          float inv = 1.0f / (eta2 + dt[l] * dt[l]);
          float q = wt[l] * inv;
          fre[l] = fre[l] + q * dt[l];
          fim[l] = fim[l] + q;
        }
      }
    } else {
      stack[top++] = nd.right;
      stack[top++] = node + 1;
    }
  }
  float hr = (fre[0] + fre[1]) + (fre[2] + fre[3]);
  float hi = (fim[0] + fim[1]) + (fim[2] + fim[3]);
  *re_o = leaf_re + (double)hr;
  *im_o = leaf_im + eta * (double)hi;
}

// chebcode.rs:939-998.
bool cheb_preset(int method, ChebPreset* out) {
  switch (method) {
    case CHEBCODE: *out = {0.5, 11, 32, false}; return true;
    case CHEBCODE_FAST: *out = {1.0, 8, 32, true}; return true;
    case CHEBCODE_XTREME: *out = {0.25, 11, 16, false}; return true;
    case CHEBCODE_BALANCED: *out = {0.55, 11, 32, false}; return true;
    default: return false;
  }
}

// mod.rs:361-370.
size_t grid_leaf_cap(size_t n, size_t p, size_t nq, size_t preset_leaf) {
  const size_t MAX_GRID_LEAF = 8192;
  if (nq == 0 || p == 0) return preset_leaf;
  double optimal = (double)n * std::sqrt(2.0 * (double)p / (double)nq);
  size_t r = (size_t)std::round(optimal);
  size_t hi = std::max(MAX_GRID_LEAF, preset_leaf);
  return std::min(std::max(r, preset_leaf), hi);
}

// chebcode.rs:1079-1120 and ChebCodeBatch::evaluate_points 1241-1277: the
// tree is built over the ascending copy of the spectrum and evaluated at
// the query points in their given order (parallel and sequential
// evaluation are bit-identical: queries are independent).
void chebcode_points(const double* q, size_t nq, const double* ev, size_t p, double eta,
                     double theta, int n, int leaf_cap, bool f32, bool parallel, double* re,
                     double* im) {
  if (p == 0 || nq == 0) return;
  std::vector<double> sorted(ev, ev + p);
  if (!is_sorted_ascending(ev, p)) std::sort(sorted.begin(), sorted.end());
  Tree T;
  build_tree(T, sorted.data(), p, n, theta, (size_t)leaf_cap);
#pragma omp parallel for schedule(dynamic, 128) if (parallel)
  for (long k = 0; k < (long)nq; ++k) {
    if (f32) contribution_fast32(T, q[k], eta, &re[k], &im[k]);
    else contribution_f64(T, q[k], eta, &re[k], &im[k]);
  }
}

// chebcode.rs:836-915 contribution_x2: two etas per traversal, one per lane
// (x86 lanes: unfused multiply-adds, true division).  A node is accepted
// only when half_w^2 < theta^2 (cl^2 + min(eta)^2), the reference's own form.
static void contribution_x2(const Tree& T, double x, double e0, double e1, double* r0,
                            double* i0, double* r1, double* i1) {
  const int n = T.n;
  const double e2a = e0 * e0, e2b = e1 * e1;
  const double e_min = std::min(e0, e1);
  int32_t stack[MAX_TREE_DEPTH + 2];
  int top = 0;
  stack[top++] = 0;
  double ar0 = 0.0, ar1 = 0.0, ai0 = 0.0, ai1 = 0.0;
  while (top > 0) {
    const int32_t node = stack[--top];
    const size_t ni = (size_t)node;
    if (T.right[ni] < 0) {
      for (size_t k = T.lo_idx[ni]; k < T.hi_idx[ni]; ++k) {
        const double d = x - T.sorted[k];
        const double dd = d * d;
        const double inv0 = 1.0 / (e2a + dd), inv1 = 1.0 / (e2b + dd);
        ar0 = ar0 + d * inv0;
        ar1 = ar1 + d * inv1;
        ai0 = ai0 + e0 * inv0;
        ai1 = ai1 + e1 * inv1;
      }
      continue;
    }
    const double lo = T.lo[ni], hi = T.hi[ni];
    const double cl = x < lo ? lo - x : (x > hi ? x - hi : 0.0);
    const double d_sq = cl * cl + e_min * e_min;
    const double half_w = 0.5 * (hi - lo);
    if (half_w * half_w < T.theta_sq * d_sq) {
      for (int j = 0; j < n; ++j) {
        const double dj = x - T.nodes[ni * n + j];
        const double wj = T.w[ni * n + j];
        const double dd = dj * dj;
        const double inv0 = 1.0 / (e2a + dd), inv1 = 1.0 / (e2b + dd);
        const double wd = wj * dj;
        ar0 = ar0 + wd * inv0;
        ar1 = ar1 + wd * inv1;
        ai0 = ai0 + (wj * e0) * inv0;
        ai1 = ai1 + (wj * e1) * inv1;
      }
    } else {
      const int32_t r = T.right[ni];
      if (r >= 0) {
        stack[top++] = r;
        stack[top++] = node + 1;
      }
    }
  }
  *r0 = ar0;
  *i0 = ai0;
  *r1 = ar1;
  *i1 = ai1;
}

// chebcode.rs:1312-1361 ChebCodeBatch::evaluate_many: RAW sums at every
// eigenvalue (input order) for each eta; etas taken in pairs (an odd last
// eta is paired with itself).  out_re/out_im: n_eta x p row-major.
void evaluate_many(const double* ev, size_t p, const double* etas, size_t n_eta, double theta,
                   int n, int leaf_cap, double* out_re, double* out_im) {
  if (p == 0 || n_eta == 0) return;
  std::vector<double> sorted(ev, ev + p);
  if (!is_sorted_ascending(ev, p)) std::sort(sorted.begin(), sorted.end());
  Tree T;
  build_tree(T, sorted.data(), p, n, theta, (size_t)leaf_cap);
  for (size_t k = 0; k < n_eta; k += 2) {
    const double e0 = etas[k], e1 = (k + 1 < n_eta) ? etas[k + 1] : etas[k];
#pragma omp parallel for schedule(dynamic, 128)
    for (long i = 0; i < (long)p; ++i) {
      double r0, i0, r1, i1;
      contribution_x2(T, ev[i], e0, e1, &r0, &i0, &r1, &i1);
      out_re[k * p + i] = r0;
      out_im[k * p + i] = i0;
      if (k + 1 < n_eta) {
        out_re[(k + 1) * p + i] = r1;
        out_im[(k + 1) * p + i] = i1;
      }
    }
  }
}

}  // namespace orc

using namespace orc;

extern "C" {

void orc_chebcode_points(const double* q, size_t nq, const double* ev, size_t p, double eta,
                         double theta, int n, int leaf_cap, int f32, int parallel, double* re,
                         double* im) {
  chebcode_points(q, nq, ev, p, eta, theta, n, leaf_cap, f32 != 0, parallel != 0, re, im);
}

void orc_evaluate_many(const double* ev, size_t p, const double* etas, size_t n_eta,
                       double theta, int n, int leaf_cap, double* out_re, double* out_im) {
  evaluate_many(ev, p, etas, n_eta, theta, n, leaf_cap, out_re, out_im);
}

size_t orc_grid_leaf_cap(size_t n, size_t p, size_t nq, size_t preset_leaf) {
  return grid_leaf_cap(n, p, nq, preset_leaf);
}

// Exports the built tree (for GPU tree-build parity): returns the node
// count; when the output pointers are non-null they receive, per node, its
// interval, index range, right link and the n node positions / weights.
size_t orc_chebtree_export(const double* sorted, size_t p, int n, double theta, size_t leaf_cap,
                           double* lo, double* hi, int64_t* lo_idx, int64_t* hi_idx,
                           int32_t* right, double* nodes, double* w) {
  Tree T;
  build_tree(T, sorted, p, n, theta, leaf_cap);
  size_t nn = T.lo.size();
  if (lo) {
    for (size_t i = 0; i < nn; ++i) {
      lo[i] = T.lo[i];
      hi[i] = T.hi[i];
      lo_idx[i] = (int64_t)T.lo_idx[i];
      hi_idx[i] = (int64_t)T.hi_idx[i];
      right[i] = T.right[i];
    }
    std::memcpy(nodes, T.nodes.data(), nn * n * sizeof(double));
    std::memcpy(w, T.w.data(), nn * n * sizeof(double));
  }
  return nn;
}

}  // extern "C"
