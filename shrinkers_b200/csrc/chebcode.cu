// Chebyshev treecode (ChebCode presets) for the Stieltjes transform.
//
// Replaces src/stieltjes/chebcode.rs: the flat pre-order tree of
// FlatChebTree::build (242-572: midpoint split, barycentric leaf fill,
// reverse-order parent merge, f32 mirrors) is built on the host in C++; the
// per-query evaluation (contribution_f64 607-711, contribution_fast32
// 722-828) runs on the GPU, one thread per query, queries in their given
// order (ascending queries keep a warp's traversals coherent).
//
// The evaluation reproduces the reference's x86 arithmetic operation by
// operation: two-lane leaf accumulation with a scalar tail, unfused lane
// multiply-adds, IEEE-rounded reciprocals (__drcp_rn / __frcp_rn equal the
// correctly rounded 1.0/x of the reference), right-then-left stack order,
// four-lane f32 far field folded once per query.  Given the same tree the
// GPU therefore returns the reference algorithm's sums bit for bit.
#include "common.cuh"
#include "epilogue.cuh"
#include "internal.h"

#include <algorithm>
#include <cmath>
#include <vector>

namespace shrk {

namespace {

constexpr int MAX_TREE_DEPTH = 48;        // chebcode.rs:95
constexpr float OUTSIDE_THETA2 = 1.69f;  // chebcode.rs:108
constexpr int MAX_N = 16;
constexpr int TREE_SLOTS = 16;  // scratch slots 16..21 hold the flat tree

struct NodeF32 {
  float lo, hi, accept_hw;
  uint32_t lo_idx, hi_idx;
  int32_t right;
};

struct HostTree {
  std::vector<double> lo, hi, accept_hw, nodes, w;
  std::vector<int64_t> lo_idx, hi_idx;
  std::vector<int32_t> right;
  int n = 0;
  double theta_sq = 0.0;
};

// chebcode.rs:309-337 barycentric_row.
void bary_row(double x, const double* t, const double* lam, double* w, double* v, int n,
              double mass) {
  double s = 0.0;
  int hit = -1;
  for (int j = 0; j < n; ++j) {
    double d = x - t[j];
    if (d == 0.0) {
      hit = j;
      break;
    }
    double q = lam[j] / d;
    v[j] = q;
    s += q;
  }
  if (hit >= 0) {
    w[hit] += mass;
    return;
  }
  double m = mass * (1.0 / s);
  for (int j = 0; j < n; ++j) w[j] = std::fma(m, v[j], w[j]);
}

// chebcode.rs:347-388 build_topology (+ set_node_positions 268-278).
int32_t build_topology(HostTree& T, const double* sorted, const std::vector<double>& sm1,
                       int64_t lo_idx, int64_t hi_idx, int64_t leaf_cap, int depth) {
  int32_t idx = (int32_t)T.lo.size();
  int64_t count = hi_idx - lo_idx;
  double lo = sorted[lo_idx], hi = sorted[hi_idx - 1];
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
  int64_t split = (int64_t)(std::upper_bound(sorted + lo_idx, sorted + hi_idx, mid) - sorted);
  if (split == lo_idx || split == hi_idx) split = (lo_idx + hi_idx) / 2;
  build_topology(T, sorted, sm1, lo_idx, split, leaf_cap, depth + 1);
  int32_t ri = build_topology(T, sorted, sm1, split, hi_idx, leaf_cap, depth + 1);
  T.right[idx] = ri;
  return idx;
}

// chebcode.rs:509-572 FlatChebTree::build (weights: fill_leaves 401-460,
// merge_all_weights 474-506).
void build_tree(HostTree& T, const double* sorted, int64_t p, int n, double theta,
                int64_t leaf_cap) {
  T.n = n;
  T.theta_sq = theta * theta;
  std::vector<double> sm1(n), lam(n);
  for (int j = 0; j < n; ++j) {
    sm1[j] = std::cos((double)j * M_PI / (double)(n - 1));
    double sign = (j % 2 == 0) ? 1.0 : -1.0;
    lam[j] = (j == 0 || j == n - 1) ? 0.5 * sign : sign;
  }
  const size_t est = (size_t)std::max<int64_t>(1, std::min<int64_t>(4 * p / std::max<int64_t>(leaf_cap, 1) + 32, 2 * p));
  T.lo.reserve(est); T.hi.reserve(est); T.accept_hw.reserve(est);
  T.lo_idx.reserve(est); T.hi_idx.reserve(est); T.right.reserve(est);
  T.nodes.reserve(est * n); T.w.reserve(est * n);
  build_topology(T, sorted, sm1, 0, p, leaf_cap, 0);
  const size_t nn = T.lo.size();
  std::vector<double> v(n);
  for (size_t i = 0; i < nn; ++i) {
    if (T.right[i] >= 0) continue;
    double* w = &T.w[i * n];
    for (int j = 0; j < n; ++j) w[j] = 0.0;
    for (int64_t k = T.lo_idx[i]; k < T.hi_idx[i]; ++k)
      bary_row(sorted[k], &T.nodes[i * n], lam.data(), w, v.data(), n, 1.0);
  }
  for (size_t pi = nn; pi-- > 0;) {
    if (T.right[pi] < 0) continue;
    double* pw = &T.w[pi * n];
    for (int j = 0; j < n; ++j) pw[j] = 0.0;
    const double* t = &T.nodes[pi * n];
    const int32_t kids[2] = {(int32_t)pi + 1, T.right[pi]};
    for (int32_t ci : kids)
      for (int ti = 0; ti < n; ++ti) {
        double m = T.w[(size_t)ci * n + ti];
        if (m == 0.0) continue;
        bary_row(T.nodes[(size_t)ci * n + ti], t, lam.data(), pw, v.data(), n, m);
      }
  }
}

// ----------------------------------------------------------- device --
struct DevTreeF64 {
  const double* lo;
  const double* hi;
  const double* accept_hw;
  const int64_t* lo_idx;
  const int64_t* hi_idx;
  const int32_t* right;
  const double* nodes;
  const double* w;
  int n;
};

struct EvalArgs {
  const double* q;
  int64_t nq;
  const double* sorted;
  double eta;
  DevTreeF64 t;
  const NodeF32* nf;
  const float* panel;
  Epilogue epi;
  int* err;
};

// Exact leaf sum, F64x2 schedule of chebcode.rs:620-649 (x86 semantics).
__device__ __forceinline__ void leaf_sum(const double* xs, int64_t len, double x, double eta2,
                                         double& lr_out, double& li_out) {
  double ar0 = 0.0, ar1 = 0.0, ai0 = 0.0, ai1 = 0.0;
  int64_t k = 0;
  for (; k + 2 <= len; k += 2) {
    const double d0 = x - xs[k], d1 = x - xs[k + 1];
    const double inv0 = __drcp_rn(eta2 + d0 * d0), inv1 = __drcp_rn(eta2 + d1 * d1);
    ar0 = ar0 + d0 * inv0;
    ar1 = ar1 + d1 * inv1;
    ai0 = ai0 + inv0;
    ai1 = ai1 + inv1;
  }
  double lr = ar0 + ar1, li = ai0 + ai1;
  for (; k < len; ++k) {
    const double d = x - xs[k];
    const double inv = __drcp_rn(d * d + eta2);
    lr += d * inv;
    li += inv;
  }
  lr_out = lr;
  li_out = li;
}

// chebcode.rs:607-711 contribution_f64.
__global__ void __launch_bounds__(128) cheb_eval_f64(const EvalArgs a) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= a.nq) return;
  const DevTreeF64& T = a.t;
  const int n = T.n;
  const double x = a.q[t], eta = a.eta, eta2 = eta * eta;
  int32_t stack[MAX_TREE_DEPTH + 2];
  int top = 0;
  stack[top++] = 0;
  double re = 0.0, im = 0.0;
  while (top > 0) {
    const int32_t node = stack[--top];
    const int32_t rt = T.right[node];
    if (rt < 0) {
      double lr, li;
      const int64_t l0 = T.lo_idx[node];
      leaf_sum(a.sorted + l0, T.hi_idx[node] - l0, x, eta2, lr, li);
      re += lr;
      im += eta * li;
      continue;
    }
    const double lo = T.lo[node], hi = T.hi[node];
    const double cl = fmax(fmax(lo - x, x - hi), 0.0);
    const double d_sq = fma(cl, cl, eta2);
    if (T.accept_hw[node] < d_sq) {
      const double* ts = T.nodes + (int64_t)node * n;
      const double* ws = T.w + (int64_t)node * n;
      double a0 = 0.0, a1 = 0.0, b0 = 0.0, b1 = 0.0;
      int j = 0;
      for (; j + 2 <= n; j += 2) {
        const double d0 = x - ts[j], d1 = x - ts[j + 1];
        const double inv0 = __drcp_rn(eta2 + d0 * d0), inv1 = __drcp_rn(eta2 + d1 * d1);
        const double q0 = ws[j] * inv0, q1 = ws[j + 1] * inv1;
        a0 = a0 + q0 * d0;
        a1 = a1 + q1 * d1;
        b0 = b0 + q0;
        b1 = b1 + q1;
      }
      double fr = a0 + a1, fi = b0 + b1;
      for (; j < n; ++j) {
        const double dj = x - ts[j];
        const double q = ws[j] / (dj * dj + eta2);
        fr += q * dj;
        fi += q;
      }
      re += fr;
      im += eta * fi;
    } else {
      if (top + 2 > MAX_TREE_DEPTH + 2) {  // cannot happen for a depth-capped tree
        atomicExch(a.err, DEV_ERR_BOUNDS);
        break;
      }
      stack[top++] = rt;
      stack[top++] = node + 1;
    }
  }
  epi_store(a.epi, t, x, re, im);
}

// chebcode.rs:722-828 contribution_fast32.
__global__ void __launch_bounds__(128) cheb_eval_f32(const EvalArgs a) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= a.nq) return;
  const int n = a.t.n;
  const double lambda = a.q[t], eta = a.eta, eta2d = eta * eta;
  const float x = (float)lambda, e32 = (float)eta, eta2 = e32 * e32;
  float fre[4] = {0.f, 0.f, 0.f, 0.f}, fim[4] = {0.f, 0.f, 0.f, 0.f};
  double leaf_re = 0.0, leaf_im = 0.0;
  int32_t stack[MAX_TREE_DEPTH + 2];
  int top = 0;
  stack[top++] = 0;
  while (top > 0) {
    const int32_t node = stack[--top];
    const NodeF32 nd = a.nf[node];
    if (nd.right < 0) {
      double lr, li;
      leaf_sum(a.sorted + nd.lo_idx, (int64_t)(nd.hi_idx - nd.lo_idx), lambda, eta2d, lr, li);
      leaf_re += lr;
      leaf_im += eta * li;
      continue;
    }
    const float cl = fmaxf(fmaxf(nd.lo - x, x - nd.hi), 0.0f);
    const float d_sq = fmaf(cl, cl, eta2);
    const float outside = (cl == 0.0f) ? d_sq : OUTSIDE_THETA2 * d_sq;
    if (nd.accept_hw < outside) {
      const float* ts = a.panel + (int64_t)node * 2 * n;
      const float* ws = ts + n;
      int j = 0;
      for (; j + 4 <= n; j += 4) {
#pragma unroll
        for (int l = 0; l < 4; ++l) {
          const float d = x - ts[j + l];
          const float inv = __frcp_rn(eta2 + d * d);
          const float q = ws[j + l] * inv;
          fre[l] = fre[l] + q * d;
          fim[l] = fim[l] + q;
        }
      }
      if (j < n) {
        float dt[4] = {0.f, 0.f, 0.f, 0.f}, wt[4] = {0.f, 0.f, 0.f, 0.f};
        for (int k = 0; k < n - j; ++k) {
          dt[k] = x - ts[j + k];
          wt[k] = ws[j + k];
        }
#pragma unroll
        for (int l = 0; l < 4; ++l) {
          const float inv = __frcp_rn(eta2 + dt[l] * dt[l]);
          const float q = wt[l] * inv;
          fre[l] = fre[l] + q * dt[l];
          fim[l] = fim[l] + q;
        }
      }
    } else {
      if (top + 2 > MAX_TREE_DEPTH + 2) {
        atomicExch(a.err, DEV_ERR_BOUNDS);
        break;
      }
      stack[top++] = nd.right;
      stack[top++] = node + 1;
    }
  }
  const float hr = (fre[0] + fre[1]) + (fre[2] + fre[3]);
  const float hi = (fim[0] + fim[1]) + (fim[2] + fim[3]);
  epi_store(a.epi, t, lambda, leaf_re + (double)hr, leaf_im + eta * (double)hi);
}

template <typename T>
shrk_status upload(int slot_base, int slot, const std::vector<T>& v, T** out, cudaStream_t s) {
  void* p = nullptr;
  SHRK_TRY(scratch_get(slot_base + slot, sizeof(T) * std::max<size_t>(v.size(), 1), &p));
  if (!v.empty())
    SHRK_CUDA(cudaMemcpyAsync(p, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice, s));
  *out = (T*)p;
  return SHRK_OK;
}

}  // namespace

// chebcode.rs:939-998.
bool cheb_preset(int method, ChebParams* out) {
  switch (method) {
    case SHRK_M_CHEBCODE: *out = {0.5, 11, 32, false}; return true;
    case SHRK_M_CHEBCODE_FAST: *out = {1.0, 8, 32, true}; return true;
    case SHRK_M_CHEBCODE_XTREME: *out = {0.25, 11, 16, false}; return true;
    case SHRK_M_CHEBCODE_BALANCED: *out = {0.55, 11, 32, false}; return true;
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

shrk_status chebcode_points(const double* d_q, int64_t nq, const double* h_sorted_src,
                            const double* d_sorted_src, int64_t ns, double eta,
                            const ChebParams& prm, const Epilogue& epi, cudaStream_t s) {
  if (nq <= 0 || ns <= 0) return SHRK_OK;
  if (prm.n < 2 || prm.n > MAX_N) {
    set_error("chebcode: interpolation order must be in [2, 16]");
    return SHRK_EINVAL;
  }
  HostTree T;
  build_tree(T, h_sorted_src, ns, prm.n, prm.theta, prm.leaf_cap);
  const size_t nn = T.lo.size();
  EvalArgs a;
  a.q = d_q;
  a.nq = nq;
  a.sorted = d_sorted_src;
  a.eta = eta;
  a.epi = epi;
  a.err = device_error_word();
  a.t.n = prm.n;
  a.nf = nullptr;
  a.panel = nullptr;
  if (!prm.f32) {
    double *lo, *hi, *acc, *nodes, *w;
    int64_t *li, *hix;
    int32_t* right;
    SHRK_TRY(upload(TREE_SLOTS, 0, T.lo, &lo, s));
    SHRK_TRY(upload(TREE_SLOTS, 1, T.hi, &hi, s));
    SHRK_TRY(upload(TREE_SLOTS, 2, T.accept_hw, &acc, s));
    std::vector<int64_t> idx(2 * nn);
    for (size_t i = 0; i < nn; ++i) {
      idx[i] = T.lo_idx[i];
      idx[nn + i] = T.hi_idx[i];
    }
    int64_t* didx;
    SHRK_TRY(upload(TREE_SLOTS, 3, idx, &didx, s));
    li = didx;
    hix = didx + nn;
    SHRK_TRY(upload(TREE_SLOTS, 4, T.right, &right, s));
    std::vector<double> nw(2 * nn * prm.n);
    std::copy(T.nodes.begin(), T.nodes.end(), nw.begin());
    std::copy(T.w.begin(), T.w.end(), nw.begin() + nn * prm.n);
    double* dnw;
    SHRK_TRY(upload(TREE_SLOTS, 5, nw, &dnw, s));
    nodes = dnw;
    w = dnw + nn * prm.n;
    a.t.lo = lo;
    a.t.hi = hi;
    a.t.accept_hw = acc;
    a.t.lo_idx = li;
    a.t.hi_idx = hix;
    a.t.right = right;
    a.t.nodes = nodes;
    a.t.w = w;
    LaunchScope ls("cheb_eval_f64", s);
    cheb_eval_f64<<<(unsigned)((nq + 127) / 128), 128, 0, s>>>(a);
    SHRK_CUDA(cudaGetLastError());
  } else {
    std::vector<NodeF32> nf(nn);
    std::vector<float> panel(nn * 2 * prm.n);
    for (size_t i = 0; i < nn; ++i) {
      nf[i] = {(float)T.lo[i], (float)T.hi[i], (float)T.accept_hw[i], (uint32_t)T.lo_idx[i],
               (uint32_t)T.hi_idx[i], T.right[i]};
      for (int j = 0; j < prm.n; ++j) {
        panel[i * 2 * prm.n + j] = (float)T.nodes[i * prm.n + j];
        panel[i * 2 * prm.n + prm.n + j] = (float)T.w[i * prm.n + j];
      }
    }
    NodeF32* dnf;
    float* dpanel;
    SHRK_TRY(upload(TREE_SLOTS, 0, nf, &dnf, s));
    SHRK_TRY(upload(TREE_SLOTS, 1, panel, &dpanel, s));
    a.nf = dnf;
    a.panel = dpanel;
    LaunchScope ls("cheb_eval_f32", s);
    cheb_eval_f32<<<(unsigned)((nq + 127) / 128), 128, 0, s>>>(a);
    SHRK_CUDA(cudaGetLastError());
  }
  // The host vectors feeding the uploads must outlive the copies.
  SHRK_CUDA(cudaStreamSynchronize(s));
  return SHRK_OK;
}

}  // namespace shrk
