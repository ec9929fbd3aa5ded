// Dyadic Chebyshev FMM for the Stieltjes sums S(x_t) = sum_j 1/((x_t - s_j) - i eta)
// at every source (all points), on sm_100a.
//
// No reference counterpart: the crate's ChebCode (src/stieltjes/chebcode.rs)
// is a treecode -- node expansions evaluated directly at each query (M2P) --
// and is reproduced bit for bit by chebcode.cu.  This is the dual-tree
// variant with P2M / M2M / M2L / L2L / L2P on a dyadic tree, where the
// kernel's translation invariance makes every M2L matrix depend only on the
// level and the box offset, so the far field is a batch of small dense
// contractions with shared matrices.  Its accuracy class is set by the
// expansion order n (measured against the exact sums).
//
// Tree: the spectrum's range [a, a + W) is cut into 2^l boxes at level l;
// the leaf level L is the coarsest at which no box holds more than
// FMM_OCC sources (at most FMM_LMAX).  Only boxes that hold sources exist:
// the leaves are the runs of equal leaf keys of the sorted sources, and the
// boxes of level l are the runs of leaf keys >> (L - l), numbered level after
// level by one scan over (level, leaf) flags.
//
// Expansions (n Chebyshev points of the first kind tau_j on [-1, 1],
// barycentric weights lambda_j): the multipole of a box is the vector of
// Lagrange-basis sums W_j = sum_{s in box} l_j((s - c)/(h/2)); a child's
// vector moves to its parent through the fixed matrices T_side[j][k] =
// l_j(side/2 + tau_k/2); M2L from source box A to target box B at offset
// o = key_B - key_A (|o| in {2, 3}: the children of the parent's neighbours
// that do not touch B) is L_B[i] += sum_j W_A[j] / ((h/2)(2o + tau_i - tau_j) - i eta);
// L2L applies T_side^T; L2P interpolates L at the target; the leaf and its
// two neighbours are summed directly in FP64.
#include "common.cuh"

#include <atomic>
#include "internal.h"

#include <cub/cub.cuh>

#include <algorithm>
#include <cmath>
#include <string>
#include <vector>

namespace shrk {

namespace {

constexpr int FMM_MAXN = 16;
constexpr int FMM_LMAX = 22;
constexpr int FMM_OCC = 48;

// scratch slots 39..45 (see the slot map in capi.cu)
constexpr int SLOT_KEYS = 39;    // per source: leaf key, run flag / leaf index
constexpr int SLOT_LEAF = 40;    // leaves: key, first source
constexpr int SLOT_LVL = 41;     // (level, leaf) flags -> global box ids
constexpr int SLOT_BOX = 42;     // boxes: key, first leaf, level
constexpr int SLOT_EXP = 43;     // expansions W, Lre, Lim
constexpr int SLOT_TAB = 44;     // tables: tau, lambda, T_left, T_right, M2L
constexpr int SLOT_TMP = 45;     // CUB temporaries, small host-read values

struct FmmGeom {
  double a, W;       // domain [a, a + W)
  int L;             // leaf level
  int n;             // expansion order
  double eta;
};

__device__ __forceinline__ int key_at(double s, double a, double W, int l) {
  const double u = (s - a) / W;
  long long k = (long long)(u * (double)(1LL << l));
  const long long top = (1LL << l) - 1;
  return (int)(k < 0 ? 0 : (k > top ? top : k));
}

// Bit l of *mask: some FMM_OCC + 1 consecutive sorted sources share a box of
// level l (the level is too coarse).
__global__ void level_probe_kernel(const double* __restrict__ s, int64_t ns, double a, double W,
                                   unsigned* __restrict__ mask) {
  const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (j + FMM_OCC >= ns) return;
  const double x0 = s[j], x1 = s[j + FMM_OCC];
  unsigned bits = 0;
  for (int l = 2; l <= FMM_LMAX; ++l)
    if (key_at(x0, a, W, l) == key_at(x1, a, W, l)) bits |= 1u << l;
  if (bits) atomicOr(mask, bits);
}

// The leaf level: the coarsest level l >= 2 whose bit is clear in the probe
// mask (FMM_LMAX when none is).
__host__ __device__ __forceinline__ int leaf_level(unsigned mask) {
  for (int l = 2; l <= FMM_LMAX; ++l)
    if (!((mask >> l) & 1u)) return l;
  return FMM_LMAX;
}

// Leaf key of every source and the start of each run of equal keys; the leaf
// level comes from the probe mask on the device, so the host reads the mask
// back together with the leaf count.
__global__ void leaf_flags_kernel(const double* __restrict__ s, int64_t ns, double a, double W,
                                  const unsigned* __restrict__ mask, int* __restrict__ key,
                                  int* __restrict__ flag) {
  const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= ns) return;
  const int L = leaf_level(*mask);
  const int k = key_at(s[j], a, W, L);
  key[j] = k;
  flag[j] = (j == 0 || key_at(s[j - 1], a, W, L) != k) ? 1 : 0;
}

// incl = inclusive scan of the run flags: leaf index of source j = incl[j] - 1.
__global__ void leaf_compact_kernel(const int* __restrict__ key, const int* __restrict__ flag,
                                    const int* __restrict__ incl, int64_t ns,
                                    int* __restrict__ leaf_key, int* __restrict__ leaf_start) {
  const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= ns) return;
  if (flag[j]) {
    leaf_key[incl[j] - 1] = key[j];
    leaf_start[incl[j] - 1] = (int)j;
  }
  if (j == ns - 1) leaf_start[incl[j]] = (int)ns;
}

// Flags over (level l in [2, L], leaf k): leaf k starts a box of level l.
__global__ void level_flags_kernel(const int* __restrict__ leaf_key, int nl, int L,
                                   int* __restrict__ flag) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t total = (int64_t)(L - 1) * nl;
  if (t >= total) return;
  const int l = 2 + (int)(t / nl), k = (int)(t % nl), sh = L - l;
  flag[t] = (k == 0 || (leaf_key[k] >> sh) != (leaf_key[k - 1] >> sh)) ? 1 : 0;
}

// Box table from the inclusive scan `id` of the level flags (box id of leaf
// k's ancestor at level l = id[(l-2) nl + k] - 1).
__global__ void box_info_kernel(const int* __restrict__ leaf_key, int nl, int L,
                                const int* __restrict__ flag, const int* __restrict__ id,
                                int* __restrict__ box_key, int* __restrict__ box_leaf,
                                unsigned char* __restrict__ box_level) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t total = (int64_t)(L - 1) * nl;
  if (t >= total || !flag[t]) return;
  const int l = 2 + (int)(t / nl), k = (int)(t % nl);
  const int b = id[t] - 1;
  box_key[b] = leaf_key[k] >> (L - l);
  box_leaf[b] = k;
  box_level[b] = (unsigned char)l;
}

__global__ void level_ends_kernel(const int* __restrict__ id, int nl, int L, int* __restrict__ off) {
  // off[l - 2] = first box id of level l; off[L - 1] = total
  const int t = threadIdx.x;
  if (t == 0) off[0] = 0;
  if (t < L - 1) off[t + 1] = id[(int64_t)t * nl + nl - 1];
}

struct Tabs {
  const double* tau;
  const double* lam;
  const double* TL;   // [j][k] = l_j(-1/2 + tau_k/2)
  const double* TR;   // [j][k] = l_j(+1/2 + tau_k/2)
  const double* Mre;  // [l][oi][i][j], oi: o = -3, -2, 2, 3
  const double* Mim;
};

// P2M: one warp per leaf; lanes take the leaf's sources in turn, each
// accumulating the n Lagrange-basis values of its sources (barycentric form,
// reciprocals by rcp_f64, within an ulp), and a fixed reduce-scatter adds
// the lanes: 16 shuffles leave the total of node i on lanes 2i and 2i + 1
// (deterministic).  The node tables sit in shared memory (broadcast reads).
// 128-thread blocks: at ~150 registers three fit per SM (one 256-thread
// block did), and the kernel is bound by how many leaf warps stay resident.
constexpr int P2M_NT = 128;

template <int N>
__global__ void __launch_bounds__(P2M_NT) p2m_kernel(const double* __restrict__ s,
                                                  const int* __restrict__ leaf_key,
                                                  const int* __restrict__ leaf_start, int nl,
                                                  FmmGeom g, Tabs tb, int64_t leaf_box0,
                                                  double* __restrict__ Wm) {
  __shared__ double stau[N], slam[N];
  if (threadIdx.x < N) {
    stau[threadIdx.x] = tb.tau[threadIdx.x];
    slam[threadIdx.x] = tb.lam[threadIdx.x];
  }
  __syncthreads();
  const int64_t k = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (k >= nl) return;  // whole warps leave together
  double v[16];
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = 0.0;
  const double h = g.W / (double)(1LL << g.L);
  const double c = g.a + ((double)leaf_key[k] + 0.5) * h, hh = 0.5 * h;
  for (int j = leaf_start[k] + lane; j < leaf_start[k + 1]; j += 32) {
    const double x = (s[j] - c) / hh;
    double q[N], den = 0.0;
    int hit = -1;
#pragma unroll
    for (int i = 0; i < N; ++i) {
      const double d = x - stau[i];
      if (d == 0.0) hit = i;
      q[i] = slam[i] * rcp_f64(d);  // |d| >= one ulp of x unless it is 0
      den += q[i];
    }
    if (hit >= 0) {
#pragma unroll
      for (int i = 0; i < N; ++i)
        if (i == hit) v[i] += 1.0;
    } else {
      const double r = rcp_f64(den);
#pragma unroll
      for (int i = 0; i < N; ++i) v[i] = fma(q[i], r, v[i]);
    }
  }
  // reduce-scatter: at the step of width m (8, 4, 2, 1) and lane bit b, a
  // lane keeps the upper or lower m of its 2m partial totals and adds the
  // partner's copy of them
#pragma unroll
  for (int m = 8, o = 16; m >= 1; m >>= 1, o >>= 1) {
    const bool up = (lane & o) != 0;
#pragma unroll
    for (int i = 0; i < m; ++i) {
      const double send = up ? v[i] : v[m + i];
      const double keep = up ? v[m + i] : v[i];
      v[i] = keep + __shfl_xor_sync(0xffffffffu, send, o);
    }
  }
  v[0] += __shfl_xor_sync(0xffffffffu, v[0], 1);
  const int node = lane >> 1;
  if (!(lane & 1) && node < N) Wm[(leaf_box0 + k) * FMM_MAXN + node] = v[0];
}

// The expansion kernels below give each box a half-warp (lane i of the half
// = node i, n <= 16): warp w of a level takes boxes 2w and 2w + 1, warps
// striding over the level; the loop exit is uniform across the warp.

// Shared-memory tables, rows padded to an odd number of doubles so that lane
// i's row starts on its own bank pair.
constexpr int FMM_RS = FMM_MAXN + 1;

__device__ __forceinline__ void load_side_tables(double* sT, const Tabs& tb, int n) {
  const int rs = n | 1;  // [side][j][k]
  for (int t = threadIdx.x; t < 2 * n * n; t += blockDim.x) {
    const int side = t / (n * n), r = (t / n) % n, col = t % n;
    sT[(side * n + r) * rs + col] = (side ? tb.TR : tb.TL)[r * n + col];
  }
}

__device__ __forceinline__ void load_m2l_tables(double* sre, double* sim, const Tabs& tb, int l,
                                                int n) {
  const int nn4 = 4 * n * n, rs = n | 1;  // [oi][i][j]
  const double* mr = tb.Mre + (int64_t)l * nn4;
  const double* mi = tb.Mim + (int64_t)l * nn4;
  for (int t = threadIdx.x; t < nn4; t += blockDim.x) {
    const int row = t / n, col = t % n;
    sre[row * rs + col] = mr[t];
    sim[row * rs + col] = mi[t];
  }
}

// Per-box bodies, half a warp per box (lane = node).  Every lane of the warp
// calls them together (they shuffle); `live` masks the arithmetic.  The
// expansion arrays are plain pointers: the fused top-of-tree kernel reads
// what it wrote at the previous level.

// M2M: parent b (level l) gets T_side W_child from each child (level l+1,
// boxes before c1).
__device__ __forceinline__ double m2m_box(int64_t b, bool live, int64_t c1, const int* box_key,
                                          const int* box_leaf, const int* id, int nl, int l,
                                          int n, const double* sT, const double* Wm, int lane) {
  const int rs = n | 1;
  double acc = 0.0;
  const int64_t first = live ? id[(int64_t)(l + 1 - 2) * nl + box_leaf[b]] - 1 : 0;
  const int kb = live ? box_key[b] : 0;
  for (int q = 0; q < 2; ++q) {
    const int64_t ch = first + q;
    const bool has = live && ch < c1 && (box_key[ch] >> 1) == kb;
    const double* T = sT + ((has && (box_key[ch] & 1)) ? n * rs : 0);
    const double wc = (has && lane < n) ? Wm[ch * FMM_MAXN + lane] : 0.0;
    for (int kk = 0; kk < n; ++kk) {
      const double v = __shfl_sync(0xffffffffu, wc, kk, 16);
      if (has && lane < n) acc = fma(T[lane * rs + kk], v, acc);
    }
  }
  return acc;
}

// M2L: box b of level l (boxes [b0, b1)) from its three interaction
// partners, with the level's four matrices in shared memory.
__device__ __forceinline__ void m2l_box(int64_t b, bool live, int64_t b0, int64_t b1,
                                        const int* box_key, int n, const double* sre,
                                        const double* sim, const double* Wm, int lane,
                                        double& re, double& im) {
  const int rs = n | 1;
  const int kb = live ? box_key[b] : 0;
  const int odd = kb & 1;
  re = 0.0;
  im = 0.0;
  for (int q = 0; q < 3; ++q) {
    // even kb: sources at kb-2, kb+2, kb+3 (o = 2, -2, -3); odd: kb-3, kb-2, kb+2
    const int o = odd ? (q == 0 ? 3 : (q == 1 ? 2 : -2)) : (q == 0 ? 2 : (q == 1 ? -2 : -3));
    const int ka = kb - o;
    // keys of a level are sorted and distinct: a box at key offset |o| <= 3
    // sits within three positions of b
    int64_t a = -1;
    if (live && ka >= 0) {
#pragma unroll
      for (int t = 1; t <= 3; ++t) {
        const int64_t f = o > 0 ? b - t : b + t;
        if (a < 0 && f >= b0 && f < b1 && box_key[f] == ka) a = f;
      }
    }
    const int oi = o == -3 ? 0 : (o == -2 ? 1 : (o == 2 ? 2 : 3));
    const double* rr = sre + (oi * n + lane) * rs;
    const double* ri = sim + (oi * n + lane) * rs;
    const double wa = (a >= 0 && lane < n) ? Wm[a * FMM_MAXN + lane] : 0.0;
    for (int j = 0; j < n; ++j) {
      const double v = __shfl_sync(0xffffffffu, wa, j, 16);
      if (a >= 0 && lane < n) {
        re = fma(rr[j], v, re);
        im = fma(ri[j], v, im);
      }
    }
  }
}

// L2L: child c (level l + 1) gets T_side^T L_parent (parent at level l).
__device__ __forceinline__ void l2l_box(int64_t c, bool live, const int* box_key,
                                        const int* box_leaf, const int* id, int nl, int l, int n,
                                        const double* sT, const double* Lre, const double* Lim,
                                        int lane, double& re, double& im) {
  const int rs = n | 1;
  const int64_t par = live ? id[(int64_t)(l - 2) * nl + box_leaf[c]] - 1 : 0;
  const double* T = sT + ((live && (box_key[c] & 1)) ? n * rs : 0);
  const double pr = (live && lane < n) ? Lre[par * FMM_MAXN + lane] : 0.0;
  const double pi = (live && lane < n) ? Lim[par * FMM_MAXN + lane] : 0.0;
  re = 0.0;
  im = 0.0;
  for (int i = 0; i < n; ++i) {
    const double vr = __shfl_sync(0xffffffffu, pr, i, 16);
    const double vi = __shfl_sync(0xffffffffu, pi, i, 16);
    if (live && lane < n) {
      const double t = T[i * rs + lane];
      re = fma(t, vr, re);
      im = fma(t, vi, im);
    }
  }
}

// M2M for level l: parent box b gets T_side W_child from each child.
__global__ void __launch_bounds__(256) m2m_kernel(int64_t b0, int64_t b1, int64_t c1,
                                                  const int* __restrict__ box_key,
                                                  const int* __restrict__ box_leaf,
                                                  const int* __restrict__ id, int nl, int l, int n,
                                                  Tabs tb, double* __restrict__ Wm) {
  __shared__ double sT[2 * FMM_MAXN * FMM_RS];
  load_side_tables(sT, tb, n);
  __syncthreads();
  const int lane = threadIdx.x & 15;
  const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
  for (int64_t w = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;; w += warps) {
    if (b0 + 2 * w >= b1) break;
    const int64_t b = b0 + 2 * w + ((threadIdx.x >> 4) & 1);
    const bool live = b < b1;
    const double acc = m2m_box(b, live, c1, box_key, box_leaf, id, nl, l, n, sT, Wm, lane);
    if (live && lane < n) Wm[b * FMM_MAXN + lane] = acc;
  }
}

// Downward pass of level l (boxes [b0, b1)), M2L and L2L in one launch:
// L_b = M2L(partners) + T^T L_parent (the parent's L is complete: levels run
// in order; level 2 has no parent term).  A CTA takes tiles of DT_BOXES
// consecutive boxes; their partners lie within 3 positions, so the tile's
// multipole window and keys are staged in shared memory with coalesced
// loads.  Thread (box, g) computes nodes g, g+4, g+8, g+12 of its box: 8
// independent FP64 accumulators.  The kernel is bound by shared-memory
// wavefronts, so the M2L matrices are stored as {re, im} pairs (one 16-byte
// load feeds two FMAs) and the window is read two nodes at a time.  Strides
// (in 16-byte units: rows 17, offset blocks 276 = 4 mod 8; window rows 18
// doubles; side blocks 276 doubles) put the 8 distinct addresses a warp
// reads at once -- 4 node rows x the 2 offsets of even and odd boxes, or x
// the 2 sides -- in 8 different bank groups.
constexpr int DT_BOXES = 64, DT_NT = 256, DT_WIN = DT_BOXES + 6;
constexpr int DT_RS = FMM_MAXN + 1;        // matrix row stride (entries)
constexpr int DT_MS = FMM_MAXN * DT_RS + 4;  // offset / side block stride
constexpr int DT_WS = FMM_MAXN + 2;        // window row stride (doubles)

__global__ void __launch_bounds__(DT_NT, 2) down_kernel(int64_t b0, int64_t b1, int l,
                                                     const int* __restrict__ box_key,
                                                     const int* __restrict__ box_leaf,
                                                     const int* __restrict__ id, int nl, int n,
                                                     Tabs tb, const double* __restrict__ Wm,
                                                     double* __restrict__ Lre,
                                                     double* __restrict__ Lim) {
  __shared__ double2 sM[4 * DT_MS];  // [oi][i][j] = {re, im}
  __shared__ double sT[2 * DT_MS];   // [side][i][v]
  __shared__ __align__(16) double sW[DT_WIN * DT_WS];
  __shared__ int skey[DT_WIN];
  {
    const int nn = n * n;
    const double* mr = tb.Mre + (int64_t)l * 4 * nn;
    const double* mi = tb.Mim + (int64_t)l * 4 * nn;
    for (int t = threadIdx.x; t < 4 * nn; t += DT_NT) {
      const int oi = t / nn, i = (t / n) % n, j = t % n;
      sM[oi * DT_MS + i * DT_RS + j] = make_double2(mr[t], mi[t]);
    }
    for (int t = threadIdx.x; t < 2 * nn; t += DT_NT) {
      const int side = t / nn, i = (t / n) % n, j = t % n;
      sT[side * DT_MS + i * DT_RS + j] = (side ? tb.TR : tb.TL)[i * n + j];
    }
  }
  const int bl = threadIdx.x >> 2, g = threadIdx.x & 3;
  const int ne = (n + 1) & ~1;  // nodes read in pairs; the window is zero above n
  for (int64_t tile = blockIdx.x; b0 + tile * DT_BOXES < b1; tile += gridDim.x) {
    const int64_t tb0 = b0 + tile * DT_BOXES;
    const int64_t r0 = tb0 - 3 > b0 ? tb0 - 3 : b0;
    const int64_t r1 = tb0 + DT_BOXES + 3 < b1 ? tb0 + DT_BOXES + 3 : b1;
    const int rows = (int)(r1 - r0);
    __syncthreads();  // the previous tile is done with sW / skey (and tables loaded)
    for (int q = threadIdx.x; q < rows * FMM_MAXN; q += DT_NT) {
      const int r = q / FMM_MAXN, j = q % FMM_MAXN;
      sW[r * DT_WS + j] = j < n ? Wm[(r0 + r) * FMM_MAXN + j] : 0.0;
    }
    for (int r = threadIdx.x; r < rows; r += DT_NT) skey[r] = box_key[r0 + r];
    __syncthreads();
    const int64_t b = tb0 + bl;
    if (b >= b1) continue;
    double re[4] = {0.0, 0.0, 0.0, 0.0}, im[4] = {0.0, 0.0, 0.0, 0.0};
    const int kb = skey[b - r0];
    const int odd = kb & 1;
    for (int q = 0; q < 3; ++q) {
      // even kb: sources at kb-2, kb+2, kb+3 (o = 2, -2, -3); odd: kb-3, kb-2, kb+2
      const int o = odd ? (q == 0 ? 3 : (q == 1 ? 2 : -2)) : (q == 0 ? 2 : (q == 1 ? -2 : -3));
      const int ka = kb - o;
      int ar = -1;  // the partner's row in the window
      if (ka >= 0) {
#pragma unroll
        for (int t = 1; t <= 3; ++t) {
          const int64_t f = o > 0 ? b - t : b + t;
          if (ar < 0 && f >= b0 && f < b1 && skey[f - r0] == ka) ar = (int)(f - r0);
        }
      }
      if (ar < 0) continue;
      const int oi = o == -3 ? 0 : (o == -2 ? 1 : (o == 2 ? 2 : 3));
      const double2* w2 = reinterpret_cast<const double2*>(sW + ar * DT_WS);
      const double2* m = sM + oi * DT_MS + g * DT_RS;
      for (int j = 0; j < ne; j += 2) {
        const double2 v = w2[j >> 1];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          const double2 c0 = m[4 * u * DT_RS + j], c1 = m[4 * u * DT_RS + j + 1];
          re[u] = fma(c1.x, v.y, fma(c0.x, v.x, re[u]));
          im[u] = fma(c1.y, v.y, fma(c0.y, v.x, im[u]));
        }
      }
    }
    if (l > 2) {
      // L2L: child node v gets sum_i T_side[i][v] L_parent[i]
      const int64_t par = id[(int64_t)(l - 1 - 2) * nl + box_leaf[b]] - 1;
      const double* T = sT + (kb & 1) * DT_MS + g;
      const double* pr = Lre + par * FMM_MAXN;
      const double* pi = Lim + par * FMM_MAXN;
      for (int i = 0; i < n; ++i) {
        const double vr = pr[i], vi = pi[i];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          const double t = T[i * DT_RS + 4 * u];
          re[u] = fma(t, vr, re[u]);
          im[u] = fma(t, vi, im[u]);
        }
      }
    }
#pragma unroll
    for (int u = 0; u < 4; ++u)
      if (g + 4 * u < n) {
        Lre[b * FMM_MAXN + g + 4 * u] = re[u];
        Lim[b * FMM_MAXN + g + 4 * u] = im[u];
      }
  }
}

// The top of the tree in one CTA: levels 2..K hold at most FMM_TOP_BOXES
// boxes each, too few to fill the GPU, so one launch per level would cost
// more than its work.  Given W at level K, the CTA runs M2M up to level 2,
// then M2L + L2L down to level K, with a block barrier between levels (the
// writes of one level are visible to every thread of the CTA at the next).
// With tensor-core M2L the levels up to K still take this FP64 M2L.
constexpr int FMM_TOP_BOXES = 128;
constexpr int FMM_TOP_NT = 1024;

struct LevelOffs {
  int64_t o[FMM_LMAX];  // o[l - 2] = first box of level l, o[l - 1] = one past it
};

__global__ void __launch_bounds__(FMM_TOP_NT) top_kernel(LevelOffs off, int K,
                                                         const int* __restrict__ box_key,
                                                         const int* __restrict__ box_leaf,
                                                         const int* __restrict__ id, int nl,
                                                         int n, Tabs tb, double* Wm, double* Lre,
                                                         double* Lim) {
  __shared__ double sre[4 * FMM_MAXN * FMM_RS], sim[4 * FMM_MAXN * FMM_RS];
  __shared__ double sT[2 * FMM_MAXN * FMM_RS];
  load_side_tables(sT, tb, n);
  __syncthreads();
  const int lane = threadIdx.x & 15, half = (threadIdx.x >> 4) & 1;
  const int warp = threadIdx.x >> 5, nw = FMM_TOP_NT / 32;
  for (int l = K - 1; l >= 2; --l) {
    const int64_t b0 = off.o[l - 2], b1 = off.o[l - 1], c1 = off.o[l];
    for (int64_t w = warp; b0 + 2 * w < b1; w += nw) {
      const int64_t b = b0 + 2 * w + half;
      const bool live = b < b1;
      const double acc = m2m_box(b, live, c1, box_key, box_leaf, id, nl, l, n, sT, Wm, lane);
      if (live && lane < n) Wm[b * FMM_MAXN + lane] = acc;
    }
    __syncthreads();
  }
  for (int l = 2; l <= K; ++l) {
    load_m2l_tables(sre, sim, tb, l, n);
    __syncthreads();
    const int64_t b0 = off.o[l - 2], b1 = off.o[l - 1];
    for (int64_t w = warp; b0 + 2 * w < b1; w += nw) {
      const int64_t b = b0 + 2 * w + half;
      const bool live = b < b1;
      double re, im, pr = 0.0, pi = 0.0;
      m2l_box(b, live, b0, b1, box_key, n, sre, sim, Wm, lane, re, im);
      if (l > 2)
        l2l_box(b, live, box_key, box_leaf, id, nl, l - 1, n, sT, Lre, Lim, lane, pr, pi);
      if (live && lane < n) {
        Lre[b * FMM_MAXN + lane] = re + pr;
        Lim[b * FMM_MAXN + lane] = im + pi;
      }
    }
    __syncthreads();  // this level's L before the next level's L2L; tables reloaded
  }
}

// ------------------------------------------------ tensor-core M2L --
// The M2L of one level as a GEMM on the 5th-generation tensor cores: a CTA
// of 128 threads owns 128 target boxes (one per thread) and computes
//   D[b][c] = sum_k A[b][k] B[c][k],   k = offset slot * 16 + source node j,
// A[b][.] = the multipoles of b's interaction partners (zero where a slot is
// empty), B[c][.] = row c mod 16 of the four M2L matrices (real part for
// c < 16, imaginary part above), i.e. M = 128, N = 32, K = 64, as
// tcgen05.mma kind::tf32 with FP32 accumulation in tensor memory, each
// product split as hi*hi + hi*lo + lo*hi (TF32 x3).  Operands sit in shared
// memory in the K-major no-swizzle layout: 16-byte chunks (4 values) of
// chunk column kc and row r at chunk index kc*R + r (R = rows of the tile),
// so 8-row groups are 128 bytes apart and K chunks R*16 bytes apart.
constexpr int TC_M = 128, TC_N = 32, TC_K = 64;
constexpr uint32_t TC_IDESC = (1u << 4)           // D: F32
                              | (2u << 7)         // A: TF32
                              | (2u << 10)        // B: TF32
                              | ((uint32_t)(TC_N >> 3) << 17)
                              | ((uint32_t)(TC_M >> 4) << 24);  // K-major A and B
// A tile's interaction partners lie within 3 boxes of it: the multipoles of
// that window (TC_WIN rows, split into TF32 hi/lo, rows padded to TC_WS
// floats so that row-strided float4 reads do not conflict) and its keys are
// staged with coalesced loads before A is assembled in shared memory.
constexpr int TC_WIN = TC_M + 6, TC_WS = 20;
constexpr int TC_OS = FMM_MAXN + 1;  // output staging row stride (doubles)
constexpr int TC_SMEM = 2 * TC_M * TC_K * 4 + 2 * TC_N * TC_K * 4 + 2 * TC_WIN * TC_WS * 4 +
                        TC_WIN * 4 + 2 * FMM_MAXN * FMM_RS * 8 + TC_M * 4 + 256;
static_assert(2 * TC_M * TC_OS * 8 <= 2 * TC_M * TC_K * 4, "output staging reuses A");

__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);  // version 1, no swizzle
}

__device__ __forceinline__ void tf32_split(double x, float& hi, float& lo) {
  const float f = (float)x;
  hi = __uint_as_float(__float_as_uint(f) & 0xFFFFE000u);
  lo = f - hi;
}

__device__ __forceinline__ void umma_tf32(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc,
                                          uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(
          tmem_d),
      "l"(adesc), "l"(bdesc), "r"(TC_IDESC), "r"(accumulate), "r"(0u), "r"(0u), "r"(0u), "r"(0u)
      : "memory");
}

//
// The level's L2L rides in the epilogue: each box adds T_side^T L_parent
// (summed from zero in node order, then added, as l2l_box), so a level takes
// one launch; the parent level is complete (levels run in order).
__global__ void __launch_bounds__(TC_M) m2l_tc_kernel(int64_t b0, int64_t b1, int l,
                                                      const int* __restrict__ box_key,
                                                      const int* __restrict__ box_leaf,
                                                      const int* __restrict__ id, int nl, int n,
                                                      Tabs tb, const double* __restrict__ Wm,
                                                      double* __restrict__ Lre,
                                                      double* __restrict__ Lim,
                                                      int* __restrict__ err) {
  extern __shared__ __align__(1024) unsigned char tsm[];
  float4* Ahi = reinterpret_cast<float4*>(tsm);
  float4* Alo = Ahi + TC_M * TC_K / 4;
  float4* Bhi = Alo + TC_M * TC_K / 4;
  float4* Blo = Bhi + TC_N * TC_K / 4;
  float* Whi = reinterpret_cast<float*>(Blo + TC_N * TC_K / 4);
  float* Wlo = Whi + TC_WIN * TC_WS;
  int* skey = reinterpret_cast<int*>(Wlo + TC_WIN * TC_WS);
  double* sT = reinterpret_cast<double*>(skey + TC_WIN + (TC_WIN & 1));  // [side][i][v]
  int* spar = reinterpret_cast<int*>(sT + 2 * FMM_MAXN * FMM_RS);  // 2 parent + side per row
  uint64_t* bar = reinterpret_cast<uint64_t*>(spar + TC_M);
  uint32_t* taddr_slot = reinterpret_cast<uint32_t*>(bar + 1);
  double* Ore = reinterpret_cast<double*>(tsm);  // after the MMAs: [row][TC_OS]
  double* Oim = Ore + TC_M * TC_OS;
  const int t = threadIdx.x, warp = t >> 5;

  // TMEM: 32 columns (the F32 accumulator of N = 32), held for all tiles
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(taddr_slot)),
                 "r"(32u)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (t == 0) {
    mbar_init(bar, 1);
    fence_mbar_init();
  }
  // B (the level's matrices), built once per CTA: row c, chunk kc
  const double* mr = tb.Mre + (int64_t)l * 4 * n * n;
  const double* mi = tb.Mim + (int64_t)l * 4 * n * n;
  for (int q = t; q < TC_N * (TC_K / 4); q += TC_M) {
    const int c = q / (TC_K / 4), kc = q % (TC_K / 4);
    const int i = c & 15, oi = kc / 4;
    const double* src = (c < 16 ? mr : mi) + ((int64_t)oi * n + i) * n;
    float h[4], lo[4];
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      const int j = (kc % 4) * 4 + e;
      const double v = (i < n && j < n) ? src[j] : 0.0;
      tf32_split(v, h[e], lo[e]);
    }
    Bhi[kc * TC_N + c] = make_float4(h[0], h[1], h[2], h[3]);
    Blo[kc * TC_N + c] = make_float4(lo[0], lo[1], lo[2], lo[3]);
  }
  load_side_tables(sT, tb, n);
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *taddr_slot;
  bool ok = true;
  uint32_t phase = 0;

  for (int64_t tile = blockIdx.x; b0 + tile * TC_M < b1 && ok; tile += gridDim.x) {
    const int64_t tb0 = b0 + tile * TC_M;
    const int64_t r0 = tb0 - 3 > b0 ? tb0 - 3 : b0;
    const int64_t r1 = tb0 + TC_M + 3 < b1 ? tb0 + TC_M + 3 : b1;
    const int rows = (int)(r1 - r0);
    for (int q = t; q < rows * FMM_MAXN; q += TC_M) {
      const int r = q / FMM_MAXN, j = q % FMM_MAXN;
      const double w = j < n ? Wm[(r0 + r) * FMM_MAXN + j] : 0.0;
      float h, lo;
      tf32_split(w, h, lo);
      Whi[r * TC_WS + j] = h;
      Wlo[r * TC_WS + j] = lo;
    }
    for (int r = t; r < rows; r += TC_M) skey[r] = box_key[r0 + r];
    __syncthreads();
    // A: row t = target box b, slot oi = offset o in {-3, -2, 2, 3}
    const int64_t b = tb0 + t;
    const bool live = b < b1;
    const int kb = live ? skey[b - r0] : 0;
    spar[t] = live ? 2 * (id[(int64_t)(l - 1 - 2) * nl + box_leaf[b]] - 1) + (kb & 1) : 0;
    for (int oi = 0; oi < 4; ++oi) {
      const int o = oi == 0 ? -3 : (oi == 1 ? -2 : (oi == 2 ? 2 : 3));
      // even kb: partners at o = 2, -2, -3; odd kb: o = 3, 2, -2
      const bool inlist = (kb & 1) ? (o != -3) : (o != 3);
      const int ka = kb - o;
      int ar = -1;  // the partner's row in the window
      if (live && inlist && ka >= 0) {
#pragma unroll
        for (int q = 1; q <= 3; ++q) {
          const int64_t f = o > 0 ? b - q : b + q;
          if (ar < 0 && f >= b0 && f < b1 && skey[f - r0] == ka) ar = (int)(f - r0);
        }
      }
      const float4 z = make_float4(0.f, 0.f, 0.f, 0.f);
      const float4* wh = reinterpret_cast<const float4*>(Whi + (ar < 0 ? 0 : ar) * TC_WS);
      const float4* wl = reinterpret_cast<const float4*>(Wlo + (ar < 0 ? 0 : ar) * TC_WS);
#pragma unroll
      for (int c4 = 0; c4 < 4; ++c4) {
        const int kc = oi * 4 + c4;
        Ahi[kc * TC_M + t] = ar < 0 ? z : wh[c4];
        Alo[kc * TC_M + t] = ar < 0 ? z : wl[c4];
      }
    }
    fence_proxy_async();  // generic-proxy writes -> tensor-core (async proxy) reads
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (t == 0) {
      const uint32_t a_hi = smem_u32(Ahi), a_lo = smem_u32(Alo);
      const uint32_t b_hi = smem_u32(Bhi), b_lo = smem_u32(Blo);
      constexpr uint32_t ALBO = TC_M * 16, BLBO = TC_N * 16, SBO = 128;
      for (int st = 0; st < TC_K / 8; ++st) {  // K = 8 per instruction = 2 chunks
        const uint32_t ao = st * 2 * TC_M * 16, bo = st * 2 * TC_N * 16;
        umma_tf32(tmem, umma_desc(a_hi + ao, ALBO, SBO), umma_desc(b_hi + bo, BLBO, SBO),
                  st > 0 ? 1u : 0u);
        umma_tf32(tmem, umma_desc(a_hi + ao, ALBO, SBO), umma_desc(b_lo + bo, BLBO, SBO), 1u);
        umma_tf32(tmem, umma_desc(a_lo + ao, ALBO, SBO), umma_desc(b_hi + bo, BLBO, SBO), 1u);
      }
      asm volatile(
          "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
              smem_u32(bar))
          : "memory");
    }
    const bool done = mbar_wait(bar, phase);
    if (!done) {
      atomicExch(err, DEV_ERR_TIMEOUT);
      mbar_wait(bar, phase, 200000000LL);  // the MMAs may still be in flight
    }
    phase ^= 1u;
    ok = __syncthreads_and(done) != 0;  // tcgen05.ld below is warp-collective
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (ok) {
      uint32_t v[32];
      asm volatile(
          "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, "
          "%11, %12, %13, %14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, "
          "%28, %29, %30, %31}, [%32];"
          : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]),
            "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]),
            "=r"(v[13]), "=r"(v[14]), "=r"(v[15]), "=r"(v[16]), "=r"(v[17]), "=r"(v[18]),
            "=r"(v[19]), "=r"(v[20]), "=r"(v[21]), "=r"(v[22]), "=r"(v[23]), "=r"(v[24]),
            "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]), "=r"(v[30]),
            "=r"(v[31])
          : "r"(tmem + ((uint32_t)(warp * 32) << 16))
          : "memory");
      asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
      // A is no longer read (the MMAs completed): stage the rows there, each
      // plus its L2L term (this thread's box: its parent's row in registers)
      double lpr[FMM_MAXN], lpi[FMM_MAXN];
      const int64_t par = spar[t] >> 1;
      const double* T = sT + (spar[t] & 1) * n * (n | 1);
#pragma unroll
      for (int i = 0; i < FMM_MAXN; ++i) {
        lpr[i] = (live && i < n) ? Lre[par * FMM_MAXN + i] : 0.0;
        lpi[i] = (live && i < n) ? Lim[par * FMM_MAXN + i] : 0.0;
      }
#pragma unroll
      for (int i = 0; i < 16; ++i) {
        double are = 0.0, aim = 0.0;
#pragma unroll
        for (int k = 0; k < FMM_MAXN; ++k)
          if (k < n) {
            const double tk = T[k * (n | 1) + i];
            are = fma(tk, lpr[k], are);
            aim = fma(tk, lpi[k], aim);
          }
        Ore[t * TC_OS + i] = (double)__uint_as_float(v[i]) + are;
        Oim[t * TC_OS + i] = (double)__uint_as_float(v[16 + i]) + aim;
      }
    }
    __syncthreads();
    if (ok) {
      const int live_rows = (int)(b1 - tb0 < TC_M ? b1 - tb0 : TC_M);
      for (int q = t; q < live_rows * FMM_MAXN; q += TC_M) {
        const int r = q / FMM_MAXN, i = q % FMM_MAXN;
        if (i < n) {
          Lre[tb0 * FMM_MAXN + q] = Ore[r * TC_OS + i];
          Lim[tb0 * FMM_MAXN + q] = Oim[r * TC_OS + i];
        }
      }
    }
    // the next tile rewrites A and the accumulator only after every thread
    // has read its row; a timeout anywhere ends the loop for the whole CTA
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    ok = __syncthreads_and(ok) != 0;
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(32u)
                 : "memory");
  }
}

// L2P + near field: one thread per (sorted) target; reciprocals by rcp_f64
// (within an ulp).
__global__ void l2p_near_kernel(const double* __restrict__ s, int64_t ns,
                                const int* __restrict__ leaf_of, const int* __restrict__ leaf_key,
                                const int* __restrict__ leaf_start, int nl, FmmGeom g, Tabs tb,
                                int64_t leaf_box0, const double* __restrict__ Lre,
                                const double* __restrict__ Lim, const int* __restrict__ perm,
                                double scale, double* __restrict__ out_re,
                                double* __restrict__ out_im) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= ns) return;
  const int n = g.n;
  const double x = s[t];
  const int k = leaf_of[t] - 1, key = leaf_key[k];  // leaf_of: inclusive run count
  const double h = g.W / (double)(1LL << g.L);
  const double c = g.a + ((double)key + 0.5) * h;
  const double xp = (x - c) / (0.5 * h);
  // barycentric interpolation of the local expansion
  double num_r = 0.0, num_i = 0.0, den = 0.0;
  int hit = -1;
  const double* lr = Lre + (leaf_box0 + k) * FMM_MAXN;
  const double* li = Lim + (leaf_box0 + k) * FMM_MAXN;
  for (int i = 0; i < n; ++i) {
    const double d = xp - tb.tau[i];
    if (d == 0.0) {
      hit = i;
      break;
    }
    const double q = tb.lam[i] * rcp_f64(d);  // |d| >= one ulp of xp
    num_r = fma(q, lr[i], num_r);
    num_i = fma(q, li[i], num_i);
    den += q;
  }
  double re, im;
  if (hit >= 0) {
    re = lr[hit];
    im = li[hit];
  } else {
    const double r = rcp_f64(den);
    re = num_r * r;
    im = num_i * r;
  }
  // near field: this leaf and the adjacent ones
  const int ka = (k > 0 && leaf_key[k - 1] == key - 1) ? k - 1 : k;
  const int kz = (k + 1 < nl && leaf_key[k + 1] == key + 1) ? k + 1 : k;
  const double eta = g.eta, eta2 = eta * eta;
  double nr = 0.0, ni = 0.0;
  for (int j = leaf_start[ka]; j < leaf_start[kz + 1]; ++j) {
    const double d = x - s[j];
    const double inv = rcp_f64(fma(d, d, eta2));
    nr = fma(d, inv, nr);
    ni += inv;
  }
  re += nr;
  im += eta * ni;
  const int64_t o = perm ? perm[t] : t;
  out_re[o] = re * scale;
  out_im[o] = im * scale;
}

unsigned blocks(int64_t n, int t) { return (unsigned)((n + t - 1) / t); }

// CTAs of 8 warps for nb boxes at two boxes per warp, at most 4 per SM (the
// kernels stride).
unsigned half_grid(int64_t nb) {
  const int64_t need = (nb + 15) / 16;
  return (unsigned)std::max<int64_t>(1, std::min<int64_t>(need, 148 * 4));
}

// Host tables: first-kind Chebyshev points, barycentric weights and the
// M2M / L2L matrices (double precision, computed here once per call; the
// M2L matrices are made on the device by m2l_tables_kernel).
void host_tables(int n, std::vector<double>& tab) {
  std::vector<double> tau(n), lam(n);
  for (int j = 0; j < n; ++j) {
    const double th = M_PI * (2.0 * j + 1.0) / (2.0 * n);
    tau[j] = std::cos(th);
    lam[j] = ((j & 1) ? -1.0 : 1.0) * std::sin(th);
  }
  auto lag = [&](double x, int j) {
    for (int k = 0; k < n; ++k)
      if (x == tau[k]) return k == j ? 1.0 : 0.0;
    double den = 0.0;
    for (int k = 0; k < n; ++k) den += lam[k] / (x - tau[k]);
    return (lam[j] / (x - tau[j])) / den;
  };
  const size_t nn = (size_t)n * n;
  tab.assign(2 * n + 2 * nn, 0.0);
  double* T = tab.data();
  std::copy(tau.begin(), tau.end(), T);
  std::copy(lam.begin(), lam.end(), T + n);
  double* TL = T + 2 * n;
  double* TR = TL + nn;
  for (int j = 0; j < n; ++j)
    for (int k = 0; k < n; ++k) {
      TL[j * n + k] = lag(-0.5 + 0.5 * tau[k], j);
      TR[j * n + k] = lag(0.5 + 0.5 * tau[k], j);
    }
}

// The M2L matrices of levels 2..L on the device (the host uploads only the
// node tables): Mre + i Mim [l][oi][i][j] = 1/(d - i eta) = (d + i eta) /
// (d^2 + eta^2), d = (h_l / 2)(2 o + tau_i - tau_j), h_l = W / 2^l.
__global__ void m2l_tables_kernel(const double* __restrict__ tau, int n, int L, double W,
                                  double eta, double* __restrict__ Mre,
                                  double* __restrict__ Mim) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t per = 4LL * n * n;
  if (t >= (int64_t)(L - 1) * per) return;
  const int l = 2 + (int)(t / per), r = (int)(t % per);
  const int oi = r / (n * n), i = (r / n) % n, j = r % n;
  const int o = oi == 0 ? -3 : (oi == 1 ? -2 : (oi == 2 ? 2 : 3));
  const double hh = 0.5 * W / (double)(1LL << l);
  const double d = hh * (2.0 * o + tau[i] - tau[j]);
  const double den = d * d + eta * eta;
  const int64_t q = (((int64_t)l * 4 + oi) * n + i) * n + j;
  Mre[q] = d / den;
  Mim[q] = eta / den;
}

}  // namespace

shrk_status fmm_all(const double* d_ev, int64_t p, double eta, int n, int m2l_tc, double* d_re,
                    double* d_im, cudaStream_t s) {
  if (p <= 0) return SHRK_OK;
  const double* ds = nullptr;
  const int* perm = nullptr;
  double ends[2];
  SHRK_TRY(sorted_sources_perm(d_ev, p, &ds, &perm, s, &ends[0], &ends[1]));
  FmmGeom g;
  g.a = ends[0];
  g.W = (ends[1] - ends[0]) * (1.0 + 0x1p-20);
  if (!(g.W > 0.0) || !std::isfinite(g.W)) g.W = 1.0;
  g.n = n;
  g.eta = eta;
  // leaves: keys at the leaf level (the coarsest with at most FMM_OCC
  // sources per box, found by the probe) and their runs; one read-back for
  // the probe mask and the leaf count
  void* kw = nullptr;
  SHRK_TRY(scratch_get(SLOT_KEYS, sizeof(int) * 3 * (size_t)p + 256, &kw));
  int* key = (int*)kw;
  int* flag = key + p;
  int* incl = flag + p;  // becomes the leaf index per source
  size_t cub_bytes = 0;
  SHRK_CUDA(cub::DeviceScan::InclusiveSum(nullptr, cub_bytes, flag, incl, (int)p, s));
  void* lw = nullptr;
  SHRK_TRY(scratch_get(SLOT_LEAF, sizeof(int) * (2 * (size_t)p + 2), &lw));
  int* leaf_key = (int*)lw;
  int* leaf_start = leaf_key + p;
  void* tmp = nullptr;
  SHRK_TRY(scratch_get(SLOT_TMP, 4096 + cub_bytes, &tmp));
  unsigned* d_mask = (unsigned*)tmp;
  void* cubt = (char*)tmp + 4096;
  SHRK_CUDA(cudaMemsetAsync(d_mask, 0, sizeof(unsigned), s));
  {
    LaunchScope ls("fmm_build", s);
    level_probe_kernel<<<blocks(p, 256), 256, 0, s>>>(ds, p, g.a, g.W, d_mask);
    SHRK_CUDA(cudaGetLastError());
    leaf_flags_kernel<<<blocks(p, 256), 256, 0, s>>>(ds, p, g.a, g.W, d_mask, key, flag);
    SHRK_CUDA(cudaGetLastError());
    SHRK_CUDA(cub::DeviceScan::InclusiveSum(cubt, cub_bytes, flag, incl, (int)p, s));
    leaf_compact_kernel<<<blocks(p, 256), 256, 0, s>>>(key, flag, incl, p, leaf_key, leaf_start);
    SHRK_CUDA(cudaGetLastError());
    add_launches(4);  // five kernels, the scan's two included
  }
  unsigned mask = 0;
  int nl = 0;
  SHRK_CUDA(cudaMemcpyAsync(&mask, d_mask, sizeof(unsigned), cudaMemcpyDeviceToHost, s));
  SHRK_CUDA(cudaMemcpyAsync(&nl, incl + p - 1, sizeof(int), cudaMemcpyDeviceToHost, s));
  SHRK_CUDA(cudaStreamSynchronize(s));
  g.L = leaf_level(mask);
  const int L = g.L;
  // boxes of levels 2..L
  const int64_t nlev = (int64_t)(L - 1) * nl;
  void* vw = nullptr;
  SHRK_TRY(scratch_get(SLOT_LVL, sizeof(int) * (2 * (size_t)nlev + 64), &vw));
  int* lflag = (int*)vw;
  int* lid = lflag + nlev;
  int* d_off = lid + nlev;  // L entries
  size_t cub2 = 0;
  SHRK_CUDA(cub::DeviceScan::InclusiveSum(nullptr, cub2, lflag, lid, (int)nlev, s));
  SHRK_TRY(scratch_get(SLOT_TMP, 4096 + std::max(cub_bytes, cub2), &tmp));
  cubt = (char*)tmp + 4096;
  {
    LaunchScope ls("fmm_build", s);
    level_flags_kernel<<<blocks(nlev, 256), 256, 0, s>>>(leaf_key, nl, L, lflag);
    SHRK_CUDA(cudaGetLastError());
    SHRK_CUDA(cub::DeviceScan::InclusiveSum(cubt, cub2, lflag, lid, (int)nlev, s));
    level_ends_kernel<<<1, 32, 0, s>>>(lid, nl, L, d_off);
    SHRK_CUDA(cudaGetLastError());
  }
  std::vector<int> off(L);
  SHRK_CUDA(cudaMemcpyAsync(off.data(), d_off, sizeof(int) * L, cudaMemcpyDeviceToHost, s));
  SHRK_CUDA(cudaStreamSynchronize(s));
  const int64_t nbox = off[L - 1];
  // off[l - 2] = first box of level l, off[l - 1] = one past it
  void* bw = nullptr;
  SHRK_TRY(scratch_get(SLOT_BOX, (sizeof(int) * 2 + 1) * (size_t)nbox + 64, &bw));
  int* box_key = (int*)bw;
  int* box_leaf = box_key + nbox;
  unsigned char* box_level = (unsigned char*)(box_leaf + nbox);
  void* ew = nullptr;
  SHRK_TRY(scratch_get(SLOT_EXP, sizeof(double) * 3 * FMM_MAXN * (size_t)nbox, &ew));
  double* Wm = (double*)ew;
  double* Lre = Wm + FMM_MAXN * nbox;
  double* Lim = Lre + FMM_MAXN * nbox;
  std::vector<double> htab;
  host_tables(n, htab);
  const size_t nn = (size_t)n * n, nm = (size_t)(FMM_LMAX + 1) * 4 * nn;
  void* tw = nullptr;
  SHRK_TRY(scratch_get(SLOT_TAB, sizeof(double) * (htab.size() + 2 * nm), &tw));
  SHRK_CUDA(cudaMemcpyAsync(tw, htab.data(), sizeof(double) * htab.size(), cudaMemcpyHostToDevice,
                            s));
  Tabs tb;
  tb.tau = (const double*)tw;
  tb.lam = tb.tau + n;
  tb.TL = tb.lam + n;
  tb.TR = tb.TL + nn;
  tb.Mre = tb.TR + nn;
  tb.Mim = tb.Mre + nm;
  {
    LaunchScope ls("fmm_build", s);
    const int64_t nt = (int64_t)(L - 1) * 4 * n * n;
    m2l_tables_kernel<<<blocks(nt, 256), 256, 0, s>>>(tb.tau, n, L, g.W, eta,
                                                      const_cast<double*>(tb.Mre),
                                                      const_cast<double*>(tb.Mim));
    SHRK_CUDA(cudaGetLastError());
  }
  {
    LaunchScope ls("fmm_build", s);
    box_info_kernel<<<blocks(nlev, 256), 256, 0, s>>>(leaf_key, nl, L, lflag, lid, box_key,
                                                     box_leaf, box_level);
    SHRK_CUDA(cudaGetLastError());
  }
  const int64_t leaf_box0 = off[L - 2];
  {
    LaunchScope ls("fmm_p2m", s);
    const unsigned nb = blocks((int64_t)nl * 32, P2M_NT);
    switch (n) {
      case 4: p2m_kernel<4><<<nb, P2M_NT, 0, s>>>(ds, leaf_key, leaf_start, nl, g, tb, leaf_box0, Wm); break;
      case 5: p2m_kernel<5><<<nb, P2M_NT, 0, s>>>(ds, leaf_key, leaf_start, nl, g, tb, leaf_box0, Wm); break;
      case 6: p2m_kernel<6><<<nb, P2M_NT, 0, s>>>(ds, leaf_key, leaf_start, nl, g, tb, leaf_box0, Wm); break;
      case 7: p2m_kernel<7><<<nb, P2M_NT, 0, s>>>(ds, leaf_key, leaf_start, nl, g, tb, leaf_box0, Wm); break;
      case 8: p2m_kernel<8><<<nb, P2M_NT, 0, s>>>(ds, leaf_key, leaf_start, nl, g, tb, leaf_box0, Wm); break;
      case 9: p2m_kernel<9><<<nb, P2M_NT, 0, s>>>(ds, leaf_key, leaf_start, nl, g, tb, leaf_box0, Wm); break;
      case 10: p2m_kernel<10><<<nb, P2M_NT, 0, s>>>(ds, leaf_key, leaf_start, nl, g, tb, leaf_box0, Wm); break;
      case 11: p2m_kernel<11><<<nb, P2M_NT, 0, s>>>(ds, leaf_key, leaf_start, nl, g, tb, leaf_box0, Wm); break;
      case 12: p2m_kernel<12><<<nb, P2M_NT, 0, s>>>(ds, leaf_key, leaf_start, nl, g, tb, leaf_box0, Wm); break;
      case 13: p2m_kernel<13><<<nb, P2M_NT, 0, s>>>(ds, leaf_key, leaf_start, nl, g, tb, leaf_box0, Wm); break;
      case 14: p2m_kernel<14><<<nb, P2M_NT, 0, s>>>(ds, leaf_key, leaf_start, nl, g, tb, leaf_box0, Wm); break;
      case 15: p2m_kernel<15><<<nb, P2M_NT, 0, s>>>(ds, leaf_key, leaf_start, nl, g, tb, leaf_box0, Wm); break;
      default: p2m_kernel<16><<<nb, P2M_NT, 0, s>>>(ds, leaf_key, leaf_start, nl, g, tb, leaf_box0, Wm); break;
    }
    SHRK_CUDA(cudaGetLastError());
  }
  // K: the deepest level with at most FMM_TOP_BOXES boxes (box counts grow
  // with the level); levels 2..K run in the single-CTA top kernel.
  int K = 2;
  while (K < L && off[K - 1] - off[K - 2] <= FMM_TOP_BOXES) ++K;
  if (off[K - 1] - off[K - 2] > FMM_TOP_BOXES && K > 2) --K;
  if (L - 1 >= K) {
    LaunchScope ls("fmm_m2m", s);
    for (int l = L - 1; l >= K; --l) {
      const int64_t b0 = off[l - 2], b1 = off[l - 1], c1 = off[l];
      m2m_kernel<<<half_grid(b1 - b0), 256, 0, s>>>(b0, b1, c1, box_key, box_leaf, lid, nl, l, n,
                                                    tb, Wm);
      SHRK_CUDA(cudaGetLastError());
    }
    add_launches(L - 1 - K);
  }
  {
    LevelOffs lo{};
    for (int l = 2; l <= L; ++l) {
      lo.o[l - 2] = off[l - 2];
      lo.o[l - 1] = off[l - 1];
    }
    LaunchScope ls("fmm_top", s);
    top_kernel<<<1, FMM_TOP_NT, 0, s>>>(lo, K, box_key, box_leaf, lid, nl, n, tb, Wm, Lre, Lim);
    SHRK_CUDA(cudaGetLastError());
  }
  if (L > K && m2l_tc) {
    static std::atomic<bool> opted[64];
    int dev = 0;
    SHRK_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64 || !opted[dev].load()) {
      SHRK_CUDA(cudaFuncSetAttribute(m2l_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     TC_SMEM));
      if (dev >= 0 && dev < 64) opted[dev] = true;
    }
    LaunchScope ls("fmm_m2l_tc", s);
    for (int l = K + 1; l <= L; ++l) {
      const int64_t b0 = off[l - 2], b1 = off[l - 1];
      m2l_tc_kernel<<<(unsigned)std::min<int64_t>(blocks(b1 - b0, TC_M), 2 * 148), TC_M, TC_SMEM,
                      s>>>(b0, b1, l, box_key, box_leaf, lid, nl, n, tb, Wm, Lre, Lim,
                           device_error_word());
      SHRK_CUDA(cudaGetLastError());
    }
    add_launches(L - K - 1);
  } else if (L > K) {
    LaunchScope ls("fmm_down", s);
    for (int l = K + 1; l <= L; ++l) {
      const int64_t b0 = off[l - 2], b1 = off[l - 1];
      down_kernel<<<(unsigned)std::min<int64_t>(blocks(b1 - b0, DT_BOXES), 148 * 4), DT_NT, 0,
                    s>>>(b0, b1, l, box_key, box_leaf, lid, nl, n, tb, Wm, Lre, Lim);
      SHRK_CUDA(cudaGetLastError());
    }
    add_launches(L - K - 1);
  }
  {
    LaunchScope ls("fmm_l2p_near", s);
    l2p_near_kernel<<<blocks(p, 128), 128, 0, s>>>(ds, p, incl, leaf_key, leaf_start, nl, g, tb,
                                                   leaf_box0, Lre, Lim, perm, 1.0 / (double)p,
                                                   d_re, d_im);
    SHRK_CUDA(cudaGetLastError());
  }
  return SHRK_OK;
}

}  // namespace shrk
