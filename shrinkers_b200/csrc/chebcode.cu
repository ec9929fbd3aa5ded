// Chebyshev treecode (ChebCode presets) for the Stieltjes transform.
//
// Replaces src/stieltjes/chebcode.rs: the flat pre-order tree of
// FlatChebTree::build (242-572: midpoint split, barycentric leaf fill,
// reverse-order parent merge, f32 mirrors) is built on the GPU, breadth
// first, with every weight accumulated in the reference's order; the
// per-query evaluation (contribution_f64 607-711, contribution_fast32
// 722-828) runs one thread per query, queries in their given order
// (ascending queries keep a warp's traversals coherent).
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

#include <cub/device/device_scan.cuh>

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

// --------------------------------------------------- tree (device) --
// FlatChebTree::build (chebcode.rs:509-572) on the GPU, breadth first:
//   1. split: every node of a level with more than leaf_cap sources (and
//      depth < 48) splits at the midpoint of its value range (upper_bound of
//      mid, or the index midpoint when one side would be empty,
//      chebcode.rs:347-388); children take slots from an atomic counter and
//      are linked explicitly, so slot order does not matter;
//   2. subtree sizes and pre-order indices (node, left subtree, right
//      subtree -- the reference's flat layout): from a scan of the leaves'
//      start flags for large trees, level by level in one CTA for small ones;
//   3. flat arrays at the pre-order indices: bounds, acceptance radius,
//      Chebyshev nodes c + l cos(j pi/(n-1)) (set_node_positions 268-278);
//   4. P2M: a warp per leaf adds the barycentric rows of its sources in
//      index order (fill_leaves 401-460), 32 rows per step;
//   5. M2M: from the deepest level up, a warp per internal node merges the
//      left then the right child's node masses (merge_all_weights 474-506)
//      -- a launch per level for large trees, the P2M warps climbing from
//      their leaves for small ones.
// Every weight is accumulated in the reference's order with the same
// operations (IEEE division, fused fma where it uses mul_add), so the tree is
// identical to the sequential build.

struct ChebConsts {
  double sm1[MAX_N];  // cos(j pi / (n - 1)), computed on the host
  double lam[MAX_N];  // barycentric weights of the 2nd-kind nodes
  int n;
};


struct BuildArrays {
  int64_t* blo;  // BFS slot -> source index range [blo, bhi)
  int64_t* bhi;
  int32_t* lc;   // children (-1: leaf)
  int32_t* rc;
  int32_t* size;
  int32_t* pre;  // pre-order index
  int* counter;  // next free BFS slot
  int* levels;   // level L = BFS slots [levels[2L], levels[2L+1])
  int32_t* parent;  // parent slot (-1 at the root)
  int32_t* arrive;  // children finished per node (the climbing P2M/M2M)
  int32_t* dep;     // depth
  int32_t* rturn;   // right turns on the path from the root
  int32_t* leafpre; // [ns + 1]: leaf starts, then their exclusive prefix count
};

__device__ __forceinline__ void tree_split_node(const double* __restrict__ sorted, BuildArrays b,
                                                int i, int depth, int64_t leaf_cap) {
  const int64_t lo_idx = b.blo[i], hi_idx = b.bhi[i];
  if (hi_idx - lo_idx <= leaf_cap || depth >= MAX_TREE_DEPTH) {
    b.lc[i] = b.rc[i] = -1;
    return;
  }
  const double lo = sorted[lo_idx], hi = sorted[hi_idx - 1];
  const double mid = lo + 0.5 * (hi - lo);
  int64_t a = lo_idx, e = hi_idx;  // upper_bound: first element > mid
  while (a < e) {
    const int64_t m = (a + e) >> 1;
    if (mid < sorted[m]) e = m;
    else a = m + 1;
  }
  int64_t split = a;
  if (split == lo_idx || split == hi_idx) split = (lo_idx + hi_idx) / 2;
  const int slot = atomicAdd(b.counter, 2);
  b.blo[slot] = lo_idx;
  b.bhi[slot] = split;
  b.blo[slot + 1] = split;
  b.bhi[slot + 1] = hi_idx;
  b.lc[i] = slot;
  b.rc[i] = slot + 1;
  b.parent[slot] = b.parent[slot + 1] = i;
  b.dep[slot] = b.dep[slot + 1] = depth + 1;
  b.rturn[slot] = b.rturn[i];
  b.rturn[slot + 1] = b.rturn[i] + 1;
}

// A warp splits a node: its upper_bound of mid probes 32 evenly spaced
// positions per step (the range shrinks 33-fold), then scans the last
// <= 32 -- the index tree_split_node's binary search finds.
__device__ __forceinline__ void tree_split_node_warp(const double* __restrict__ sorted,
                                                     BuildArrays b, int i, int depth,
                                                     int64_t leaf_cap, int lane) {
  const int64_t lo_idx = b.blo[i], hi_idx = b.bhi[i];
  if (hi_idx - lo_idx <= leaf_cap || depth >= MAX_TREE_DEPTH) {
    if (lane == 0) b.lc[i] = b.rc[i] = -1;
    return;
  }
  const double lo = sorted[lo_idx], hi = sorted[hi_idx - 1];
  const double mid = lo + 0.5 * (hi - lo);
  // invariant: sorted[< a] <= mid, sorted[>= e] > mid (or e = hi_idx)
  int64_t a = lo_idx, e = hi_idx;
  while (e - a > 32) {
    const int64_t span = e - a;
    const int64_t pos = a + span * (lane + 1) / 33;  // strictly increasing, in [a, e)
    const unsigned gt = __ballot_sync(0xffffffffu, mid < sorted[pos]);
    if (gt) {
      const int f = __ffs(gt) - 1;  // first probe above mid
      const int64_t pf = a + span * (f + 1) / 33, pprev = a + span * f / 33;
      if (f > 0) a = pprev + 1;  // probe f - 1 was <= mid
      e = pf;
    } else {
      a = a + span * 32 / 33 + 1;
    }
  }
  const unsigned gt = __ballot_sync(0xffffffffu, a + lane < e && mid < sorted[a + lane]);
  int64_t split = gt ? a + (__ffs(gt) - 1) : e;
  if (split == lo_idx || split == hi_idx) split = (lo_idx + hi_idx) / 2;
  if (lane == 0) {
    const int slot = atomicAdd(b.counter, 2);
    b.blo[slot] = lo_idx;
    b.bhi[slot] = split;
    b.blo[slot + 1] = split;
    b.bhi[slot + 1] = hi_idx;
    b.lc[i] = slot;
    b.rc[i] = slot + 1;
    if (b.parent) b.parent[slot] = b.parent[slot + 1] = i;  // absent in the one-CTA build
    if (b.dep) {
      b.dep[slot] = b.dep[slot + 1] = depth + 1;
      b.rturn[slot] = b.rturn[i];
      b.rturn[slot + 1] = b.rturn[i] + 1;
    }
  }
}

// Splits the nodes of level `depth` (its slot range read from b.levels, so
// successive levels launch without host round trips).  The last CTA to
// finish (a ticket taken after a fence) records the next level: exactly the
// children allocated while splitting this one.
__global__ void tree_split_kernel(const double* __restrict__ sorted, BuildArrays b, int depth,
                                  int64_t leaf_cap) {
  const int begin = b.levels[2 * depth], end = b.levels[2 * depth + 1];
  const int nw = (int)((gridDim.x * blockDim.x) >> 5);
  if (end - begin <= nw) {
    // few nodes (the upper levels, long ranges): a warp per node
    const int w = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    if (begin + w < end) tree_split_node_warp(sorted, b, begin + w, depth, leaf_cap,
                                              threadIdx.x & 31);
  } else {
    for (int i = begin + (int)(blockIdx.x * blockDim.x + threadIdx.x); i < end;
         i += (int)(gridDim.x * blockDim.x))
      tree_split_node(sorted, b, i, depth, leaf_cap);
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    const unsigned ticket = atomicAdd(reinterpret_cast<unsigned*>(b.counter + 1), 1u);
    if (ticket == gridDim.x - 1) {
      __threadfence();
      b.levels[2 * depth + 2] = end;
      b.levels[2 * depth + 3] = atomicAdd(b.counter, 0);
      b.counter[1] = 0;  // the next level's launch counts again from zero
    }
  }
}

// Subtree sizes and pre-order indices without a level loop.  The tree is
// full (every internal node has two children), so a node over sources
// [lo, hi) with L leaves has 2 L - 1 nodes, and in pre-order it follows its
// ancestors and, for each right turn on its path, the whole left subtree it
// turned away from; those subtrees hold exactly the leaves before lo:
//   size = 2 L - 1,   pre = depth + 2 * (leaves before lo) - right turns,
// with leaf counts from an exclusive prefix sum of the leaves' start flags.
__global__ void tree_leaf_flags_kernel(BuildArrays b, int nn) {
  const int i = (int)(blockIdx.x * blockDim.x + threadIdx.x);
  if (i < nn && b.lc[i] < 0) b.leafpre[b.blo[i]] = 1;
}

__global__ void tree_order_kernel(BuildArrays b, int nn, const int* __restrict__ prefix) {
  const int i = (int)(blockIdx.x * blockDim.x + threadIdx.x);
  if (i >= nn) return;
  const int before = prefix[b.blo[i]];
  b.size[i] = 2 * (prefix[b.bhi[i]] - before) - 1;
  b.pre[i] = b.dep[i] + 2 * before - b.rturn[i];
}

struct FlatTree {
  double* lo;
  double* hi;
  double* accept_hw;
  int64_t* lo_idx;
  int64_t* hi_idx;
  int32_t* right;
  double* nodes;  // [nn][n]
  double* w;      // [nn][n]
};

__device__ __forceinline__ void tree_fill_node(const double* __restrict__ sorted,
                                               const BuildArrays& b, int i, const FlatTree& f,
                                               const ChebConsts& k, double theta_sq) {
  const int idx = b.pre[i];
  const int64_t lo_idx = b.blo[i], hi_idx = b.bhi[i];
  const double lo = sorted[lo_idx], hi = sorted[hi_idx - 1];
  f.lo[idx] = lo;
  f.hi[idx] = hi;
  const double hw = 0.5 * (hi - lo);
  f.accept_hw[idx] = hw * hw / theta_sq;
  f.lo_idx[idx] = lo_idx;
  f.hi_idx[idx] = hi_idx;
  f.right[idx] = b.lc[i] < 0 ? -1 : b.pre[b.rc[i]];
  const double c = 0.5 * (lo + hi), l = 0.5 * (hi - lo);
  for (int j = 0; j < k.n; ++j) f.nodes[(int64_t)idx * k.n + j] = c + l * k.sm1[j];
}

__global__ void tree_fill_kernel(const double* __restrict__ sorted, BuildArrays b, int nn,
                                 FlatTree f, ChebConsts k, double theta_sq) {
  const int i = (int)(blockIdx.x * blockDim.x + threadIdx.x);
  if (i >= nn) return;
  tree_fill_node(sorted, b, i, f, k, theta_sq);
}

// The topology of a small tree in one CTA (no launch or read-back per
// level): splits level by level with a barrier between levels, subtree sizes
// bottom-up, pre-order indices top-down, the flat arrays.  A warp splits a
// node: its upper_bound of mid probes 32 evenly spaced positions per step
// (the range shrinks 33-fold), then scans the last <= 32 -- the same index as
// tree_split_node's binary search, so the tree is identical.  The levels
// table is left for the host to read once.
constexpr int TOPO_NT = 1024;
// Trees of at most this many leaf-capacities of sources (ns / leaf_cap) are
// built by tree_topology_cta_kernel: a few hundred to ~2 000 nodes, where one
// CTA beats two launches per level (a query-grid tree, a small spectrum).
constexpr int64_t SMALL_TREE_LEAVES = 512;

// The body, for a CTA of any size; parent, dep, rturn and arrive may be null
// (the one-CTA build of tiny trees keeps its node arrays in shared memory and
// needs none of them).  Returns the number of levels.
__device__ int topology_cta(const double* __restrict__ sorted, BuildArrays b, int64_t ns,
                            int64_t leaf_cap, FlatTree f, ChebConsts k, double theta_sq) {
  constexpr int NLEV = MAX_TREE_DEPTH + 2;
  const int nt = blockDim.x;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nw = nt / 32;
  if (tid == 0) {
    b.blo[0] = 0;
    b.bhi[0] = ns;
    b.pre[0] = 0;
    if (b.parent) b.parent[0] = -1;
    if (b.dep) {
      b.dep[0] = 0;
      b.rturn[0] = 0;
    }
    *b.counter = 1;
    b.levels[0] = 0;
    b.levels[1] = 1;
  }
  __syncthreads();
  int last = NLEV - 1;  // first empty level
  for (int depth = 0; depth < NLEV - 1; ++depth) {
    const int begin = b.levels[2 * depth], end = b.levels[2 * depth + 1];
    if (begin == end) {
      last = depth;
      break;
    }
    for (int i = begin + warp; i < end; i += nw)
      tree_split_node_warp(sorted, b, i, depth, leaf_cap, lane);
    __syncthreads();
    if (tid == 0) {
      b.levels[2 * depth + 2] = end;
      b.levels[2 * depth + 3] = *b.counter;
    }
    __syncthreads();
  }
  for (int L = last - 1; L >= 0; --L) {
    const int begin = b.levels[2 * L], end = b.levels[2 * L + 1];
    for (int i = begin + tid; i < end; i += nt)
      b.size[i] = b.lc[i] < 0 ? 1 : 1 + b.size[b.lc[i]] + b.size[b.rc[i]];
    __syncthreads();
  }
  for (int L = 0; L < last; ++L) {
    const int begin = b.levels[2 * L], end = b.levels[2 * L + 1];
    for (int i = begin + tid; i < end; i += nt) {
      if (b.arrive) b.arrive[i] = 0;
      if (b.parent && L == 0) b.parent[i] = -1;
      if (b.lc[i] >= 0) {
        b.pre[b.lc[i]] = b.pre[i] + 1;
        b.pre[b.rc[i]] = b.pre[i] + 1 + b.size[b.lc[i]];
        if (b.parent) {
          b.parent[b.lc[i]] = i;
          b.parent[b.rc[i]] = i;
        }
      }
    }
    __syncthreads();
  }
  const int nn = b.levels[2 * last - 1];
  for (int i = tid; i < nn; i += nt) tree_fill_node(sorted, b, i, f, k, theta_sq);
  return last;
}

__global__ void __launch_bounds__(TOPO_NT, 1) tree_topology_cta_kernel(
    const double* __restrict__ sorted, BuildArrays b, int64_t ns, int64_t leaf_cap, FlatTree f,
    ChebConsts k, double theta_sq) {
  (void)topology_cta(sorted, b, ns, leaf_cap, f, k, theta_sq);
}

// Up to 32 barycentric rows at once, one warp: lane r computes row r's
// parallel part (the first node hit exactly, or the quotients
// q_j = lam_j / (x - t_j) into the warp's shared tile, their sum in order and
// m = mass * (1 / sum)); then lane j < n adds the rows in order,
// w_j = fma(m_r, q_rj, w_j) (w_j + mass_r on a hit at j).  These are the
// operations of chebcode.rs:309-337 barycentric_row (IEEE divisions, the
// sum in node order, the first exact hit taking the whole mass, a fused
// update) applied row after row, so w is the sequential result bit for bit;
// the divisions of 32 rows run in parallel.  Invalid rows (zero masses, the
// tail of a batch) are skipped.
constexpr int ROW_RS = MAX_N + 1;  // shared tile row stride (doubles)
constexpr int WEIGHT_NT = 128;     // threads per block of the weight kernels

struct RowTile {
  double q[32 * ROW_RS];
  double t[MAX_N];
  double lam[MAX_N];
  double m[32];  // row r's scaled mass and exact-hit node (-2: no row)
  int hit[32];
};

__device__ __forceinline__ void bary_rows_batch(double x, double mass, bool valid, int cnt, int n,
                                                int lane, RowTile& rt, double& w) {
  int hit = -2;
  double m = 0.0;
  if (valid) {
    hit = -1;
    for (int j = 0; j < n; ++j)
      if (hit < 0 && x - rt.t[j] == 0.0) hit = j;
    if (hit >= 0) {
      m = mass;
    } else {
      double sum = 0.0;
      for (int j = 0; j < n; ++j) {
        const double q = rt.lam[j] / (x - rt.t[j]);
        rt.q[lane * ROW_RS + j] = q;
        sum += q;
      }
      m = mass * (1.0 / sum);
    }
  }
  rt.m[lane] = m;
  rt.hit[lane] = hit;
  __syncwarp();
  // Rows in order, four at a time: their operands are loaded together (they
  // do not depend on w), then applied one after the other.
  for (int r0 = 0; r0 < cnt; r0 += 4) {
    int hh[4];
    double mm[4], qq[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const int r = r0 + u;
      const bool ok = r < cnt && lane < n;
      hh[u] = ok ? rt.hit[r] : -2;
      mm[u] = ok ? rt.m[r] : 0.0;
      qq[u] = ok ? rt.q[r * ROW_RS + lane] : 0.0;
    }
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      if (hh[u] != -2) {
        if (hh[u] >= 0) {
          if (hh[u] == lane) w = w + mm[u];
        } else {
          w = fma(mm[u], qq[u], w);
        }
      }
    }
  }
  __syncwarp();  // the tile is rewritten by the next batch
}

__device__ __forceinline__ void row_tile_node(RowTile& rt, const FlatTree& f, int idx, int n,
                                              const ChebConsts& k, int lane) {
  if (lane < n) {
    rt.t[lane] = f.nodes[(int64_t)idx * n + lane];
    rt.lam[lane] = k.lam[lane];
  }
  __syncwarp();
}

// P2M, one warp per leaf, its sources 32 at a time in index order.  charges:
// per sorted source (null = unit masses, the reference's P2M); wout: the
// node-weight array [nn][n] to fill.
__device__ __forceinline__ void p2m_leaf(const double* __restrict__ sorted,
                                         const double* __restrict__ charges, const BuildArrays& b,
                                         int i, int lane, const FlatTree& f, double* wout,
                                         const ChebConsts& k, RowTile& rt) {
  const int idx = b.pre[i];
  const int n = k.n;
  row_tile_node(rt, f, idx, n, k, lane);
  double w = 0.0;
  const int64_t q1 = b.bhi[i];
  for (int64_t q0 = b.blo[i]; q0 < q1; q0 += 32) {
    const int cnt = (int)min((int64_t)32, q1 - q0);
    const bool in = lane < cnt;
    const double x = in ? sorted[q0 + lane] : 0.0;
    const double mass = in ? (charges ? charges[q0 + lane] : 1.0) : 0.0;
    bary_rows_batch(x, mass, in, cnt, n, lane, rt, w);
  }
  if (lane < n) wout[(int64_t)idx * n + lane] = w;
}

__global__ void __launch_bounds__(WEIGHT_NT) tree_p2m_kernel(const double* __restrict__ sorted,
                                                             const double* __restrict__ charges,
                                                             BuildArrays b, int nn, FlatTree f,
                                                             double* wout, ChebConsts k) {
  __shared__ RowTile tiles[WEIGHT_NT / 32];
  const int i = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
  const int lane = threadIdx.x & 31;
  if (i >= nn || b.lc[i] >= 0) return;  // whole warps leave together
  p2m_leaf(sorted, charges, b, i, lane, f, wout, k, tiles[threadIdx.x >> 5]);
}

// M2M of node i: rows (child c, child node ti), the left child first, in
// node order, zero masses skipped (2 n <= 32 rows, one batch).  cg: read the
// children's weights past L1 (they may come from another SM in this launch).
__device__ __forceinline__ void m2m_node(const BuildArrays& b, int i, int lane, const FlatTree& f,
                                         double* wts, const ChebConsts& k, bool cg, RowTile& rt) {
  const int idx = b.pre[i];
  const int n = k.n;
  row_tile_node(rt, f, idx, n, k, lane);
  double x = 0.0, mass = 0.0;
  if (lane < 2 * n) {
    const int kid = b.pre[lane < n ? b.lc[i] : b.rc[i]], ti = lane % n;
    const double* mp = wts + (int64_t)kid * n + ti;
    mass = cg ? __ldcg(mp) : *mp;
    x = f.nodes[(int64_t)kid * n + ti];
  }
  double w = 0.0;
  bary_rows_batch(x, mass, lane < 2 * n && mass != 0.0, 2 * n, n, lane, rt, w);
  if (lane < n) wts[(int64_t)idx * n + lane] = w;
}

__global__ void __launch_bounds__(WEIGHT_NT) tree_m2m_kernel(BuildArrays b, int begin, int end,
                                                             FlatTree f, double* wts,
                                                             ChebConsts k) {
  __shared__ RowTile tiles[WEIGHT_NT / 32];
  const int i = begin + (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
  const int lane = threadIdx.x & 31;
  if (i >= end || b.lc[i] < 0) return;  // whole warps leave together
  m2m_node(b, i, lane, f, wts, k, false, tiles[threadIdx.x >> 5]);
}

__device__ __forceinline__ void mirror_f32(const FlatTree& f, int idx, int n, int lane,
                                           NodeF32* nf, float* panel) {
  if (lane == 0)
    nf[idx] = {(float)f.lo[idx], (float)f.hi[idx], (float)f.accept_hw[idx],
               (uint32_t)f.lo_idx[idx], (uint32_t)f.hi_idx[idx], f.right[idx]};
  if (lane < n) {
    panel[(int64_t)idx * 2 * n + lane] = (float)f.nodes[(int64_t)idx * n + lane];
    panel[(int64_t)idx * 2 * n + n + lane] = (float)__ldcg(f.w + (int64_t)idx * n + lane);
  }
}

// P2M and M2M of a small tree in one launch over a fixed grid, with no
// read-back (the node count is the breadth-first slot counter): a warp
// fills a leaf, then climbs -- it fences its weights and counts itself in at
// the parent; the warp that brings the count to two (the last child done)
// merges the parent (m2m_node, children's weights read past L1) and goes on
// up, the other stops.  No warp waits on another.  Each node's f32 mirror
// entry is written once its weights are final (nf null: none).
__global__ void __launch_bounds__(WEIGHT_NT, 1) tree_p2m_grid_kernel(
    const double* __restrict__ sorted, BuildArrays b, FlatTree f, double* wout, ChebConsts k,
    NodeF32* nf, float* panel) {
  __shared__ RowTile tiles[WEIGHT_NT / 32];
  RowTile& rt = tiles[threadIdx.x >> 5];
  const int nn = *b.counter;
  const int lane = threadIdx.x & 31;
  const int nw = (int)((gridDim.x * blockDim.x) >> 5);
  for (int i = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5); i < nn; i += nw) {
    if (b.lc[i] >= 0) continue;  // warp-uniform
    p2m_leaf(sorted, nullptr, b, i, lane, f, wout, k, rt);
    if (nf) mirror_f32(f, b.pre[i], k.n, lane, nf, panel);
    for (int node = i;;) {
      const int par = b.parent[node];
      if (par < 0) break;
      __threadfence();  // this node's weights before the count
      int seen = 0;
      if (lane == 0) seen = atomicAdd(&b.arrive[par], 1);
      seen = __shfl_sync(0xffffffffu, seen, 0);
      if (seen == 0) break;  // the sibling's warp merges the parent
      __threadfence();
      m2m_node(b, par, lane, f, wout, k, true, rt);
      if (nf) mirror_f32(f, b.pre[par], k.n, lane, nf, panel);
      node = par;
    }
  }
}

// The whole build of a tiny tree (ns <= TINY_NS sources) in one CTA and one
// launch: the spectrum and every node array of the topology in shared memory
// (a tree over ns sources has at most 2 ns - 1 nodes), the flat arrays, the
// P2M of the leaves, then the M2M level by level from the deepest with a
// barrier between levels, and the f32 mirror.  The same device functions as
// the multi-launch builds, node by node, so the same tree and the same
// weights bit for bit; what goes is a launch, the per-level round trips to
// global memory and the climbing warps' fences and arrival counters.
constexpr int64_t TINY_NS = 2048;
constexpr int TINY_NT = 1024;
constexpr int TINY_TILES = 16;  // warps with a row tile (P2M / M2M)

__device__ __forceinline__ unsigned dyn_smem_size() {
  unsigned r;
  asm volatile("mov.u32 %0, %%dynamic_smem_size;" : "=r"(r));
  return r;
}

__host__ __device__ size_t tiny_smem_bytes(int64_t ns) {
  constexpr int NLEV = MAX_TREE_DEPTH + 2;
  const size_t cap = (size_t)(2 * ns > 2 ? 2 * ns : 2);
  return sizeof(RowTile) * TINY_TILES + sizeof(double) * (size_t)ns +
         sizeof(int64_t) * 2 * cap + sizeof(int32_t) * (4 * cap + 8 + 2 * NLEV);
}

__global__ void __launch_bounds__(TINY_NT, 1) tree_tiny_kernel(
    const double* __restrict__ sorted_g, int64_t ns, int64_t leaf_cap, FlatTree f, ChebConsts k,
    double theta_sq, NodeF32* nf, float* panel, int* nn_out) {
  extern __shared__ __align__(16) unsigned char tiny_sm[];
  const int64_t cap = ns * 2 > 2 ? ns * 2 : 2;
  RowTile* tiles = reinterpret_cast<RowTile*>(tiny_sm);
  double* s_sorted = reinterpret_cast<double*>(tiles + TINY_TILES);
  BuildArrays b;
  b.blo = reinterpret_cast<int64_t*>(s_sorted + ns);
  b.bhi = b.blo + cap;
  b.lc = reinterpret_cast<int32_t*>(b.bhi + cap);
  b.rc = b.lc + cap;
  b.size = b.rc + cap;
  b.pre = b.size + cap;
  b.counter = b.pre + cap;
  b.levels = b.counter + 8;
  b.parent = b.arrive = b.dep = b.rturn = b.leafpre = nullptr;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  for (int64_t i = tid; i < ns; i += blockDim.x) s_sorted[i] = sorted_g[i];
  __syncthreads();
  const int last = topology_cta(s_sorted, b, ns, leaf_cap, f, k, theta_sq);
  __syncthreads();
  const int nn = b.levels[2 * last - 1];
  // The Chebyshev nodes and weights in the shared memory left over when the
  // tree is small enough (typically: nn is far below its bound 2 ns - 1):
  // the M2M chain, one level after another, then runs without an L2 round
  // trip per level; the weights are copied out at the end.
  const size_t used = tiny_smem_bytes(ns);
  const size_t need = sizeof(double) * 2 * (size_t)nn * k.n;
  FlatTree fw = f;
  const bool in_smem = used + need <= (size_t)dyn_smem_size();
  if (in_smem) {
    double* sn = reinterpret_cast<double*>(tiny_sm + used);
    for (int i = tid; i < nn * k.n; i += blockDim.x) sn[i] = f.nodes[i];
    fw.nodes = sn;
    fw.w = sn + (size_t)nn * k.n;
    __syncthreads();
  }
  if (warp < TINY_TILES)
    for (int i = warp; i < nn; i += TINY_TILES)
      if (b.lc[i] < 0) p2m_leaf(s_sorted, nullptr, b, i, lane, fw, fw.w, k, tiles[warp]);
  __syncthreads();
  for (int L = last - 2; L >= 0; --L) {  // level last - 1 holds leaves only
    const int begin = b.levels[2 * L], end = b.levels[2 * L + 1];
    if (warp < TINY_TILES)
      for (int i = begin + warp; i < end; i += TINY_TILES)
        if (b.lc[i] >= 0) m2m_node(b, i, lane, fw, fw.w, k, !in_smem, tiles[warp]);
    __syncthreads();
  }
  if (in_smem) {
    for (int i = tid; i < nn * k.n; i += blockDim.x) f.w[i] = fw.w[i];
    __syncthreads();
  }
  if (nf)
    for (int idx = warp; idx < nn; idx += (int)(blockDim.x >> 5))
      mirror_f32(f, idx, k.n, lane, nf, panel);
  if (tid == 0) *nn_out = nn;
}

// M2M, one warp per internal node of a level: the left then the right
// child's node masses, in node order.


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

// Up to this many queries the evaluation takes a warp per query (a thread per
// query leaves most of the GPU idle and each traversal serial).
constexpr int64_t CHEB_WARP_NQ = 16384;

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
  // Node count (nn_dev on the device when the build kept it there, else
  // nn_host) and the dynamic shared memory each CTA may fill with a copy of
  // the tree's node records (0: read them from global memory).  A traversal
  // is a chain of dependent node loads; from shared memory each costs tens
  // of cycles instead of an L2 round trip.
  const int* nn_dev;
  int nn_host;
  int stage_bytes;
};

// Staged node record of the FP64 traversal.
struct NodeHdr64 {
  double lo, hi, accept_hw;
  int64_t lo_idx, hi_idx;
  int32_t right, pad;
};

constexpr int CHEB_STAGE_BYTES = 48 * 1024;

__device__ __forceinline__ int eval_node_count(const EvalArgs& a) {
  return a.nn_dev ? *a.nn_dev : a.nn_host;
}

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

// The same leaf sum with a warp per query (every lane holds the same x):
// lane l computes the terms of sources base + l in parallel, then every lane
// adds them in the sequential order through shuffles -- the two chains of
// the F64x2 schedule, their sum, then the odd tail -- so the result equals
// leaf_sum bit for bit.  Used when there are too few queries to fill the GPU
// with one thread each (the reciprocals dominate, the ordered adds are cheap).
__device__ __forceinline__ void leaf_sum_warp(const double* xs, int64_t len, double x,
                                              double eta2, int lane, double& lr_out,
                                              double& li_out) {
  double ar0 = 0.0, ar1 = 0.0, ai0 = 0.0, ai1 = 0.0, tr = 0.0, ti = 0.0;
  const int64_t pair_end = len & ~(int64_t)1;
  for (int64_t base = 0; base < len; base += 32) {
    const int64_t k = base + lane;
    double vr = 0.0, vi = 0.0;
    if (k < len) {
      const double d = x - xs[k];
      const double inv = __drcp_rn(eta2 + d * d);  // = d * d + eta2 for the tail
      vr = d * inv;
      vi = inv;
    }
    const int cnt = (int)min((int64_t)32, len - base);
    // four terms' shuffles issued together (they do not depend on the
    // sums), then added one after the other in source order
    for (int j0 = 0; j0 < cnt; j0 += 4) {
      double rr[4], ii[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        rr[u] = __shfl_sync(0xffffffffu, vr, j0 + u);
        ii[u] = __shfl_sync(0xffffffffu, vi, j0 + u);
      }
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        if (j0 + u >= cnt) break;
        const int64_t kk = base + j0 + u;
        if (kk >= pair_end) {
          tr = rr[u];
          ti = ii[u];
        } else if (kk & 1) {
          ar1 = ar1 + rr[u];
          ai1 = ai1 + ii[u];
        } else {
          ar0 = ar0 + rr[u];
          ai0 = ai0 + ii[u];
        }
      }
    }
  }
  double lr = ar0 + ar1, li = ai0 + ai1;
  if (len & 1) {
    lr += tr;
    li += ti;
  }
  lr_out = lr;
  li_out = li;
}

// chebcode.rs:607-711 contribution_f64.  WARP: a warp per query (all lanes
// walk the same nodes; leaf sums by leaf_sum_warp; lane 0 stores).
template <bool WARP>
__global__ void __launch_bounds__(128) cheb_eval_f64(const EvalArgs a) {
  extern __shared__ __align__(16) unsigned char stage_raw[];
  const int64_t gt = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t t = WARP ? gt >> 5 : gt;
  const int lane = WARP ? (int)(threadIdx.x & 31) : 0;
  const DevTreeF64& T = a.t;
  const int n = T.n;
  // Node records in shared memory when they fit (the same values, so the
  // same arithmetic); the node count is uniform, so is the branch.
  const NodeHdr64* sh = nullptr;
  const double* s_nodes = nullptr;
  if (a.stage_bytes > 0) {
    const int nn = eval_node_count(a);
    const size_t hb = (size_t)nn * sizeof(NodeHdr64), pb = (size_t)nn * 2 * n * sizeof(double);
    if (hb <= (size_t)a.stage_bytes) {
      NodeHdr64* h = reinterpret_cast<NodeHdr64*>(stage_raw);
      for (int i = threadIdx.x; i < nn; i += blockDim.x)
        h[i] = NodeHdr64{T.lo[i], T.hi[i], T.accept_hw[i], T.lo_idx[i], T.hi_idx[i], T.right[i], 0};
      sh = h;
      if (hb + pb <= (size_t)a.stage_bytes) {
        double* d = reinterpret_cast<double*>(stage_raw + hb);
        for (int i = threadIdx.x; i < nn * n; i += blockDim.x) {
          d[i] = T.nodes[i];
          d[nn * n + i] = T.w[i];
        }
        s_nodes = d;
      }
    }
    __syncthreads();
  }
  if (t >= a.nq) return;  // WARP: whole warps leave together
  const int nn_s = s_nodes ? eval_node_count(a) : 0;
  const double x = a.q[t], eta = a.eta, eta2 = eta * eta;
  int32_t stack[MAX_TREE_DEPTH + 2];
  int top = 0;
  stack[top++] = 0;
  double re = 0.0, im = 0.0;
  while (top > 0) {
    const int32_t node = stack[--top];
    const int32_t rt = sh ? sh[node].right : T.right[node];
    if (rt < 0) {
      double lr, li;
      const int64_t l0 = sh ? sh[node].lo_idx : T.lo_idx[node];
      const int64_t l1 = sh ? sh[node].hi_idx : T.hi_idx[node];
      if (WARP) leaf_sum_warp(a.sorted + l0, l1 - l0, x, eta2, lane, lr, li);
      else leaf_sum(a.sorted + l0, l1 - l0, x, eta2, lr, li);
      re += lr;
      im += eta * li;
      continue;
    }
    const double lo = sh ? sh[node].lo : T.lo[node], hi = sh ? sh[node].hi : T.hi[node];
    const double cl = fmax(fmax(lo - x, x - hi), 0.0);
    const double d_sq = fma(cl, cl, eta2);
    if ((sh ? sh[node].accept_hw : T.accept_hw[node]) < d_sq) {
      const double* ts = (s_nodes ? s_nodes : T.nodes) + (int64_t)node * n;
      const double* ws = (s_nodes ? s_nodes + (int64_t)nn_s * n : T.w) + (int64_t)node * n;
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
  if (lane == 0) epi_store(a.epi, t, x, re, im);
}

// chebcode.rs:722-828 contribution_fast32.  WARP as cheb_eval_f64.
template <bool WARP>
__global__ void __launch_bounds__(128) cheb_eval_f32(const EvalArgs a) {
  extern __shared__ __align__(16) unsigned char stage_raw[];
  const int64_t gt = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t t = WARP ? gt >> 5 : gt;
  const int lane = WARP ? (int)(threadIdx.x & 31) : 0;
  const int n = a.t.n;
  // Node records and panel in shared memory when they fit (see cheb_eval_f64).
  const NodeF32* nfp = a.nf;
  const float* panel = a.panel;
  if (a.stage_bytes > 0) {
    const int nn = eval_node_count(a);
    const size_t hb = (size_t)nn * sizeof(NodeF32), pb = (size_t)nn * 2 * n * sizeof(float);
    if (hb <= (size_t)a.stage_bytes) {
      NodeF32* h = reinterpret_cast<NodeF32*>(stage_raw);
      for (int i = threadIdx.x; i < nn; i += blockDim.x) h[i] = a.nf[i];
      nfp = h;
      if (hb + pb <= (size_t)a.stage_bytes) {
        float* d = reinterpret_cast<float*>(stage_raw + hb);
        for (int i = threadIdx.x; i < nn * 2 * n; i += blockDim.x) d[i] = a.panel[i];
        panel = d;
      }
    }
    __syncthreads();
  }
  if (t >= a.nq) return;  // WARP: whole warps leave together
  const double lambda = a.q[t], eta = a.eta, eta2d = eta * eta;
  const float x = (float)lambda, e32 = (float)eta, eta2 = e32 * e32;
  float fre[4] = {0.f, 0.f, 0.f, 0.f}, fim[4] = {0.f, 0.f, 0.f, 0.f};
  double leaf_re = 0.0, leaf_im = 0.0;
  int32_t stack[MAX_TREE_DEPTH + 2];
  int top = 0;
  stack[top++] = 0;
  while (top > 0) {
    const int32_t node = stack[--top];
    const NodeF32 nd = nfp[node];
    if (nd.right < 0) {
      double lr, li;
      if (WARP)
        leaf_sum_warp(a.sorted + nd.lo_idx, (int64_t)(nd.hi_idx - nd.lo_idx), lambda, eta2d,
                      lane, lr, li);
      else
        leaf_sum(a.sorted + nd.lo_idx, (int64_t)(nd.hi_idx - nd.lo_idx), lambda, eta2d, lr, li);
      leaf_re += lr;
      leaf_im += eta * li;
      continue;
    }
    const float cl = fmaxf(fmaxf(nd.lo - x, x - nd.hi), 0.0f);
    const float d_sq = fmaf(cl, cl, eta2);
    const float outside = (cl == 0.0f) ? d_sq : OUTSIDE_THETA2 * d_sq;
    if (nd.accept_hw < outside) {
      const float* ts = panel + (int64_t)node * 2 * n;
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
  if (lane == 0) epi_store(a.epi, t, lambda, leaf_re + (double)hr, leaf_im + eta * (double)hi);
}

__global__ void tree_init_kernel(BuildArrays b, int64_t ns) {
  b.blo[0] = 0;
  b.bhi[0] = ns;
  b.pre[0] = 0;
  b.parent[0] = -1;
  b.dep[0] = 0;
  b.rturn[0] = 0;
  b.counter[1] = 0;
  *b.counter = 1;
  b.levels[0] = 0;
  b.levels[1] = 1;
}

// F32 mirror of the flat tree for the fast preset (NodeF32 + node panels).
__global__ void tree_f32_kernel(FlatTree f, int nn, int n, NodeF32* nf, float* panel) {
  const int i = (int)(blockIdx.x * blockDim.x + threadIdx.x);
  if (i >= nn) return;
  nf[i] = {(float)f.lo[i], (float)f.hi[i], (float)f.accept_hw[i], (uint32_t)f.lo_idx[i],
           (uint32_t)f.hi_idx[i], f.right[i]};
  for (int j = 0; j < n; ++j) {
    panel[(int64_t)i * 2 * n + j] = (float)f.nodes[(int64_t)i * n + j];
    panel[(int64_t)i * 2 * n + n + j] = (float)f.w[(int64_t)i * n + j];
  }
}

unsigned blocks_for(int64_t n, int bs) { return (unsigned)((n + bs - 1) / bs); }

// A built tree: the flat arrays plus what further weight sets need (the
// breadth-first arrays stay valid in scratch until the next build).
struct TreeBuild {
  FlatTree f;
  int nn = 0;
  std::vector<int> lb, le;  // breadth-first level ranges
  BuildArrays b;
  ChebConsts k;
};

// Node weights of `charges` (per sorted source; null = unit masses) into
// wout: P2M at the leaves, then M2M from the deepest internal level up.
shrk_status tree_weights(const TreeBuild& tb, const double* d_sorted, const double* charges,
                         double* wout, cudaStream_t s) {
  tree_p2m_kernel<<<blocks_for((int64_t)tb.nn * 32, WEIGHT_NT), WEIGHT_NT, 0, s>>>(d_sorted, charges, tb.b,
                                                                       tb.nn, tb.f, wout, tb.k);
  SHRK_CUDA(cudaGetLastError());
  const int levels = (int)tb.lb.size();
  for (int L = levels - 2; L >= 0; --L) {
    tree_m2m_kernel<<<blocks_for((int64_t)(tb.le[L] - tb.lb[L]) * 32, WEIGHT_NT), WEIGHT_NT, 0, s>>>(
        tb.b, tb.lb[L], tb.le[L], tb.f, wout, tb.k);
    SHRK_CUDA(cudaGetLastError());
  }
  add_launches(1 + std::max(levels - 1, 0));
  return SHRK_OK;
}

// Builds the flat tree of d_sorted (ascending) into the TREE_SLOTS scratch.
// Scratch slots 25/26 hold the breadth-first build arrays.
shrk_status build_tree_gpu(const double* d_sorted, int64_t ns, const ChebParams& prm,
                           TreeBuild& tb, cudaStream_t s) {
  FlatTree& f = tb.f;
  const int64_t cap = std::max<int64_t>(2 * ns, 2);
  if (cap > (int64_t)INT32_MAX / 2) {
    set_error("chebcode: too many eigenvalues for the tree build");
    return SHRK_EINVAL;
  }
  ChebConsts k;
  k.n = prm.n;
  for (int j = 0; j < prm.n; ++j) {
    k.sm1[j] = std::cos((double)j * M_PI / (double)(prm.n - 1));
    const double sign = (j % 2 == 0) ? 1.0 : -1.0;
    k.lam[j] = (j == 0 || j == prm.n - 1) ? 0.5 * sign : sign;
  }
  void* p64 = nullptr;
  void* p32 = nullptr;
  SHRK_TRY(scratch_get(25, sizeof(int64_t) * 2 * (size_t)cap, &p64));
  constexpr int NLEV = MAX_TREE_DEPTH + 2;  // levels 0..48 split, level 49 is empty
  SHRK_TRY(scratch_get(26, sizeof(int32_t) * (8 * (size_t)cap + (size_t)ns + 2 + 8 + 2 * NLEV),
                       &p32));
  BuildArrays b;
  b.blo = (int64_t*)p64;
  b.bhi = b.blo + cap;
  b.lc = (int32_t*)p32;
  b.rc = b.lc + cap;
  b.size = b.rc + cap;
  b.pre = b.size + cap;
  b.counter = (int*)(b.pre + cap);
  b.levels = b.counter + 8;
  b.parent = b.levels + 2 * NLEV;
  b.arrive = b.parent + cap;
  b.dep = b.arrive + cap;
  b.rturn = b.dep + cap;
  b.leafpre = b.rturn + cap;
  constexpr int BS = 256;
  if (ns / std::max<int64_t>(prm.leaf_cap, 1) <= SMALL_TREE_LEAVES) {
    // small tree: the whole topology in one CTA, one read-back of the levels
    // (the flat arrays are sized for the 2 ns node bound)
    void* q = nullptr;
    SHRK_TRY(scratch_get(TREE_SLOTS + 0, sizeof(double) * 3 * (size_t)cap, &q));
    f.lo = (double*)q;
    f.hi = f.lo + cap;
    f.accept_hw = f.hi + cap;
    SHRK_TRY(scratch_get(TREE_SLOTS + 1, sizeof(int64_t) * 2 * (size_t)cap, &q));
    f.lo_idx = (int64_t*)q;
    f.hi_idx = f.lo_idx + cap;
    SHRK_TRY(scratch_get(TREE_SLOTS + 2, sizeof(int32_t) * (size_t)cap, &q));
    f.right = (int32_t*)q;
    SHRK_TRY(scratch_get(TREE_SLOTS + 3, sizeof(double) * 2 * (size_t)cap * prm.n, &q));
    f.nodes = (double*)q;
    f.w = f.nodes + (size_t)cap * prm.n;
    {
      LaunchScope ls("cheb_build", s);
      tree_topology_cta_kernel<<<1, TOPO_NT, 0, s>>>(d_sorted, b, ns, (int64_t)prm.leaf_cap, f, k,
                                                     prm.theta * prm.theta);
      SHRK_CUDA(cudaGetLastError());
    }
    int h_lev[2 * NLEV];
    SHRK_CUDA(cudaMemcpyAsync(h_lev, b.levels, sizeof(h_lev), cudaMemcpyDeviceToHost, s));
    SHRK_CUDA(cudaStreamSynchronize(s));
    int last = NLEV - 1;
    for (int L = 1; L < NLEV; ++L)
      if (h_lev[2 * L] == h_lev[2 * L + 1]) {
        last = L;
        break;
      }
    std::vector<int> lb, le;
    for (int L = 0; L < last; ++L) {
      lb.push_back(h_lev[2 * L]);
      le.push_back(h_lev[2 * L + 1]);
    }
    tb.nn = le.back();
    tb.lb = lb;
    tb.le = le;
    tb.b = b;
    tb.k = k;
    return tree_weights(tb, d_sorted, nullptr, f.w, s);
  }
  {
    LaunchScope ls("cheb_build", s);
    tree_init_kernel<<<1, 1, 0, s>>>(b, ns);
    SHRK_CUDA(cudaGetLastError());
  }
  // 1. split, level by level (each level's children fill the next slots);
  //    levels run in batches with one read-back of the level table per batch
  //    to see whether a level came out empty: the first batch covers the
  //    depth a balanced tree would need plus a margin, later ones 8 levels.
  const int split_grid = std::max(1, sm_count() * 4);
  int h_lev[2 * NLEV];
  int last = -1;  // first empty level
  const int64_t leaves_est = std::max<int64_t>(ns / std::max<int64_t>(prm.leaf_cap, 1), 1);
  int batch = 8;
  while ((int64_t{1} << (batch - 8)) < leaves_est && batch < NLEV - 1) ++batch;
  for (int L0 = 0; last < 0;) {
    const int L1 = std::min(L0 + batch, NLEV - 1);
    batch = 8;
    for (int L = L0; L < L1; ++L) {
      tree_split_kernel<<<split_grid, BS, 0, s>>>(d_sorted, b, L, (int64_t)prm.leaf_cap);
      SHRK_CUDA(cudaGetLastError());
    }
    add_launches(L1 - L0);
    SHRK_CUDA(cudaMemcpyAsync(h_lev, b.levels, sizeof(h_lev), cudaMemcpyDeviceToHost, s));
    SHRK_CUDA(cudaStreamSynchronize(s));
    for (int L = L0 + 1; L <= L1; ++L)
      if (h_lev[2 * L] == h_lev[2 * L + 1]) {
        last = L;
        break;
      }
    if (last < 0 && L1 == NLEV - 1) last = L1;  // cannot happen: depth 48 never splits
    L0 = L1;
  }
  std::vector<int> lb, le;
  for (int L = 0; L < last; ++L) {
    lb.push_back(h_lev[2 * L]);
    le.push_back(h_lev[2 * L + 1]);
  }
  const int nn = le.back();
  // 2. subtree sizes and pre-order indices from the leaves' start flags
  //    (tree_order_kernel); the arrival counters hold the prefix meanwhile
  {
    LaunchScope ls("cheb_build", s);
    SHRK_CUDA(cudaMemsetAsync(b.leafpre, 0, sizeof(int32_t) * ((size_t)ns + 1), s));
    tree_leaf_flags_kernel<<<blocks_for(nn, BS), BS, 0, s>>>(b, nn);
    SHRK_CUDA(cudaGetLastError());
    size_t temp_bytes = 0;
    SHRK_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, temp_bytes, b.leafpre, b.arrive,
                                            (int)(ns + 1), s));
    void* temp = nullptr;
    SHRK_TRY(scratch_get(28, std::max<size_t>(temp_bytes, 256), &temp));
    SHRK_CUDA(cub::DeviceScan::ExclusiveSum(temp, temp_bytes, b.leafpre, b.arrive,
                                            (int)(ns + 1), s));
    tree_order_kernel<<<blocks_for(nn, BS), BS, 0, s>>>(b, nn, b.arrive);
    SHRK_CUDA(cudaGetLastError());
    add_launches(3);  // flags, the scan's two kernels, order
  }
  // 3. flat arrays
  void* q = nullptr;
  SHRK_TRY(scratch_get(TREE_SLOTS + 0, sizeof(double) * 3 * (size_t)nn, &q));
  f.lo = (double*)q;
  f.hi = f.lo + nn;
  f.accept_hw = f.hi + nn;
  SHRK_TRY(scratch_get(TREE_SLOTS + 1, sizeof(int64_t) * 2 * (size_t)nn, &q));
  f.lo_idx = (int64_t*)q;
  f.hi_idx = f.lo_idx + nn;
  SHRK_TRY(scratch_get(TREE_SLOTS + 2, sizeof(int32_t) * (size_t)nn, &q));
  f.right = (int32_t*)q;
  SHRK_TRY(scratch_get(TREE_SLOTS + 3, sizeof(double) * 2 * (size_t)nn * prm.n, &q));
  f.nodes = (double*)q;
  f.w = f.nodes + (size_t)nn * prm.n;
  tree_fill_kernel<<<blocks_for(nn, BS), BS, 0, s>>>(d_sorted, b, nn, f, k,
                                                     prm.theta * prm.theta);
  SHRK_CUDA(cudaGetLastError());
  add_launches(1);
  tb.nn = nn;
  tb.lb = lb;
  tb.le = le;
  tb.b = b;
  tb.k = k;
  // 4. P2M at the leaves; 5. M2M from the deepest internal level up (a
  //    level-parallel launch per level: at this size the climbing form of
  //    the small trees was measured 2.3x slower)
  return tree_weights(tb, d_sorted, nullptr, f.w, s);
}

// ------------------------------------------------------ multi-eta --
// chebcode.rs:836-915 contribution_x2: two etas per traversal (the
// reference's F64x2 lanes; on its x86 target lane multiply-adds are unfused
// and the reciprocal is a true division -- both reproduced here, the build
// contracts nothing).  A node is accepted when half_w^2 < theta^2 (cl^2 +
// min(eta)^2), i.e. only if both lanes would accept it.  One thread per
// (point, eta pair); results bit-exact with the reference algorithm.
struct ManyArgs {
  const double* x;       // evaluation points (the eigenvalues, caller's order)
  int64_t p;
  const double* sorted;
  const double* etas;
  int64_t n_eta;
  DevTreeF64 t;
  double theta_sq;
  double* out_re;        // [n_eta][p]
  double* out_im;
  int* err;
};

__global__ void __launch_bounds__(128) cheb_eval_x2(const ManyArgs a) {
  const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t n_pairs = (a.n_eta + 1) / 2;
  if (g >= a.p * n_pairs) return;
  const int64_t i = g % a.p, k = (g / a.p) * 2;
  const bool two = k + 1 < a.n_eta;
  const double e0 = a.etas[k], e1 = two ? a.etas[k + 1] : e0;
  const double e2a = e0 * e0, e2b = e1 * e1, e_min = fmin(e0, e1);
  const DevTreeF64& T = a.t;
  const int n = T.n;
  const double x = a.x[i];
  int32_t stack[MAX_TREE_DEPTH + 2];
  int top = 0;
  stack[top++] = 0;
  double ar0 = 0.0, ar1 = 0.0, ai0 = 0.0, ai1 = 0.0;
  while (top > 0) {
    const int32_t node = stack[--top];
    const int32_t rt = T.right[node];
    if (rt < 0) {
      for (int64_t q = T.lo_idx[node]; q < T.hi_idx[node]; ++q) {
        const double d = x - a.sorted[q];
        const double dd = d * d;
        const double inv0 = 1.0 / (e2a + dd), inv1 = 1.0 / (e2b + dd);
        ar0 = ar0 + d * inv0;
        ar1 = ar1 + d * inv1;
        ai0 = ai0 + e0 * inv0;
        ai1 = ai1 + e1 * inv1;
      }
      continue;
    }
    const double lo = T.lo[node], hi = T.hi[node];
    const double cl = x < lo ? lo - x : (x > hi ? x - hi : 0.0);
    const double d_sq = cl * cl + e_min * e_min;
    const double half_w = 0.5 * (hi - lo);
    if (half_w * half_w < a.theta_sq * d_sq) {
      const int64_t base = (int64_t)node * n;
      for (int j = 0; j < n; ++j) {
        const double dj = x - T.nodes[base + j];
        const double wj = T.w[base + j];
        const double dd = dj * dj;
        const double inv0 = 1.0 / (e2a + dd), inv1 = 1.0 / (e2b + dd);
        const double wd = wj * dj;
        ar0 = ar0 + wd * inv0;
        ar1 = ar1 + wd * inv1;
        ai0 = ai0 + (wj * e0) * inv0;
        ai1 = ai1 + (wj * e1) * inv1;
      }
    } else {
      if (top + 2 > MAX_TREE_DEPTH + 2) {  // cannot happen for a depth-capped tree
        atomicExch(a.err, DEV_ERR_BOUNDS);
        break;
      }
      stack[top++] = rt;
      stack[top++] = node + 1;
    }
  }
  a.out_re[k * a.p + i] = ar0;
  a.out_im[k * a.p + i] = ai0;
  if (two) {
    a.out_re[(k + 1) * a.p + i] = ar1;
    a.out_im[(k + 1) * a.p + i] = ai1;
  }
}

// ------------------------------------------------ treecode adjoint --
// Gradient of L = sum_j (w_j Re m_j + v_j Im m_j) (the adjoint of the
// all-points transform, no reference counterpart) with the source sums of
// the squared kernel K2(a) = 1/(a - i eta)^2 = (A + iB), a = x_k - y_j,
//   A = (a^2 - eta^2)/D^2 = r - 2 eta^2 r^2,  B = 2 a eta/D^2,  r = 1/D,
// evaluated by the same tree: grad_k = (1/p)[w_k Re T1 - Re Tw - v_k Im T1
// - Im Tv] with T_c = sum_j c_j K2(x_k - y_j) for the charges c = 1, w, v.
// Leaves sum exactly; an accepted node (the forward's acceptance test)
// contributes sum_i W^c_i K2(x_k - t_i) with its Chebyshev node weights of
// charge c (P2M with masses c_j, then M2M).
struct AdjEvalArgs {
  const double* x;   // targets = the eigenvalues, caller's order
  const double* w;   // cotangents, caller's order
  const double* v;
  int64_t p;
  const double* sorted;
  const double* cw;  // charges in sorted order
  const double* cv;
  double eta;
  DevTreeF64 t;      // t.w: unit-mass node weights
  const double* ww;  // node weights of charges w
  const double* wv;  // node weights of charges v
  double* grad;
  int* err;
};

__device__ __forceinline__ void k2_terms(double d, double eta2, double m2e2, double teta,
                                         double& A, double& B) {
  const double r = rcp_f64(fma(d, d, eta2));
  const double r2 = r * r;
  A = fma(m2e2, r2, r);
  B = teta * d * r2;
}

__global__ void __launch_bounds__(128) cheb_adjoint_f64(const AdjEvalArgs a) {
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= a.p) return;
  const DevTreeF64& T = a.t;
  const int n = T.n;
  const double x = a.x[k], eta = a.eta, eta2 = eta * eta;
  const double m2e2 = -2.0 * eta2, teta = 2.0 * eta;
  int32_t stack[MAX_TREE_DEPTH + 2];
  int top = 0;
  stack[top++] = 0;
  double s1r = 0.0, s1i = 0.0, swr = 0.0, svi = 0.0;
  while (top > 0) {
    const int32_t node = stack[--top];
    const int32_t rt = T.right[node];
    if (rt < 0) {
      for (int64_t q = T.lo_idx[node]; q < T.hi_idx[node]; ++q) {
        double A, B;
        k2_terms(x - a.sorted[q], eta2, m2e2, teta, A, B);
        s1r += A;
        s1i += B;
        swr = fma(a.cw[q], A, swr);
        svi = fma(a.cv[q], B, svi);
      }
      continue;
    }
    const double lo = T.lo[node], hi = T.hi[node];
    const double cl = fmax(fmax(lo - x, x - hi), 0.0);
    if (T.accept_hw[node] < fma(cl, cl, eta2)) {
      const int64_t base = (int64_t)node * n;
      for (int j = 0; j < n; ++j) {
        double A, B;
        k2_terms(x - T.nodes[base + j], eta2, m2e2, teta, A, B);
        const double w1 = T.w[base + j];
        s1r = fma(w1, A, s1r);
        s1i = fma(w1, B, s1i);
        swr = fma(a.ww[base + j], A, swr);
        svi = fma(a.wv[base + j], B, svi);
      }
    } else {
      if (top + 2 > MAX_TREE_DEPTH + 2) {  // cannot happen for a depth-capped tree
        atomicExch(a.err, DEV_ERR_BOUNDS);
        break;
      }
      stack[top++] = rt;
      stack[top++] = node + 1;
    }
  }
  a.grad[k] = (a.w[k] * s1r - swr - a.v[k] * s1i - svi) / (double)a.p;
}

// Charges in sorted order: out[i] = c[perm[i]] (perm null: identity).
__global__ void gather_charges_kernel(const double* __restrict__ gw, const double* __restrict__ gv,
                                      const int* __restrict__ perm, int64_t n, double* cw,
                                      double* cv) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int64_t j = perm ? perm[i] : i;
  cw[i] = gw[j];
  cv[i] = gv[j];
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

// The forward evaluation's tree for a small spectrum (ns / leaf_cap <=
// SMALL_TREE_LEAVES) with no read-back: the topology in one CTA, then P2M,
// M2M and the f32 mirror in one launch over a fixed grid
// (tree_p2m_grid_kernel).
static bool fused_build_ok(int64_t ns, const ChebParams& prm) {
  return ns / std::max<int64_t>(prm.leaf_cap, 1) <= SMALL_TREE_LEAVES;
}

static shrk_status build_tree_fused(const double* d_sorted, int64_t ns, const ChebParams& prm,
                                    FlatTree& f, NodeF32** nf, float** panel, const int** d_nn,
                                    cudaStream_t s) {
  const int64_t cap = std::max<int64_t>(2 * ns, 2);
  const int n = prm.n;
  ChebConsts k;
  k.n = n;
  for (int j = 0; j < n; ++j) {
    k.sm1[j] = std::cos((double)j * M_PI / (double)(n - 1));
    const double sign = (j % 2 == 0) ? 1.0 : -1.0;
    k.lam[j] = (j == 0 || j == n - 1) ? 0.5 * sign : sign;
  }
  constexpr int NLEV = MAX_TREE_DEPTH + 2;
  void* p64 = nullptr;
  void* p32 = nullptr;
  SHRK_TRY(scratch_get(25, sizeof(int64_t) * 2 * (size_t)cap, &p64));
  SHRK_TRY(scratch_get(26, sizeof(int32_t) * (8 * (size_t)cap + (size_t)ns + 2 + 8 + 2 * NLEV),
                       &p32));
  BuildArrays b;
  b.blo = (int64_t*)p64;
  b.bhi = b.blo + cap;
  b.lc = (int32_t*)p32;
  b.rc = b.lc + cap;
  b.size = b.rc + cap;
  b.pre = b.size + cap;
  b.counter = (int*)(b.pre + cap);
  b.levels = b.counter + 8;
  b.parent = b.levels + 2 * NLEV;
  b.arrive = b.parent + cap;
  b.dep = b.arrive + cap;
  b.rturn = b.dep + cap;
  b.leafpre = b.rturn + cap;
  void* q = nullptr;
  SHRK_TRY(scratch_get(TREE_SLOTS + 0, sizeof(double) * 3 * (size_t)cap, &q));
  f.lo = (double*)q;
  f.hi = f.lo + cap;
  f.accept_hw = f.hi + cap;
  SHRK_TRY(scratch_get(TREE_SLOTS + 1, sizeof(int64_t) * 2 * (size_t)cap, &q));
  f.lo_idx = (int64_t*)q;
  f.hi_idx = f.lo_idx + cap;
  SHRK_TRY(scratch_get(TREE_SLOTS + 2, sizeof(int32_t) * (size_t)cap, &q));
  f.right = (int32_t*)q;
  SHRK_TRY(scratch_get(TREE_SLOTS + 3, sizeof(double) * 2 * (size_t)cap * n, &q));
  f.nodes = (double*)q;
  f.w = f.nodes + (size_t)cap * n;
  NodeF32* mirror = nullptr;
  float* mpanel = nullptr;
  if (prm.f32) {
    SHRK_TRY(scratch_get(TREE_SLOTS + 4, sizeof(NodeF32) * (size_t)cap, &q));
    mirror = (NodeF32*)q;
    SHRK_TRY(scratch_get(TREE_SLOTS + 5, sizeof(float) * 2 * (size_t)cap * n, &q));
    mpanel = (float*)q;
  }
  if (ns <= TINY_NS && prm.leaf_cap >= 1) {
    // all the shared memory a CTA may have: what the arrays leave over holds
    // the nodes and weights of a small enough tree
    static std::atomic<int> optin[64];
    int dev = 0;
    SHRK_CUDA(cudaGetDevice(&dev));
    int smem = dev >= 0 && dev < 64 ? optin[dev].load() : 0;
    if (smem == 0) {
      SHRK_CUDA(cudaDeviceGetAttribute(&smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
      SHRK_CUDA(cudaFuncSetAttribute(tree_tiny_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     smem));
      if (dev >= 0 && dev < 64) optin[dev] = smem;
    }
    if ((size_t)smem < tiny_smem_bytes(ns)) {
      set_error("chebcode: the device has too little shared memory per block");
      return SHRK_ECUDA;
    }
    LaunchScope ls("cheb_build", s);
    tree_tiny_kernel<<<1, TINY_NT, (size_t)smem, s>>>(
        d_sorted, ns, (int64_t)prm.leaf_cap, f, k, prm.theta * prm.theta, mirror, mpanel,
        b.counter);
    SHRK_CUDA(cudaGetLastError());
  } else {
    {
      LaunchScope ls("cheb_build", s);
      tree_topology_cta_kernel<<<1, TOPO_NT, 0, s>>>(d_sorted, b, ns, (int64_t)prm.leaf_cap, f,
                                                     k, prm.theta * prm.theta);
      SHRK_CUDA(cudaGetLastError());
    }
    {
      LaunchScope ls("cheb_build_weights", s);
      tree_p2m_grid_kernel<<<sm_count() * 4, WEIGHT_NT, 0, s>>>(d_sorted, b, f, f.w, k, mirror,
                                                                mpanel);
      SHRK_CUDA(cudaGetLastError());
    }
  }
  *nf = mirror;
  *panel = mpanel;
  *d_nn = b.counter;  // the node count, left on the device by the build
  return SHRK_OK;
}

shrk_status chebcode_points(const double* d_q, int64_t nq, const double* d_sorted_src, int64_t ns,
                            double eta, const ChebParams& prm, const Epilogue& epi,
                            cudaStream_t s) {
  if (nq <= 0 || ns <= 0) return SHRK_OK;
  if (prm.n < 2 || prm.n > MAX_N) {
    set_error("chebcode: interpolation order must be in [2, 16]");
    return SHRK_EINVAL;
  }
  TreeBuild tb;
  NodeF32* fused_nf = nullptr;
  float* fused_panel = nullptr;
  const int* d_nn = nullptr;
  const bool fused = fused_build_ok(ns, prm);
  if (fused)
    SHRK_TRY(build_tree_fused(d_sorted_src, ns, prm, tb.f, &fused_nf, &fused_panel, &d_nn, s));
  else SHRK_TRY(build_tree_gpu(d_sorted_src, ns, prm, tb, s));
  const FlatTree& f = tb.f;
  const int nn = tb.nn;
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
  a.nn_dev = d_nn;
  a.nn_host = nn;
  // A warp (or a thread) per query, 128 threads per CTA; the CTAs copy the
  // tree's node records into shared memory when there are few enough CTAs
  // that the copies cost less than the L2 round trips they save.
  const bool warp = nq <= CHEB_WARP_NQ;
  const unsigned ctas = (unsigned)(((warp ? nq * 32 : nq) + 127) / 128);
  a.stage_bytes = ctas <= (unsigned)(8 * sm_count()) ? CHEB_STAGE_BYTES : 0;
  const size_t smem = (size_t)a.stage_bytes;
  if (!prm.f32) {
    a.t.lo = f.lo;
    a.t.hi = f.hi;
    a.t.accept_hw = f.accept_hw;
    a.t.lo_idx = f.lo_idx;
    a.t.hi_idx = f.hi_idx;
    a.t.right = f.right;
    a.t.nodes = f.nodes;
    a.t.w = f.w;
    LaunchScope ls("cheb_eval_f64", s);
    if (warp) cheb_eval_f64<true><<<ctas, 128, smem, s>>>(a);
    else cheb_eval_f64<false><<<ctas, 128, smem, s>>>(a);
    SHRK_CUDA(cudaGetLastError());
  } else {
    NodeF32* nf = fused_nf;
    float* panel = fused_panel;
    if (!fused) {
      void* q = nullptr;
      SHRK_TRY(scratch_get(TREE_SLOTS + 4, sizeof(NodeF32) * (size_t)nn, &q));
      nf = (NodeF32*)q;
      SHRK_TRY(scratch_get(TREE_SLOTS + 5, sizeof(float) * 2 * (size_t)nn * prm.n, &q));
      panel = (float*)q;
      LaunchScope ls("cheb_build", s);
      tree_f32_kernel<<<blocks_for(nn, 256), 256, 0, s>>>(f, nn, prm.n, nf, panel);
      SHRK_CUDA(cudaGetLastError());
    }
    a.nf = nf;
    a.panel = panel;
    LaunchScope ls("cheb_eval_f32", s);
    if (warp) cheb_eval_f32<true><<<ctas, 128, smem, s>>>(a);
    else cheb_eval_f32<false><<<ctas, 128, smem, s>>>(a);
    SHRK_CUDA(cudaGetLastError());
  }
  return SHRK_OK;
}

shrk_status chebcode_adjoint(const double* d_ev, int64_t p, double eta, const double* d_gre,
                             const double* d_gim, const ChebParams& prm, double* d_grad,
                             cudaStream_t s) {
  if (p <= 0) return SHRK_OK;
  if (prm.n < 2 || prm.n > MAX_N) {
    set_error("chebcode: interpolation order must be in [2, 16]");
    return SHRK_EINVAL;
  }
  const double* ds = nullptr;
  const int* perm = nullptr;
  SHRK_TRY(sorted_sources_perm(d_ev, p, &ds, &perm, s));
  // Scratch slot 30: the charges in sorted order; slot 31: their node weights.
  void* q = nullptr;
  SHRK_TRY(scratch_get(30, sizeof(double) * 2 * (size_t)p, &q));
  double* cw = (double*)q;
  double* cv = cw + p;
  {
    LaunchScope ls("cheb_build", s);
    gather_charges_kernel<<<blocks_for(p, 256), 256, 0, s>>>(d_gre, d_gim, perm, p, cw, cv);
    SHRK_CUDA(cudaGetLastError());
  }
  TreeBuild tb;
  SHRK_TRY(build_tree_gpu(ds, p, prm, tb, s));
  SHRK_TRY(scratch_get(31, sizeof(double) * 2 * (size_t)tb.nn * prm.n, &q));
  double* ww = (double*)q;
  double* wv = ww + (size_t)tb.nn * prm.n;
  SHRK_TRY(tree_weights(tb, ds, cw, ww, s));
  SHRK_TRY(tree_weights(tb, ds, cv, wv, s));
  AdjEvalArgs a;
  a.x = d_ev;
  a.w = d_gre;
  a.v = d_gim;
  a.p = p;
  a.sorted = ds;
  a.cw = cw;
  a.cv = cv;
  a.eta = eta;
  a.t.lo = tb.f.lo;
  a.t.hi = tb.f.hi;
  a.t.accept_hw = tb.f.accept_hw;
  a.t.lo_idx = tb.f.lo_idx;
  a.t.hi_idx = tb.f.hi_idx;
  a.t.right = tb.f.right;
  a.t.nodes = tb.f.nodes;
  a.t.w = tb.f.w;
  a.t.n = prm.n;
  a.ww = ww;
  a.wv = wv;
  a.grad = d_grad;
  a.err = device_error_word();
  LaunchScope ls("cheb_adjoint", s);
  cheb_adjoint_f64<<<blocks_for(p, 128), 128, 0, s>>>(a);
  SHRK_CUDA(cudaGetLastError());
  return SHRK_OK;
}

shrk_status chebcode_evaluate_many(const double* d_ev, int64_t p, const double* d_etas,
                                   int64_t n_eta, const ChebParams& prm, double* d_re,
                                   double* d_im, cudaStream_t s) {
  if (p <= 0 || n_eta <= 0) return SHRK_OK;
  if (prm.n < 2 || prm.n > MAX_N) {
    set_error("chebcode: interpolation order must be in [2, 16]");
    return SHRK_EINVAL;
  }
  const double* ds = nullptr;
  double first = 0.0, last = 0.0;
  SHRK_TRY(sorted_sources(d_ev, p, &ds, &first, &last, s));
  TreeBuild tb;
  SHRK_TRY(build_tree_gpu(ds, p, prm, tb, s));
  ManyArgs a;
  a.x = d_ev;
  a.p = p;
  a.sorted = ds;
  a.etas = d_etas;
  a.n_eta = n_eta;
  a.t.lo = tb.f.lo;
  a.t.hi = tb.f.hi;
  a.t.accept_hw = tb.f.accept_hw;
  a.t.lo_idx = tb.f.lo_idx;
  a.t.hi_idx = tb.f.hi_idx;
  a.t.right = tb.f.right;
  a.t.nodes = tb.f.nodes;
  a.t.w = tb.f.w;
  a.t.n = prm.n;
  a.theta_sq = prm.theta * prm.theta;
  a.out_re = d_re;
  a.out_im = d_im;
  a.err = device_error_word();
  LaunchScope ls("cheb_eval_x2", s);
  cheb_eval_x2<<<blocks_for(p * ((n_eta + 1) / 2), 128), 128, 0, s>>>(a);
  SHRK_CUDA(cudaGetLastError());
  return SHRK_OK;
}

}  // namespace shrk
