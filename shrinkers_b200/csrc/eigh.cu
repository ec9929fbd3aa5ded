// Dense symmetric eigendecomposition and FP64 GEMM on sm_100a, for the matrix
// front-end (src/pipeline/mod.rs:502-585 symmetric_eigh; the reference runs a
// cyclic Jacobi iteration, and its docs name LAPACK's dsyevd as the fast
// path).  Written for the GPU instead of restating Jacobi:
//
//   1. tridiagonalisation  Householder reflections H_j = I - beta_j v_j v_j^T,
//                          one cooperative persistent kernel: every warp owns
//                          columns of the (full, symmetric, column-major)
//                          trailing matrix; per column j one grid barrier
//                          after the symmetric product p = beta A22 v and one
//                          after the rank-2 update A22 -= v w^T + w v^T,
//                          w = p - (beta/2)(p^T v) v.  The reflectors stay in
//                          the strict lower part of A (v_{j+1} and beta_j
//                          aside), as in LAPACK's dsytrd.
//   2. eigenvalues         the tridiagonal T splits where an off-diagonal is
//                          negligible; each eigenvalue of each unreduced block
//                          by 32-way multisection on Sturm counts, one warp
//                          per eigenvalue.
//   3. eigenvectors of T   inverse iteration (LU with partial pivoting,
//                          three solves from a fixed pseudo-random start),
//                          one thread per cluster of eigenvalues closer than
//                          CLUSTER_TOL ||T||, modified Gram-Schmidt inside a
//                          cluster; then one Newton-Schulz step
//                          Z <- Z (3I - Z^T Z)/2 on the whole basis, which
//                          takes the remaining O(eps ||T|| / gap) overlaps
//                          of close eigenvectors to rounding level.
//   4. back-transformation U = H_0 ... H_{p-3} Z in blocks of NB reflectors,
//                          each (I - Y T Y^T) in compact WY form (three
//                          GEMMs).
//
// The GEMM (dgemm) is a plain FP64 tiled kernel: 64 x 64 outputs per CTA of
// 256 threads, 4 x 4 per thread, k staged 16 at a time in shared memory.
#include "common.cuh"
#include "internal.h"

#include <cooperative_groups.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <numeric>
#include <string>
#include <vector>

namespace shrk {

namespace cg = cooperative_groups;

namespace {

// ------------------------------------------------------------------ GEMM --
constexpr int GT = 64;   // output tile
constexpr int GK = 16;   // k per shared-memory stage

// Split-K: CTA z of gridDim.z sums k in [z kz, (z+1) kz) and, when the grid
// has several, writes alpha times its partial product to its own m x n slab
// of C (ldc = m, beta = 0); dgemm then adds the slabs in a fixed order.
template <bool TA, bool TB>
__global__ void __launch_bounds__(256) dgemm_kernel(int m, int n, int k, int kz, double alpha,
                                                    const double* __restrict__ A, int64_t lda,
                                                    const double* __restrict__ B, int64_t ldb,
                                                    double beta, double* __restrict__ C,
                                                    int64_t ldc, int lower) {
  if (lower && blockIdx.y > blockIdx.x) return;  // a tile wholly above the diagonal
  const int kb = blockIdx.z * kz, ke = min(k, kb + kz);
  if (gridDim.z > 1) C += (int64_t)blockIdx.z * m * n;
  __shared__ double As[GK][GT + 1];  // As[kk][i] = op(A)[i0 + i, k0 + kk]
  __shared__ double Bs[GK][GT + 1];  // Bs[kk][j] = op(B)[k0 + kk, j0 + j]
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  const int i0 = blockIdx.x * GT, j0 = blockIdx.y * GT;
  double acc[4][4];
#pragma unroll
  for (int r = 0; r < 4; ++r)
#pragma unroll
    for (int c = 0; c < 4; ++c) acc[r][c] = 0.0;
  for (int k0 = kb; k0 < ke; k0 += GK) {
#pragma unroll
    for (int it = 0; it < 4; ++it) {
      const int t = threadIdx.x + it * 256;
      int i, kk;
      if (!TA) { i = t & 63; kk = t >> 6; }   // A(i, kk) contiguous in i
      else { kk = t & 15; i = t >> 4; }       // A(kk, i) contiguous in kk
      const int gi = i0 + i, gk = k0 + kk;
      double v = 0.0;
      if (gi < m && gk < ke) v = !TA ? A[gi + (int64_t)gk * lda] : A[gk + (int64_t)gi * lda];
      As[kk][i] = v;
    }
#pragma unroll
    for (int it = 0; it < 4; ++it) {
      const int t = threadIdx.x + it * 256;
      int j, kk;
      if (!TB) { kk = t & 15; j = t >> 4; }   // B(kk, j) contiguous in kk
      else { j = t & 63; kk = t >> 6; }       // B(j, kk) contiguous in j
      const int gj = j0 + j, gk = k0 + kk;
      double v = 0.0;
      if (gj < n && gk < ke) v = !TB ? B[gk + (int64_t)gj * ldb] : B[gj + (int64_t)gk * ldb];
      Bs[kk][j] = v;
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < GK; ++kk) {
      double a[4], b[4];
#pragma unroll
      for (int r = 0; r < 4; ++r) a[r] = As[kk][tx + 16 * r];
#pragma unroll
      for (int c = 0; c < 4; ++c) b[c] = Bs[kk][ty + 16 * c];
#pragma unroll
      for (int r = 0; r < 4; ++r)
#pragma unroll
        for (int c = 0; c < 4; ++c) acc[r][c] = fma(a[r], b[c], acc[r][c]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int c = 0; c < 4; ++c) {
    const int gj = j0 + ty + 16 * c;
    if (gj >= n) continue;
#pragma unroll
    for (int r = 0; r < 4; ++r) {
      const int gi = i0 + tx + 16 * r;
      if (gi >= m) continue;
      double* cp = C + gi + (int64_t)gj * ldc;
      *cp = beta == 0.0 ? alpha * acc[r][c] : fma(alpha, acc[r][c], beta * *cp);
    }
  }
}

// The large-problem form: 128 x 128 outputs per CTA of 256 threads on the
// FP64 tensor path (mma.sync m8n8k4 .f64; tcgen05 has no FP64 kind): each
// warp owns a 32 x 64 block, 4 x 8 tiles of 8 x 8 with two accumulators a
// lane; k staged 8 at a time through shared memory, two stages in flight
// (the next stage's global loads are issued before this stage's MMAs).  Rows
// of the staged tiles are 136 doubles apart (16 words mod 32 banks), so a
// fragment load -- 4 k rows x 8 consecutive entries -- takes the two
// wavefronts a 64-bit warp load needs and no more.
constexpr int GT2 = 128, GK2 = 8, GP2 = GT2 + 8;

// D = A B + D for one 8 x 8 x 4 FP64 tile: lane l holds A[l/4][l%4],
// B[l%4][l/4] and D[l/4][2(l%4) + {0, 1}].
__device__ __forceinline__ void mma_f64(double& d0, double& d1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
               : "+d"(d0), "+d"(d1)
               : "d"(a), "d"(b));
}

template <bool TA, bool TB>
__global__ void __launch_bounds__(256, 1) dgemm_big_kernel(int m, int n, int k, int kz,
                                                           double alpha,
                                                           const double* __restrict__ A,
                                                           int64_t lda,
                                                           const double* __restrict__ B,
                                                           int64_t ldb, double beta,
                                                           double* __restrict__ C,
                                                           int64_t ldc, int lower) {
  if (lower && blockIdx.y > blockIdx.x) return;  // a tile wholly above the diagonal
  __shared__ double As[2][GK2][GP2];  // As[kk][i] = op(A)[i0 + i, k0 + kk]
  __shared__ double Bs[2][GK2][GP2];  // Bs[kk][j] = op(B)[k0 + kk, j0 + j]
  const int kb = blockIdx.z * kz, ke = min(k, kb + kz);
  if (gridDim.z > 1) C += (int64_t)blockIdx.z * m * n;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int wi = (warp & 3) * 32, wj = (warp >> 2) * 64;  // the warp's block
  const int fr = lane >> 2, fk = lane & 3;                 // fragment row / k
  const int i0 = blockIdx.x * GT2, j0 = blockIdx.y * GT2;
  double acc[4][8][2];
#pragma unroll
  for (int r = 0; r < 4; ++r)
#pragma unroll
    for (int c = 0; c < 8; ++c) acc[r][c][0] = acc[r][c][1] = 0.0;
  double ra[4], rb[4];
  auto fetch = [&](int k0) {
#pragma unroll
    for (int it = 0; it < 4; ++it) {
      const int t = threadIdx.x + it * 256;
      int i, kk;
      if (!TA) { i = t & 127; kk = t >> 7; }  // A(i, kk) contiguous in i
      else { kk = t & 7; i = t >> 3; }        // A(kk, i) contiguous in kk
      const int gi = i0 + i, gk = k0 + kk;
      ra[it] = (gi < m && gk < ke) ? (!TA ? A[gi + (int64_t)gk * lda] : A[gk + (int64_t)gi * lda])
                                   : 0.0;
    }
#pragma unroll
    for (int it = 0; it < 4; ++it) {
      const int t = threadIdx.x + it * 256;
      int j, kk;
      if (!TB) { kk = t & 7; j = t >> 3; }    // B(kk, j) contiguous in kk
      else { j = t & 127; kk = t >> 7; }      // B(j, kk) contiguous in j
      const int gj = j0 + j, gk = k0 + kk;
      rb[it] = (gj < n && gk < ke) ? (!TB ? B[gk + (int64_t)gj * ldb] : B[gj + (int64_t)gk * ldb])
                                   : 0.0;
    }
  };
  auto stash = [&](int buf) {
#pragma unroll
    for (int it = 0; it < 4; ++it) {
      const int t = threadIdx.x + it * 256;
      if (!TA) As[buf][t >> 7][t & 127] = ra[it];
      else As[buf][t & 7][t >> 3] = ra[it];
      if (!TB) Bs[buf][t & 7][t >> 3] = rb[it];
      else Bs[buf][t >> 7][t & 127] = rb[it];
    }
  };
  fetch(kb);
  stash(0);
  __syncthreads();
  int buf = 0;
  for (int k0 = kb; k0 < ke; k0 += GK2) {
    const bool more = k0 + GK2 < ke;
    if (more) fetch(k0 + GK2);
#pragma unroll
    for (int k4 = 0; k4 < GK2; k4 += 4) {
      double a[4], b[8];
#pragma unroll
      for (int r = 0; r < 4; ++r) a[r] = As[buf][k4 + fk][wi + 8 * r + fr];
#pragma unroll
      for (int c = 0; c < 8; ++c) b[c] = Bs[buf][k4 + fk][wj + 8 * c + fr];
#pragma unroll
      for (int r = 0; r < 4; ++r)
#pragma unroll
        for (int c = 0; c < 8; ++c) mma_f64(acc[r][c][0], acc[r][c][1], a[r], b[c]);
    }
    if (more) {
      stash(buf ^ 1);
      __syncthreads();
      buf ^= 1;
    }
  }
#pragma unroll
  for (int c = 0; c < 8; ++c) {
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int gj = j0 + wj + 8 * c + 2 * fk + h;
      if (gj >= n) continue;
#pragma unroll
      for (int r = 0; r < 4; ++r) {
        const int gi = i0 + wi + 8 * r + fr;
        if (gi >= m) continue;
        double* cp = C + gi + (int64_t)gj * ldc;
        *cp = beta == 0.0 ? alpha * acc[r][c][h] : fma(alpha, acc[r][c][h], beta * *cp);
      }
    }
  }
}

// C = sum_z slab[z] + beta C, the split-K slabs added in order.
__global__ void dgemm_reduce_kernel(const double* __restrict__ ws, int splits, int m, int n,
                                    double beta, double* __restrict__ C, int64_t ldc) {
  const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (int64_t)m * n) return;
  const int64_t i = idx % m, j = idx / m;
  double t = 0.0;
  for (int z = 0; z < splits; ++z) t += ws[(int64_t)z * m * n + idx];
  double* cp = C + i + j * ldc;
  *cp = beta == 0.0 ? t : t + beta * *cp;
}

// -------------------------------------------------------- tridiagonalise --
struct TriArgs {
  double* A;        // p x p column-major, symmetric (both triangles)
  int64_t p;
  double* d;        // [p] diagonal of T
  double* e;        // [p] off-diagonal of T (e[j] couples j and j+1)
  double* vhead;    // [p] first entry v_{j+1} of reflector j
  double* beta;     // [p] beta_j (0: no reflection)
  double* pv;       // [p] p = beta A22 v
  double* part;     // [gridDim.x] per-block partial sums of p^T v
  double* scal;     // [2] norm^2 and first entry of the next column below the diagonal
};

constexpr int TRI_NT = 512;

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Norm^2 and first entry of A[c+1 .. p-1, c] by one warp; lane 0 writes them
// (and the final diagonal entry d[c]).
__device__ __forceinline__ void column_tail(const TriArgs& a, int64_t c, int lane) {
  const int64_t p = a.p;
  const double* col = a.A + c * p;
  double s = 0.0;
  for (int64_t k = c + 1 + lane; k < p; k += 32) s += col[k] * col[k];
  s = warp_sum(s);
  if (lane == 0) {
    a.scal[0] = s;
    a.scal[1] = c + 1 < p ? col[c + 1] : 0.0;
    a.d[c] = col[c];
  }
}

__global__ void __launch_bounds__(TRI_NT, 1) tridiag_kernel(const TriArgs a) {
  cg::grid_group grid = cg::this_grid();
  __shared__ double s_red[TRI_NT / 32];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  constexpr int WPB = TRI_NT / 32;
  const int64_t gw = (int64_t)blockIdx.x * WPB + wib;  // global warp: owns columns gw mod nw
  const int64_t nw = (int64_t)gridDim.x * WPB;
  const int64_t p = a.p;
  double* A = a.A;
  if (gw == 0) column_tail(a, 0, lane);
  grid.sync();
  for (int64_t j = 0; j + 2 < p; ++j) {
    // the reflector of column j, from the norm its owner left in scal
    const double norm2 = a.scal[0], x0 = a.scal[1];
    const double sig = norm2 - x0 * x0;
    double beta = 0.0, v0 = x0;
    if (sig > 0.0) {
      const double nrm = sqrt(norm2);
      const double alpha = x0 >= 0.0 ? -nrm : nrm;
      v0 = x0 - alpha;
      beta = 2.0 / (sig + v0 * v0);
      if (gw == 0 && lane == 0) a.e[j] = alpha;
    } else if (gw == 0 && lane == 0) {
      a.e[j] = x0;  // already reduced: H_j = I
    }
    if (gw == 0 && lane == 0) {
      a.vhead[j] = v0;
      a.beta[j] = beta;
    }
    const double* vcol = A + j * p;  // v_k = vcol[k] for k >= j + 2
    const int64_t k0 = j + 1;
    // (1) p = beta A22 v over the owned columns, and p^T v
    double dot = 0.0;
    if (beta != 0.0) {
      int64_t c = k0 + ((gw - k0) % nw + nw) % nw;
      for (; c < p; c += nw) {
        const double* col = A + c * p;
        double s = 0.0;
        for (int64_t k = k0 + lane; k < p; k += 32) {
          const double vk = k == k0 ? v0 : vcol[k];
          s = fma(col[k], vk, s);
        }
        s = warp_sum(s) * beta;
        if (lane == 0) a.pv[c] = s;
        dot = fma(s, c == k0 ? v0 : vcol[c], dot);
      }
    }
    if (lane == 0) s_red[wib] = dot;
    __syncthreads();
    if (threadIdx.x == 0) {
      double t = 0.0;
      for (int w = 0; w < WPB; ++w) t += s_red[w];
      a.part[blockIdx.x] = t;
    }
    grid.sync();
    // (2) A22 -= v w^T + w v^T, w = p - (beta/2)(p^T v) v, by owned columns;
    // the owner of column j+1 then measures the next column
    if (beta != 0.0) {
      double g = 0.0;
      for (int b = lane; b < (int)gridDim.x; b += 32) g += a.part[b];
      const double K = 0.5 * beta * warp_sum(g);
      int64_t c = k0 + ((gw - k0) % nw + nw) % nw;
      for (; c < p; c += nw) {
        double* col = A + c * p;
        const double vc = c == k0 ? v0 : vcol[c];
        const double wc = a.pv[c] - K * vc;
        for (int64_t k = k0 + lane; k < p; k += 32) {
          const double vk = k == k0 ? v0 : vcol[k];
          const double wk = a.pv[k] - K * vk;
          col[k] = col[k] - (vk * wc + wk * vc);
        }
      }
    }
    if (gw == k0 % nw) {
      __syncwarp();
      column_tail(a, k0, lane);
    }
    grid.sync();
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    if (p >= 2) a.e[p - 2] = a.scal[1];
    a.d[p - 1] = A[(p - 1) + (p - 1) * p];
    if (p == 1) a.d[0] = A[0];
  }
}


// The same reduction with ONE grid barrier per column.  Phase j applies
// reflector j to the trailing columns and, in the same pass over each
// column, forms the next product p_{j+1} = beta_{j+1} A^{(j+1)} v_{j+1}.
// That needs v_{j+1} at the start of the phase: every CTA derives it itself
// from the stale column j+1 and the previous phase's p_j (w = p_j - K v_j),
// bit-identically in every CTA (same reads, same reduction order), into its
// own buffer.  Column j+1 is then never written: reflector j+1 goes to row
// j+1 of the upper triangle (a part no later phase reads), and only rows
// >= j+2 of the trailing columns are updated.  p and the partial sums of
// p^T v alternate between two buffers.
struct Tri1Args {
  double* A;       // p x p column-major, symmetric (both triangles)
  int64_t p;
  double* d;
  double* e;
  double* vhead;   // [p] reflector heads
  double* beta;    // [p]
  double* pv;      // [2][p]
  double* part;    // [2][gridDim.x]
  double* vb;      // [gridDim.x][2][p] per-CTA reflector copies (global form)
  double* wb;      // [gridDim.x][p] per-CTA w = p_j - K v_j (global form)
};

// The per-CTA vectors (two reflectors and w, 3 p doubles) live in shared
// memory up to this many bytes, else in global memory.
constexpr size_t TRI1_SMEM_MAX = 200 * 1024;

__device__ __forceinline__ double block_sum(double v, double* red) {
  v = warp_sum(v);
  __syncthreads();  // red may still be read from the previous call
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  double t = 0.0;
  const int nw = blockDim.x >> 5;
  for (int w = 0; w < nw; ++w) t += red[w];
  return t;
}

// Reflector of x = v[k0 .. p): on return v[k0] holds the head x0 - alpha and
// the rest is x; beta = 0 (and alpha = x0) when x is already reduced.
__device__ __forceinline__ void make_reflector(double* v, int64_t k0, int64_t p, double* red,
                                               double& beta, double& alpha) {
  double s = 0.0;
  for (int64_t k = k0 + threadIdx.x; k < p; k += blockDim.x) s += v[k] * v[k];
  const double norm2 = block_sum(s, red);
  const double x0 = v[k0];
  const double sig = norm2 - x0 * x0;
  double head = x0;
  beta = 0.0;
  alpha = x0;
  if (sig > 0.0) {
    const double nrm = sqrt(norm2);
    alpha = x0 >= 0.0 ? -nrm : nrm;
    head = x0 - alpha;
    beta = 2.0 / (sig + head * head);
  }
  __syncthreads();  // every thread has read v[k0]
  if (threadIdx.x == 0) v[k0] = head;
  __syncthreads();
}

template <bool SH, int R = 16>
__global__ void __launch_bounds__(TRI_NT, 1) tridiag1_kernel(const Tri1Args a) {
  cg::grid_group grid = cg::this_grid();
  __shared__ double red[TRI_NT / 32];
  extern __shared__ double tri_sh[];
  const int lane = threadIdx.x & 31;
  constexpr int WPB = TRI_NT / 32;
  const int64_t gw = (int64_t)blockIdx.x * WPB + (threadIdx.x >> 5);
  const int64_t nw = (int64_t)gridDim.x * WPB;
  const int64_t G = gridDim.x;
  const int64_t p = a.p;
  double* A = a.A;
  const bool lead = blockIdx.x == 0;
  if (p < 3) {
    if (lead && threadIdx.x == 0) {
      a.d[0] = A[0];
      if (p == 2) {
        a.e[0] = A[1];
        a.d[1] = A[3];
      }
    }
    return;
  }
  // the reflectors v_j, v_{j+1} and w_j = p_j - K v_j for the rows >= j+2,
  // read by every warp of the CTA for every trailing column
  double* vb = SH ? tri_sh : a.vb + (int64_t)blockIdx.x * 2 * p;
  double* wv = SH ? tri_sh + 2 * p : a.wb + (int64_t)blockIdx.x * p;
  // prologue: reflector 0 from column 0, p_0 over the columns c >= 1
  double* vcur = vb;
  for (int64_t k = 1 + threadIdx.x; k < p; k += blockDim.x) vcur[k] = A[k];
  double bcur = 0.0, alpha = 0.0;
  make_reflector(vcur, 1, p, red, bcur, alpha);
  if (lead) {
    if (threadIdx.x == 0) {
      a.d[0] = A[0];
      a.e[0] = alpha;
      a.vhead[0] = vcur[1];
      a.beta[0] = bcur;
    }
    for (int64_t k = 2 + threadIdx.x; k < p; k += blockDim.x) A[k * p] = vcur[k];  // row 0
  }
  {
    double dot = 0.0;
    if (bcur != 0.0)
      for (int64_t c = 1 + ((gw - 1) % nw + nw) % nw; c < p; c += nw) {
        const double* col = A + c * p;
        double s = 0.0;
        for (int64_t k = 1 + lane; k < p; k += 32) s = fma(col[k], vcur[k], s);
        s = warp_sum(s) * bcur;
        if (lane == 0) a.pv[c] = s;
        dot = fma(s, vcur[c], dot);
      }
    const double t = block_sum(lane == 0 ? dot : 0.0, red);
    if (threadIdx.x == 0) a.part[blockIdx.x] = t;
  }
  grid.sync();
  for (int64_t j = 0; j + 2 < p; ++j) {
    const int par = (int)(j & 1), nxt = par ^ 1;
    vcur = vb + par * p;
    double* vnext = vb + nxt * p;
    const double* pj = a.pv + par * p;
    const double g = block_sum(threadIdx.x < G ? a.part[par * G + threadIdx.x] : 0.0, red);
    const double K = 0.5 * bcur * g;
    const bool upd = bcur != 0.0;
    const int64_t k1 = j + 1, k2 = j + 2;
    const double vj1 = vcur[k1], wj1 = upd ? pj[k1] - K * vj1 : 0.0;
    // column j+1 of A^{(j+1)}, rows >= j+2, and its diagonal entry
    {
      const double* colj1 = A + k1 * p;
      const int64_t bd = blockDim.x;
      int64_t k = k2 + threadIdx.x;
      for (; k + 3 * bd < p; k += 4 * bd) {
        double av[4], vv[4], qv[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          av[u] = colj1[k + u * bd];
          vv[u] = vcur[k + u * bd];
          qv[u] = pj[k + u * bd];
        }
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          const double wk = upd ? qv[u] - K * vv[u] : 0.0;
          wv[k + u * bd] = wk;
          vnext[k + u * bd] = av[u] - (vv[u] * wj1 + wk * vj1);
        }
      }
      for (; k < p; k += bd) {
        const double vk = vcur[k], wk = upd ? pj[k] - K * vk : 0.0;
        wv[k] = wk;
        vnext[k] = colj1[k] - (vk * wj1 + wk * vj1);
      }
    }
    const double dnew = A[k1 + k1 * p] - 2.0 * vj1 * wj1;
    double bnext = 0.0;
    if (k1 + 2 < p) {
      make_reflector(vnext, k2, p, red, bnext, alpha);
      if (lead) {
        if (threadIdx.x == 0) {
          a.d[k1] = dnew;
          a.e[k1] = alpha;
          a.vhead[k1] = vnext[k2];
          a.beta[k1] = bnext;
        }
        for (int64_t k = k2 + 1 + threadIdx.x; k < p; k += blockDim.x) A[k1 + k * p] = vnext[k];
      }
    } else {  // the last 2 x 2 block: no further reflector
      __syncthreads();
      if (lead && threadIdx.x == 0) {
        a.d[k1] = dnew;
        a.e[k1] = vnext[k2];
      }
    }
    // trailing columns: update rows >= j+2 and form p_{j+1} from the new values
    double dot = 0.0;
    for (int64_t c = k2 + ((gw - k2) % nw + nw) % nw; c < p; c += nw) {
      double* col = A + c * p;
      const double vc = vcur[c], wc = wv[c];
      double s = 0.0;
      int64_t k = k2 + lane;
      if constexpr (SH) {
        // R rows per lane per step (one L2 round trip), the column's loads
        // issued before any store; the vectors come from shared memory; the
        // ragged end is one predicated step
        for (; k < p; k += 32 * R) {
          double av[R];
#pragma unroll
          for (int u = 0; u < R; ++u) av[u] = k + 32 * u < p ? col[k + 32 * u] : 0.0;
#pragma unroll
          for (int u = 0; u < R; ++u) {
            const int64_t kk = k + 32 * u;
            if (kk < p) {
              const double x = av[u] - (vcur[kk] * wc + wv[kk] * vc);
              col[kk] = x;
              s = fma(x, vnext[kk], s);
            }
          }
        }
      }
      // eight rows per lane per step, every load issued before any store
      // (the stores to col could alias the loads for all the compiler knows)
      for (; k + 224 < p; k += 256) {
        double av[8], vv[8], qv[8], nv[8];
#pragma unroll
        for (int u = 0; u < 8; ++u) {
          av[u] = col[k + 32 * u];
          vv[u] = vcur[k + 32 * u];
          qv[u] = wv[k + 32 * u];
          nv[u] = vnext[k + 32 * u];
        }
#pragma unroll
        for (int u = 0; u < 8; ++u) {
          const double x = av[u] - (vv[u] * wc + qv[u] * vc);
          col[k + 32 * u] = x;
          s = fma(x, nv[u], s);
        }
      }
      for (; k < p; k += 32) {
        const double x = col[k] - (vcur[k] * wc + wv[k] * vc);
        col[k] = x;
        s = fma(x, vnext[k], s);
      }
      s = warp_sum(s) * bnext;
      if (lane == 0 && bnext != 0.0) a.pv[nxt * p + c] = s;
      dot = fma(s, vnext[c], dot);
    }
    const double t = block_sum(lane == 0 ? dot : 0.0, red);
    if (threadIdx.x == 0) a.part[nxt * G + blockIdx.x] = t;
    bcur = bnext;
    grid.sync();
  }
  if (lead && threadIdx.x == 0) a.d[p - 1] = A[(p - 1) + (p - 1) * p];
}

// ------------------------------------------------------------ bisection --
// Slot k: the kloc-th smallest eigenvalue of the unreduced block [b0, b1)
// of T, searched in the block's Gershgorin interval [lo, hi].
struct EigSlot {
  int b0, b1, kloc, pad;
  double lo, hi;
};

// Number of eigenvalues of T[b0:b1) below x: the negative pivots of the
// LDL^T factorisation of T - x I, q_i = (d_i - x) - e_{i-1}^2 / q_{i-1}, a
// pivot smaller than pivmin counting as -pivmin.  q_i is carried as a
// fraction num / den, num_i = (d_i - x) num_{i-1} - e_{i-1}^2 den_{i-1},
// den_i = num_{i-1}, so the chain through the block is one FMA a row
// instead of one division (the count of a 2 048-row block is a chain of
// 2 048 of them); the pair is rescaled by exact powers of two to stay in
// range, and reset to (-pivmin, 1) when |q| falls below pivmin.
__device__ __forceinline__ int sturm(const double* __restrict__ d, const double* __restrict__ e2,
                                     int b0, int b1, double x, double pivmin) {
  double num = d[b0] - x, den = 1.0;
  if (fabs(num) < pivmin) num = -pivmin;
  int cnt = num < 0.0;
  for (int i = b0 + 1; i < b1; ++i) {
    const double nn = fma(d[i] - x, num, -e2[i - 1] * den);
    den = num;
    num = nn;
    const double an = fabs(num), ad = fabs(den);
    if (an < pivmin * ad) {
      num = -pivmin;
      den = 1.0;
    } else {
      const double mx = fmax(an, ad);
      if (mx > 0x1p+256 || mx < 0x1p-256) {
        const double sc = mx > 1.0 ? 0x1p-256 : 0x1p+256;
        num *= sc;
        den *= sc;
      }
    }
    cnt += (num < 0.0) != (den < 0.0);
  }
  return cnt;
}

// G-way multisection, G lanes per eigenvalue (32 / G eigenvalues a warp):
// each step probes G evenly spaced points of the bracket and keeps the
// sub-interval where the Sturm count crosses kloc (log2(G + 1) bits a step).
// A wide G takes fewer steps (latency); a narrow one fewer Sturm counts in
// all (each is a chain of divisions over the block), which is what bounds
// large matrices.  Every lane stays in the loop until its warp is done (the
// shuffles span the warp).
template <int G>
__global__ void __launch_bounds__(256) bisect_kernel(const double* __restrict__ d,
                                                     const double* __restrict__ e2,
                                                     const EigSlot* __restrict__ slots, int n,
                                                     double pivmin, double* __restrict__ lam) {
  const int64_t gt = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int k = (int)(gt / G);
  const int wl = threadIdx.x & 31, lane = wl % G, g0 = wl - lane;
  const unsigned gmask = G == 32 ? 0xffffffffu : (((1u << G) - 1u) << g0);
  EigSlot sl{0, 0, 0, 0, 0.0, 0.0};
  bool done = k >= n;
  if (!done) sl = slots[k];
  double lo = sl.lo, hi = sl.hi;
  const double eps = 2.220446049250313e-16;
  for (int it = 0; it < 64; ++it) {
    if (!done && hi - lo <= 2.0 * eps * fmax(fabs(lo), fabs(hi)) + pivmin) done = true;
    if (__ballot_sync(0xffffffffu, !done) == 0u) break;
    const double x = lo + (hi - lo) * (double)(lane + 1) / (double)(G + 1);
    const bool above = !done && sturm(d, e2, sl.b0, sl.b1, x, pivmin) > sl.kloc;
    const unsigned m = (__ballot_sync(0xffffffffu, above) & gmask) >> g0;
    const int f = __ffs(m);  // first probe above kloc, 1-based (0: none)
    const double xl = __shfl_sync(0xffffffffu, x, g0 + (f == 0 ? G - 1 : (f >= 2 ? f - 2 : 0)));
    const double xh = __shfl_sync(0xffffffffu, x, g0 + (f == 0 ? 0 : f - 1));
    const double nlo = f == 0 ? xl : (f == 1 ? lo : xl);
    const double nhi = f == 0 ? hi : xh;
    if (!done) {
      if (!(nlo > lo || nhi < hi)) done = true;  // no representable progress
      else {
        lo = nlo;
        hi = nhi;
      }
    }
  }
  if (lane == 0 && k < n) lam[k] = 0.5 * (lo + hi);
}

// ------------------------------------------------------ inverse iteration --
// Cluster c: slots [s0, s0 + ns) of the unreduced block [b0, b1).
struct Cluster {
  int s0, ns, b0, b1;
};

// Deterministic start vector entry (hash of slot and row), in [-1, 1).
__device__ __forceinline__ double start_entry(int slot, int i) {
  uint64_t h = (uint64_t)(uint32_t)slot * 0x9E3779B97F4A7C15ull ^ (uint64_t)(uint32_t)i * 0xC2B2AE3D27D4EB4Full;
  h ^= h >> 31;
  h *= 0xBF58476D1CE4E5B9ull;
  h ^= h >> 29;
  return (double)(h >> 11) * (2.0 / 9007199254740992.0) - 1.0;
}

// One thread per cluster, a warp per CTA.  Workspace: the factorisation of
// T - lambda I (U's off-diagonals, reciprocal pivots, multipliers, row
// swaps) and the right-hand side / solution x, rows relative to the block
// start, stored per warp as [row][array][lane] so that a warp's rows are
// one contiguous range (a chunk of rows is one span of memory, prefetched
// into L2 a few chunks ahead of its use).  Each eigenvalue is factored once
// and its three solves replay the elimination with multiplications only.
// Eigenvector of slot s goes to Zt[s + i p] (row s of Z^T) for i in [b0, b1).
constexpr int II_ARRAYS = 6;  // u1, u2, 1/pivot, multiplier, swap, x
constexpr int II_CH = 16;     // rows whose loads are issued together
constexpr int II_AHEAD = 6;   // chunks prefetched ahead

__device__ __forceinline__ void prefetch_rows(const double* base, int r0, int rows) {
  // rows [r0, r0 + rows) of this warp's workspace, one bulk L2 prefetch
  const unsigned bytes = (unsigned)rows * II_ARRAYS * 32 * sizeof(double);
  const double* a = base + (int64_t)r0 * II_ARRAYS * 32;
  asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(a), "r"(bytes) : "memory");
}

constexpr int II_RS = II_ARRAYS * 32;  // doubles per workspace row of a warp
enum { II_U1 = 0, II_U2 = 1, II_RP = 2, II_MU = 3, II_SW = 4, II_X = 5 };

// One elimination step of T - lambda I with partial pivoting: rows i and
// i + 1, where row i holds (diag, sup) after the earlier steps and row i + 1
// is (sub, nd, ns).  r points at row i of this lane's workspace.  Branch
// free (the lanes of a warp pivot differently); one division.
__device__ __forceinline__ void factor_row(double* r, double sub, double nd, double ns,
                                           double small, double rsmall, double& diag,
                                           double& sup) {
  const bool swp = fabs(diag) < fabs(sub);
  const double piv = swp ? sub : diag;
  const double num = swp ? diag : sub;
  const double rinv = 1.0 / piv;
  const double m = piv != 0.0 ? num * rinv : 0.0;
  r[II_U1 * 32] = swp ? nd : sup;
  r[II_U2 * 32] = swp ? ns : 0.0;
  r[II_MU * 32] = m;
  r[II_SW * 32] = swp ? 1.0 : 0.0;
  r[II_RP * 32] = fabs(piv) < small ? (piv < 0.0 ? -rsmall : rsmall) : rinv;
  const double nd2 = swp ? sup - m * nd : nd - m * sup;
  sup = swp ? -m * ns : ns;
  diag = nd2;
}

// The factorisation's row operation on the right-hand side: x(i) is final,
// rhs carries row i + 1 (rn is the old x(i + 1)).
__device__ __forceinline__ void forward_row(double* r, double rn, double m, double sw,
                                            double& rhs) {
  const bool swp = sw != 0.0;
  const double keep = swp ? rn : rhs;
  const double other = swp ? rhs : rn;
  r[II_X * 32] = keep;
  rhs = other - m * keep;
}

__global__ void __launch_bounds__(32) inverse_iteration_kernel(
    const double* __restrict__ d, const double* __restrict__ e, const double* __restrict__ lam,
    const Cluster* __restrict__ cl, int ncl, int64_t p, double tnorm, double* __restrict__ ws,
    double* __restrict__ Zt) {
  const int lane = threadIdx.x;
  const int t = blockIdx.x * 32 + lane;
  if (t >= ncl) return;
  const Cluster c = cl[t];
  double* base = ws + (int64_t)blockIdx.x * p * II_RS;
  double* const wl = base + lane;  // row 0 of this lane
#define W(a, i) wl[(int64_t)(i) * II_RS + (a) * 32]
  // lane 0 prefetches for the warp; rows past p are outside the region
  const bool pf = lane == 0;
  auto ahead = [&](int r0) {
    if (!pf) return;
    const int lo = max(r0, 0);
    const int hi = (int)((int64_t)r0 + II_CH < p ? (int64_t)r0 + II_CH : p);
    if (hi > lo) prefetch_rows(base, lo, hi - lo);
  };
  const int n = c.b1 - c.b0;
  const double small = 2.220446049250313e-16 * tnorm + 1e-300;
  const double rsmall = 1.0 / small;
  const double* db = d + c.b0;
  const double* eb = e + c.b0;
  constexpr int CH = II_CH;
  for (int q = 0; q < c.ns; ++q) {
    const int slot = c.s0 + q;
    const double l = lam[slot];
    // factor T - l I once with partial pivoting (and write the start
    // vector); the three solves replay the elimination on their right-hand
    // sides
    {
      double diag = db[0] - l;
      double sup = n > 1 ? eb[0] : 0.0;
      int i0 = 0;
      for (; i0 + CH + 1 < n; i0 += CH) {  // full chunks: rows i0 + u + 2 < n
        double subv[CH], ndv[CH], nsv[CH];
#pragma unroll
        for (int u = 0; u < CH; ++u) {
          subv[u] = eb[i0 + u];
          ndv[u] = db[i0 + u + 1] - l;
          nsv[u] = eb[i0 + u + 1];
        }
        double* r = &W(0, i0);
#pragma unroll
        for (int u = 0; u < CH; ++u) {
          factor_row(r + u * II_RS, subv[u], ndv[u], nsv[u], small, rsmall, diag, sup);
          r[u * II_RS + II_X * 32] = start_entry(slot, i0 + u);
        }
      }
      for (int i = i0; i + 1 < n; ++i) {
        factor_row(&W(0, i), eb[i], db[i + 1] - l, i + 2 < n ? eb[i + 1] : 0.0, small, rsmall,
                   diag, sup);
        W(II_X, i) = start_entry(slot, i);
      }
      const double piv = diag;
      W(II_RP, n - 1) = fabs(piv) < small ? (piv < 0.0 ? -rsmall : rsmall) : 1.0 / piv;
      W(II_U1, n - 1) = 0.0;
      W(II_U2, n - 1) = 0.0;
      W(II_X, n - 1) = start_entry(slot, n - 1);
    }
    double scale = 1.0;  // x in memory times scale is the current vector
    for (int iter = 0; iter < 3; ++iter) {
      // the factorisation's row operations on the right-hand side
      for (int k = 0; k < II_AHEAD; ++k) ahead(k * CH);
      double rhs = W(II_X, 0) * scale;
      {
        int i0 = 0;
        for (; i0 + CH < n; i0 += CH) {  // full chunks: rows i0 + u + 1 < n
          ahead(i0 + II_AHEAD * CH);
          double* r = &W(0, i0);
          double rnv[CH], mv[CH], sv[CH];
#pragma unroll
          for (int u = 0; u < CH; ++u) {
            rnv[u] = r[(u + 1) * II_RS + II_X * 32] * scale;
            mv[u] = r[u * II_RS + II_MU * 32];
            sv[u] = r[u * II_RS + II_SW * 32];
          }
#pragma unroll
          for (int u = 0; u < CH; ++u) forward_row(r + u * II_RS, rnv[u], mv[u], sv[u], rhs);
        }
        for (int i = i0; i + 1 < n; ++i) {
          const double rn = W(II_X, i + 1) * scale;
          forward_row(&W(0, i), rn, W(II_MU, i), W(II_SW, i), rhs);
        }
      }
      W(II_X, n - 1) = rhs;
      // back substitution (the last row's U entries are zero), chunks of
      // rows [i0 - CH + 1, i0]
      for (int k = 0; k < II_AHEAD; ++k) ahead(n - (k + 1) * CH);
      double nrm2 = 0.0, x1 = 0.0, x2 = 0.0;
      {
        int i0 = n - 1;
        for (; i0 - CH + 1 >= 0; i0 -= CH) {
          ahead(i0 + 1 - (II_AHEAD + 1) * CH);
          double* r = &W(0, i0);
          double r0[CH], p1[CH], p2[CH], xv[CH];
#pragma unroll
          for (int u = 0; u < CH; ++u) {
            r0[u] = r[-u * II_RS + II_RP * 32];
            p1[u] = r[-u * II_RS + II_U1 * 32];
            p2[u] = r[-u * II_RS + II_U2 * 32];
            xv[u] = r[-u * II_RS + II_X * 32];
          }
#pragma unroll
          for (int u = 0; u < CH; ++u) {
            const double xi = (xv[u] - p1[u] * x1 - p2[u] * x2) * r0[u];
            r[-u * II_RS + II_X * 32] = xi;
            nrm2 += xi * xi;
            x2 = x1;
            x1 = xi;
          }
        }
        for (int i = i0; i >= 0; --i) {
          const double xi = (W(II_X, i) - W(II_U1, i) * x1 - W(II_U2, i) * x2) * W(II_RP, i);
          W(II_X, i) = xi;
          nrm2 += xi * xi;
          x2 = x1;
          x1 = xi;
        }
      }
      scale = 1.0 / sqrt(nrm2);
      if (q > 0) {
        // modified Gram-Schmidt against the cluster's earlier vectors (on the
        // normalised vector; rare: numerically equal eigenvalues only)
        for (int i = 0; i < n; ++i) W(II_X, i) *= scale;
        scale = 1.0;
        for (int r = 0; r < q; ++r) {
          const double* zr = Zt + (c.s0 + r);
          double dt = 0.0;
          for (int i = 0; i < n; ++i) dt += zr[(int64_t)(c.b0 + i) * p] * W(II_X, i);
          nrm2 = 0.0;
          for (int i = 0; i < n; ++i) {
            const double xi = W(II_X, i) - dt * zr[(int64_t)(c.b0 + i) * p];
            W(II_X, i) = xi;
            nrm2 += xi * xi;
          }
          const double inv = 1.0 / sqrt(nrm2);
          for (int i = 0; i < n; ++i) W(II_X, i) *= inv;
        }
      }
    }
    for (int i = 0; i < n; ++i) Zt[slot + (int64_t)(c.b0 + i) * p] = W(II_X, i) * scale;
  }
#undef W
}

// M = 1.5 I - 0.5 G (Newton-Schulz step for the polar factor).
__global__ void ns_matrix_kernel(double* __restrict__ g, int64_t p) {
  // M = (3I - G)/2 from the lower triangle of G (its upper one is not
  // computed), written to both triangles
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t j = blockIdx.y;
  if (i >= p || i < j) return;
  const double v = g[i + j * p];
  const double mv = (i == j ? 1.5 : 0.0) - 0.5 * v;
  g[i + j * p] = mv;
  g[j + i * p] = mv;
}

// Y[r, jj] = v_{j0+jj}[j0+1+r] (rows of the block's reach, zero above the
// reflector's first entry), n = p - j0 - 1 rows, nb columns.  Reflector j
// sits below the diagonal in column j (rowstore 0) or right of it in row j
// (rowstore 1), its head in vhead[j].
__global__ void build_y_kernel(const double* __restrict__ A, const double* __restrict__ vhead,
                               const double* __restrict__ beta, int64_t p, int64_t j0, int nb,
                               int rowstore, double* __restrict__ Y) {
  const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int jj = blockIdx.y;
  const int64_t n = p - j0 - 1;
  if (r >= n) return;
  const int64_t j = j0 + jj;
  const int64_t row = j0 + 1 + r;
  double v = 0.0;
  if (beta[j] == 0.0) v = 0.0;  // no reflection: a zero column of Y
  else if (row == j + 1) v = vhead[j];
  else if (row > j + 1) v = rowstore ? A[j + row * p] : A[row + j * p];
  Y[r + (int64_t)jj * n] = v;
}

// T of the compact WY form, H_{j0} ... H_{j0+nb-1} = I - Y T Y^T (forward),
// from T^{-1} = U = triu(S, 1) + diag(1 / beta), S = Y^T Y (the inverse of T
// is the strictly upper part of Y^T Y plus the reflectors' v^T v / 2 on the
// diagonal; a reflector with beta = 0 has a zero column in Y and a unit
// diagonal here).  A warp per column j of T solves U x = e_j: lane l keeps
// the running right-hand sides of rows l, l + 32, ...; from row j up, the
// owner of row i forms x_i = r_i beta_i (1 / U_ii = beta_i exactly) and
// every lane removes x_i's share from its rows above.  Each step is a
// shuffle and a few FMAs, so the 128-step chain of a column takes a few
// microseconds, all columns at once.  U lives in dynamic shared memory.
constexpr int WY_NB = 128;
constexpr int WY_T_WARPS = 32;  // columns per CTA
constexpr size_t wy_t_smem() { return sizeof(double) * (WY_NB * (WY_NB + 1) + WY_NB); }

__global__ void __launch_bounds__(WY_T_WARPS * 32) wy_t_kernel(const double* __restrict__ S,
                                                              const double* __restrict__ beta,
                                                              int64_t j0, int nb,
                                                              double* __restrict__ T) {
  extern __shared__ double u[];  // u[i LD + k] = U[i][k], i < k
  constexpr int LD = WY_NB + 1, QN = WY_NB / 32;
  double* rd = u + WY_NB * LD;   // 1 / U_ii
  for (int idx = threadIdx.x; idx < nb * nb; idx += blockDim.x) {
    const int i = idx % nb, k = idx / nb;
    if (i < k) u[i * LD + k] = S[i + k * nb];
  }
  for (int i = threadIdx.x; i < nb; i += blockDim.x)
    rd[i] = beta[j0 + i] != 0.0 ? beta[j0 + i] : 1.0;
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const int j = blockIdx.x * WY_T_WARPS + (threadIdx.x >> 5);
  if (j >= nb) return;  // no barrier follows
  double r[QN];
#pragma unroll
  for (int q = 0; q < QN; ++q) r[q] = lane + 32 * q == j ? 1.0 : 0.0;
  for (int i = j; i >= 0; --i) {
    const int owner = i & 31, qi = i >> 5;
    double xi = 0.0;
#pragma unroll
    for (int q = 0; q < QN; ++q)
      if (q == qi && lane == owner) {
        xi = r[q] * rd[i];
        r[q] = xi;  // row i is final: it now holds T[i][j]
      }
    xi = __shfl_sync(0xffffffffu, xi, owner);
#pragma unroll
    for (int q = 0; q < QN; ++q) {
      const int row = lane + 32 * q;
      if (row < i) r[q] -= u[row * LD + i] * xi;
    }
  }
#pragma unroll
  for (int q = 0; q < QN; ++q) {
    const int row = lane + 32 * q;
    if (row < nb) T[row + (int64_t)j * nb] = row <= j ? r[q] : 0.0;
  }
}

// out[:, k] = U[:, perm[k]]
__global__ void permute_columns_kernel(const double* __restrict__ U, int64_t p,
                                       const int* __restrict__ perm, double* __restrict__ out) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t k = blockIdx.y;
  if (i < p) out[i + k * p] = U[i + (int64_t)perm[k] * p];
}

// Column-major transpose: out[j + i p] = in[i + j p].
__global__ void transpose_sq_kernel(const double* __restrict__ in, int64_t p,
                                    double* __restrict__ out) {
  __shared__ double tile[32][33];
  const int64_t i0 = (int64_t)blockIdx.x * 32, j0 = (int64_t)blockIdx.y * 32;
  for (int dy = threadIdx.y; dy < 32; dy += blockDim.y) {
    const int64_t i = i0 + threadIdx.x, j = j0 + dy;
    if (i < p && j < p) tile[dy][threadIdx.x] = in[i + j * p];
  }
  __syncthreads();
  for (int dy = threadIdx.y; dy < 32; dy += blockDim.y) {
    const int64_t j = j0 + threadIdx.x, i = i0 + dy;
    if (i < p && j < p) out[j + i * p] = tile[threadIdx.x][dy];
  }
}

// A = the lower triangle mirrored (the eigensolver reads the lower triangle).
__global__ void mirror_lower_kernel(double* __restrict__ A, int64_t p) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t j = blockIdx.y;
  if (i < j && j < p) A[i + j * p] = A[j + i * p];
}

unsigned cdiv(int64_t a, int64_t b) { return (unsigned)((a + b - 1) / b); }

constexpr int NB = WY_NB;              // reflectors per WY block
// Eigenvalues closer than CLUSTER_TOL ||T|| (numerically equal) share one
// thread and are orthogonalised by Gram-Schmidt during inverse iteration;
// every other pair is left to inverse iteration, whose vectors then overlap
// by about eps ||T|| / gap, and to the Newton-Schulz steps (each squares
// the overlap), as many as the smallest such gap needs.
constexpr double CLUSTER_TOL = 1e-12;

// Scratch slots 46..54 belong to this file.
constexpr int SLOT_U = 46, SLOT_Z = 47, SLOT_G = 48, SLOT_SMALL = 49, SLOT_WS = 50,
              SLOT_WY = 51, SLOT_META = 52, SLOT_VB = 53, SLOT_SPLITK = 54;

}  // namespace

template <bool TA, bool TB>
static void launch_gemm(bool big, dim3 grid, int m, int n, int k, int kz, double alpha,
                        const double* A, int64_t lda, const double* B, int64_t ldb, double beta,
                        double* C, int64_t ldc, int lower, cudaStream_t s) {
  if (big)
    dgemm_big_kernel<TA, TB><<<grid, 256, 0, s>>>(m, n, k, kz, alpha, A, lda, B, ldb, beta, C,
                                                  ldc, lower);
  else
    dgemm_kernel<TA, TB><<<grid, 256, 0, s>>>(m, n, k, kz, alpha, A, lda, B, ldb, beta, C, ldc,
                                              lower);
}

shrk_status dgemm(bool ta, bool tb, int64_t m, int64_t n, int64_t k, double alpha, const double* A,
                  int64_t lda, const double* B, int64_t ldb, double beta, double* C, int64_t ldc,
                  cudaStream_t s, const char* family, bool lower) {
  if (m <= 0 || n <= 0) return SHRK_OK;
  if (lower && m != n) {
    set_error("dgemm: a lower-triangle product must be square");
    return SHRK_EINVAL;
  }
  if (m > INT32_MAX || n > INT32_MAX || k > INT32_MAX) {
    set_error("dgemm: dimensions must be below 2^31");
    return SHRK_EINVAL;
  }
  const bool big = m >= GT2 && n >= GT2 && k >= 64;
  const int tile = big ? GT2 : GT;
  const int64_t tiles = (int64_t)cdiv(m, tile) * cdiv(n, tile);
  // too few output tiles to fill the GPU and a long k: split k
  const int64_t want = 2LL * sm_count();
  int splits = 1;
  if (tiles < want && k >= 512)
    splits = (int)std::min<int64_t>({(want + tiles - 1) / tiles, k / 256, 16});
  double* out = C;
  int64_t ldo = ldc;
  double b = beta;
  if (splits > 1) {
    void* ws = nullptr;
    SHRK_TRY(scratch_get(SLOT_SPLITK, sizeof(double) * (size_t)splits * (size_t)m * (size_t)n, &ws));
    out = (double*)ws;
    ldo = m;
    b = 0.0;
  }
  const int kz = (int)((k + splits - 1) / splits);
  const dim3 grid(cdiv(m, tile), cdiv(n, tile), (unsigned)splits);
  {
    LaunchScope ls(family, s);
    if (!ta && !tb) launch_gemm<false, false>(big, grid, (int)m, (int)n, (int)k, kz, alpha, A, lda, B, ldb, b, out, ldo, lower ? 1 : 0, s);
    else if (!ta && tb) launch_gemm<false, true>(big, grid, (int)m, (int)n, (int)k, kz, alpha, A, lda, B, ldb, b, out, ldo, lower ? 1 : 0, s);
    else if (ta && !tb) launch_gemm<true, false>(big, grid, (int)m, (int)n, (int)k, kz, alpha, A, lda, B, ldb, b, out, ldo, lower ? 1 : 0, s);
    else launch_gemm<true, true>(big, grid, (int)m, (int)n, (int)k, kz, alpha, A, lda, B, ldb, b, out, ldo, lower ? 1 : 0, s);
    SHRK_CUDA(cudaGetLastError());
  }
  if (splits > 1) {
    LaunchScope ls(family, s);
    dgemm_reduce_kernel<<<cdiv(m * n, 256), 256, 0, s>>>(out, splits, (int)m, (int)n, beta, C, ldc);
    SHRK_CUDA(cudaGetLastError());
  }
  return SHRK_OK;
}

shrk_status eigh_device(double* A, int64_t p, std::vector<double>& w_host, cudaStream_t s) {
  w_host.assign((size_t)p, 0.0);
  if (p <= 0) return SHRK_OK;
  const int64_t P2 = p * p;
  void *small = nullptr, *zt = nullptr, *u = nullptr;
  // small: d, e, e2, vhead, beta, pv, scal (+2), part (<= 4096), lam, perm
  SHRK_TRY(scratch_get(SLOT_SMALL, sizeof(double) * (8 * (size_t)p + 4096 + 16), &small));
  double* d = (double*)small;
  double* e = d + p;
  double* e2 = e + p;
  double* vhead = e2 + p;
  double* beta = vhead + p;
  double* pv = beta + p;
  double* lam = pv + p;
  int* perm = (int*)(lam + p);  // p ints in the room of p/2 doubles (8p doubles reserved)
  double* scal = lam + 2 * p;
  double* part = scal + 16;
  SHRK_TRY(scratch_get(SLOT_Z, sizeof(double) * (size_t)P2, &zt));
  SHRK_TRY(scratch_get(SLOT_U, sizeof(double) * (size_t)P2, &u));
  double* Zt = (double*)zt;
  double* U = (double*)u;

  // 0. symmetric input from its lower triangle
  {
    LaunchScope ls("eigh_tridiag", s);
    mirror_lower_kernel<<<dim3(cdiv(p, 256), (unsigned)p), 256, 0, s>>>(A, p);
    SHRK_CUDA(cudaGetLastError());
  }
  // 1. tridiagonalisation (cooperative: all CTAs resident); one grid barrier
  // per column (tridiag1_kernel, reflectors in the upper triangle) unless
  // SHRK_EIGH_TRIDIAG=2 selects the two-barrier form
  const char* tri_env = std::getenv("SHRK_EIGH_TRIDIAG");
  const int rowstore = (tri_env && std::strcmp(tri_env, "2") == 0) ? 0 : 1;
  {
    int dev = 0, sms = 0, per_sm = 0;
    SHRK_CUDA(cudaGetDevice(&dev));
    SHRK_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    // one-barrier form: the per-CTA vectors in shared memory when they fit
    // (SHRK_EIGH_TRI1_GLOBAL=1 keeps them in global memory at any size)
    const size_t sh_bytes = sizeof(double) * 3 * (size_t)p;
    const char* glob_env = std::getenv("SHRK_EIGH_TRI1_GLOBAL");
    const bool sh = sh_bytes <= TRI1_SMEM_MAX && !(glob_env && std::strcmp(glob_env, "1") == 0);
    // rows per lane per step of the trailing update: SHRK_EIGH_TRI1_ROWS (8,
    // 16 or 32) or by size (measured: 8 best at p = 2 048, 18.8 ms; 16 at
    // 4 096, 87.3 ms; 32 slower at both)
    const char* rows_env = std::getenv("SHRK_EIGH_TRI1_ROWS");
    const int rows = rows_env ? std::atoi(rows_env) : (p >= 3072 ? 16 : 8);
    const void* tri1 = !sh          ? (const void*)tridiag1_kernel<false>
                       : rows == 32 ? (const void*)tridiag1_kernel<true, 32>
                       : rows == 8  ? (const void*)tridiag1_kernel<true, 8>
                                    : (const void*)tridiag1_kernel<true, 16>;
    const size_t dyn = rowstore && sh ? sh_bytes : 0;
    if (dyn > 0)
      SHRK_CUDA(cudaFuncSetAttribute(tri1, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dyn));
    SHRK_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(
        &per_sm, rowstore ? tri1 : (const void*)tridiag_kernel, TRI_NT, dyn));
    if (per_sm < 1) {
      set_error("eigensolver: the tridiagonalisation kernel cannot be resident");
      return SHRK_ECUDA;
    }
    const int blocks = std::min(sms, 2048);
    if (rowstore) {
      // p_j [2][p] and the partial sums [2][blocks]; the per-CTA vectors
      // [blocks][3][p] only when they are not in shared memory
      const size_t per_cta = sh ? 0 : (size_t)blocks * 3 * (size_t)p;
      void* vbuf = nullptr;
      SHRK_TRY(scratch_get(SLOT_VB, sizeof(double) * (per_cta + 2 * (size_t)p + 2 * (size_t)blocks),
                           &vbuf));
      double* vbd = (double*)vbuf;
      Tri1Args ta{A,          p,
                  d,          e,
                  vhead,      beta,
                  vbd + per_cta, vbd + per_cta + 2 * p,
                  sh ? nullptr : vbd, sh ? nullptr : vbd + (size_t)blocks * 2 * p};
      void* args[] = {&ta};
      LaunchScope ls("eigh_tridiag", s);
      SHRK_CUDA(cudaLaunchCooperativeKernel(tri1, dim3(blocks), dim3(TRI_NT), args, dyn, s));
    } else {
      TriArgs ta{A, p, d, e, vhead, beta, pv, part, scal};
      void* args[] = {&ta};
      LaunchScope ls("eigh_tridiag", s);
      SHRK_CUDA(cudaLaunchCooperativeKernel((const void*)tridiag_kernel, dim3(blocks),
                                            dim3(TRI_NT), args, 0, s));
    }
  }
  // 2. split T, Gershgorin bounds per block, eigenvalue slots (host; O(p))
  std::vector<double> hd(p), he(std::max<int64_t>(p - 1, 1), 0.0);
  SHRK_CUDA(cudaMemcpyAsync(hd.data(), d, sizeof(double) * p, cudaMemcpyDeviceToHost, s));
  if (p > 1)
    SHRK_CUDA(cudaMemcpyAsync(he.data(), e, sizeof(double) * (p - 1), cudaMemcpyDeviceToHost, s));
  SHRK_CUDA(cudaStreamSynchronize(s));
  const double eps = 2.220446049250313e-16;
  double tnorm = 0.0;
  for (int64_t i = 0; i < p; ++i) {
    const double r = (i > 0 ? std::fabs(he[i - 1]) : 0.0) + (i + 1 < p ? std::fabs(he[i]) : 0.0);
    tnorm = std::max(tnorm, std::fabs(hd[i]) + r);
  }
  if (!(tnorm > 0.0)) tnorm = 1.0;
  if (!std::isfinite(tnorm)) {
    set_error("symmetric eigendecomposition: the matrix has non-finite entries");
    return SHRK_EINVAL;
  }
  // negligible off-diagonals split T: relative to their diagonal neighbours
  // (dstebz's criterion) or below eps ||T|| (setting them to zero moves no
  // eigenvalue by more than the tridiagonalisation's own backward error;
  // without it a block of rounding noise -- the null space of a low-rank
  // matrix -- would stay one huge cluster)
  std::vector<double> he2(std::max<int64_t>(p - 1, 1), 0.0);
  std::vector<int> bstart{0};
  for (int64_t i = 0; i + 1 < p; ++i) {
    const double t2 = he[i] * he[i];
    if (t2 <= eps * eps * std::fabs(hd[i] * hd[i + 1]) + 1e-300 ||
        std::fabs(he[i]) <= eps * tnorm) {
      he[i] = 0.0;
      bstart.push_back((int)(i + 1));
    }
    he2[i] = he[i] * he[i];
  }
  bstart.push_back((int)p);
  const double pivmin = 1e-300 * std::max(1.0, tnorm * tnorm);
  std::vector<EigSlot> hslots(p);
  for (size_t b = 0; b + 1 < bstart.size(); ++b) {
    const int b0 = bstart[b], b1 = bstart[b + 1];
    double lo = INFINITY, hi = -INFINITY;
    for (int i = b0; i < b1; ++i) {
      const double r = (i > b0 ? std::fabs(he[i - 1]) : 0.0) + (i + 1 < b1 ? std::fabs(he[i]) : 0.0);
      lo = std::min(lo, hd[i] - r);
      hi = std::max(hi, hd[i] + r);
    }
    const double pad = 2.0 * eps * tnorm + 2.0 * pivmin;
    for (int i = b0; i < b1; ++i) hslots[i] = EigSlot{b0, b1, i - b0, 0, lo - pad, hi + pad};
  }
  void* meta = nullptr;
  SHRK_TRY(scratch_get(SLOT_META, sizeof(EigSlot) * (size_t)p + sizeof(Cluster) * (size_t)p + 256,
                       &meta));
  EigSlot* dslots = (EigSlot*)meta;
  Cluster* dcl = (Cluster*)(dslots + p);
  SHRK_CUDA(cudaMemcpyAsync(e, he.data(), sizeof(double) * std::max<int64_t>(p - 1, 0),
                            cudaMemcpyHostToDevice, s));
  SHRK_CUDA(cudaMemcpyAsync(e2, he2.data(), sizeof(double) * std::max<int64_t>(p - 1, 0),
                            cudaMemcpyHostToDevice, s));
  SHRK_CUDA(cudaMemcpyAsync(dslots, hslots.data(), sizeof(EigSlot) * p, cudaMemcpyHostToDevice, s));
  {
    LaunchScope ls("eigh_bisect", s);
    // probes per eigenvalue: SHRK_EIGH_PROBES (4, 8, 16 or 32) or by size
    // (measured: 16 best at p = 2 048, 3.1 ms; 8 at 4 096, 7.9 ms)
    int probes = p >= 3072 ? 8 : (p >= 1024 ? 16 : 32);
    if (const char* pe = std::getenv("SHRK_EIGH_PROBES")) {
      const int v = std::atoi(pe);
      if (v == 4 || v == 8 || v == 16 || v == 32) probes = v;
    }
    switch (probes) {
      case 4:
        bisect_kernel<4><<<cdiv(p * 4, 256), 256, 0, s>>>(d, e2, dslots, (int)p, pivmin, lam);
        break;
      case 8:
        bisect_kernel<8><<<cdiv(p * 8, 256), 256, 0, s>>>(d, e2, dslots, (int)p, pivmin, lam);
        break;
      case 16:
        bisect_kernel<16><<<cdiv(p * 16, 256), 256, 0, s>>>(d, e2, dslots, (int)p, pivmin, lam);
        break;
      default:
        bisect_kernel<32><<<cdiv(p * 32, 256), 256, 0, s>>>(d, e2, dslots, (int)p, pivmin, lam);
    }
    SHRK_CUDA(cudaGetLastError());
  }
  // 3. clusters of close eigenvalues inside each block (host), inverse iteration
  std::vector<double> hl(p);
  SHRK_CUDA(cudaMemcpyAsync(hl.data(), lam, sizeof(double) * p, cudaMemcpyDeviceToHost, s));
  SHRK_CUDA(cudaStreamSynchronize(s));
  std::vector<Cluster> hcl;
  double min_gap = INFINITY;  // smallest gap inside a block between clusters
  for (size_t b = 0; b + 1 < bstart.size(); ++b) {
    const int b0 = bstart[b], b1 = bstart[b + 1];
    int k = b0;
    while (k < b1) {
      int g = k + 1;
      while (g < b1 && hl[g] - hl[g - 1] < CLUSTER_TOL * tnorm) ++g;
      hcl.push_back(Cluster{k, g - k, b0, b1});
      if (g < b1) min_gap = std::min(min_gap, hl[g] - hl[g - 1]);
      k = g;
    }
  }
  // expected overlap of distinct inverse-iteration vectors, and the
  // Newton-Schulz steps that take it below rounding (e -> ~1.5 e^2)
  const double overlap = min_gap < INFINITY ? 8.0 * eps * tnorm / min_gap : 0.0;
  const int ns_steps = overlap <= 1e-15 ? 0 : (overlap <= 1e-7 ? 1 : 2);
  const int ncl = (int)hcl.size();
  SHRK_CUDA(cudaMemcpyAsync(dcl, hcl.data(), sizeof(Cluster) * ncl, cudaMemcpyHostToDevice, s));
  void* ws = nullptr;
  // per warp of clusters: p rows of II_ARRAYS x 32 doubles
  SHRK_TRY(scratch_get(SLOT_WS,
                       sizeof(double) * II_ARRAYS * 32 * (size_t)cdiv(ncl, 32) * (size_t)p, &ws));
  SHRK_CUDA(cudaMemsetAsync(Zt, 0, sizeof(double) * (size_t)P2, s));
  {
    LaunchScope ls("eigh_inverse_iteration", s);
    inverse_iteration_kernel<<<cdiv(ncl, 32), 32, 0, s>>>(d, e, lam, dcl, ncl, p, tnorm,
                                                            (double*)ws, Zt);
    SHRK_CUDA(cudaGetLastError());
  }
  // Newton-Schulz steps on the basis: Z <- Z (3I - Z^T Z)/2, in the
  // transposed storage Zt: G = Zt Zt^T, Zt <- M Zt
  void* gbuf = nullptr;
  SHRK_TRY(scratch_get(SLOT_G, sizeof(double) * (size_t)P2, &gbuf));
  double* G = (double*)gbuf;
  double* zcur = Zt;  // current Z^T
  double* other = U;
  for (int it = 0; it < ns_steps; ++it) {
    // G is symmetric: its lower triangle's tiles only, mirrored by the
    // kernel that forms M
    SHRK_TRY(dgemm(false, true, p, p, p, 1.0, zcur, p, zcur, p, 0.0, G, p, s, "dgemm", true));
    {
      LaunchScope ls("eigh_orthogonalise", s);
      ns_matrix_kernel<<<dim3(cdiv(p, 256), (unsigned)p), 256, 0, s>>>(G, p);
      SHRK_CUDA(cudaGetLastError());
    }
    SHRK_TRY(dgemm(false, false, p, p, p, 1.0, G, p, zcur, p, 0.0, other, p, s));  // (Z M)^T
    std::swap(zcur, other);
  }
  {
    LaunchScope ls("eigh_orthogonalise", s);
    transpose_sq_kernel<<<dim3(cdiv(p, 32), cdiv(p, 32)), dim3(32, 8), 0, s>>>(zcur, p, other);
    SHRK_CUDA(cudaGetLastError());
  }
  double* Zc = other;  // Z, column-major
  // 4. back-transformation Zc <- H_0 ... H_{p-3} Zc, blocks from the last
  const int64_t nref = std::max<int64_t>(p - 2, 0);
  if (nref > 0) {
    void* wy = nullptr;
    SHRK_TRY(scratch_get(SLOT_WY, sizeof(double) * ((size_t)p * NB * 3 + 2 * NB * NB), &wy));
    double* Y = (double*)wy;
    double* W = Y + (size_t)p * NB;
    double* W2 = W + (size_t)p * NB;
    double* S = W2 + (size_t)p * NB;
    double* T = S + NB * NB;
    for (int64_t j0 = ((nref - 1) / NB) * NB; j0 >= 0; j0 -= NB) {
      const int nb = (int)std::min<int64_t>(NB, nref - j0);
      const int64_t n = p - j0 - 1;
      {
        LaunchScope ls("eigh_wy_y", s);
        build_y_kernel<<<dim3(cdiv(n, 256), (unsigned)nb), 256, 0, s>>>(A, vhead, beta, p, j0,
                                                                        nb, rowstore, Y);
        SHRK_CUDA(cudaGetLastError());
      }
      SHRK_TRY(dgemm(true, false, nb, nb, n, 1.0, Y, n, Y, n, 0.0, S, nb, s, "dgemm_wy_yty"));
      {
        LaunchScope ls("eigh_wy_t", s);
        static std::atomic<bool> opted[64];
        int dv = 0;
        SHRK_CUDA(cudaGetDevice(&dv));
        if (dv < 0 || dv >= 64 || !opted[dv].load()) {
          SHRK_CUDA(cudaFuncSetAttribute(wy_t_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)wy_t_smem()));
          if (dv >= 0 && dv < 64) opted[dv] = true;
        }
        wy_t_kernel<<<(unsigned)cdiv(nb, WY_T_WARPS), WY_T_WARPS * 32, wy_t_smem(), s>>>(
            S, beta, j0, nb, T);
        SHRK_CUDA(cudaGetLastError());
      }
      double* Zs = Zc + (j0 + 1);  // rows j0+1 .. p-1 of Zc (leading dimension p)
      SHRK_TRY(dgemm(true, false, nb, p, n, 1.0, Y, n, Zs, p, 0.0, W, nb, s,
                     "dgemm_wy_ytz"));  // W = Y^T Zs
      SHRK_TRY(dgemm(false, false, nb, p, nb, 1.0, T, nb, W, nb, 0.0, W2, nb, s,
                     "dgemm_wy_tw"));  // W2 = T W
      SHRK_TRY(dgemm(false, false, n, p, nb, -1.0, Y, n, W2, nb, 1.0, Zs, p, s,
                     "dgemm_wy_update"));  // Zs -= Y W2
    }
  }
  // ascending eigenvalues; eigenvector columns in that order, into A
  std::vector<int> hperm(p);
  std::iota(hperm.begin(), hperm.end(), 0);
  std::stable_sort(hperm.begin(), hperm.end(), [&](int x, int y) { return hl[x] < hl[y]; });
  for (int64_t k = 0; k < p; ++k) w_host[k] = hl[hperm[k]];
  SHRK_CUDA(cudaMemcpyAsync(perm, hperm.data(), sizeof(int) * p, cudaMemcpyHostToDevice, s));
  {
    LaunchScope ls("eigh_back_transform", s);
    permute_columns_kernel<<<dim3(cdiv(p, 256), (unsigned)p), 256, 0, s>>>(Zc, p, perm, A);
    SHRK_CUDA(cudaGetLastError());
  }
  SHRK_CUDA(cudaStreamSynchronize(s));
  return SHRK_OK;
}

}  // namespace shrk
