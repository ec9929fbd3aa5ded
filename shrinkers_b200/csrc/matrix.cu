// Matrix front-end of the shrinkage estimators on sm_100a.
//
// Replaces src/pipeline/mod.rs: reconstruct_covariance 45-111,
// compute_d_bulk 114-129, clean_eigensystem 197-242, clean_covariance_matrix
// / clean_correlation_matrix 244-329 (one estimator), renormalize_to_unit_
// diagonal 331-341, reconstruct_from_eigenvalues 376-392,
// precision_from_eigensystem 409-464, estimate_precision_matrix 466-478 and
// symmetric_eigh 502-585; and compute_angular_overlaps
// (src/eigenvector_overlaps/overlaps.rs:26-46).
//
// The O(p^3) symmetric eigendecomposition is this library's own (eigh.cu:
// Householder tridiagonalisation, multisection, inverse iteration, WY
// back-transformation; the reference runs a Jacobi iteration and its docs
// point to LAPACK's dsyevd as the fast path).  The spectrum goes through
// this library's RIE and inverse-shrinkage paths; the per-eigenvalue host
// arithmetic (noise level, overlaps, bulk level) follows the reference's
// order.  The reconstructions run on the device: the spiked covariance
// d I + sum_t s_t v_t v_t^T over the k directions with a positive overlap --
// an FP64 kernel in the reference's operation order for k <= 16, the FP64
// GEMM of eigh.cu above, since the overlap is positive for every cleaned
// eigenvalue beyond sigma^2 (1 + sqrt(c)) and k can reach a fair share of
// p -- and the precision matrix U diag(w) U^T by the same GEMM.
//
// Layouts: caller matrices are row-major p x p with eigenvectors as columns;
// the device keeps the eigenvector matrix column-major (column j contiguous).
// Scratch slots 32..38 belong to this file.
#include "common.cuh"
#include "internal.h"

#include <algorithm>
#include <cmath>
#include <map>
#include <mutex>
#include <numeric>
#include <string>
#include <vector>

namespace shrk {

namespace {


constexpr int SLOT_E = 32;      // eigenvectors, column-major p x p
constexpr int SLOT_W = 33;      // eigenvalues / small vectors
constexpr int SLOT_IDX = 35;    // column indices, scales, flags
constexpr int SLOT_OUT = 36;    // p x p result
constexpr int SLOT_OUT2 = 37;   // p x p result (renormalised / eigenvectors)
constexpr int SLOT_TMP = 38;    // p x p staging (input, scaled columns)

// Up to this many active directions the spiked covariance is summed by
// spiked_reconstruct_kernel in the reference's order; beyond, by a DGEMM.
constexpr int SMALL_K = 16;

unsigned nblocks(int64_t n, int t) { return (unsigned)((n + t - 1) / t); }

// A[j*p + r] = V[r*p + j]: row-major eigenvectors (columns) to column-major.
__global__ void transpose_kernel(const double* __restrict__ v, int64_t p, double* __restrict__ a) {
  __shared__ double tile[32][33];
  const int64_t r0 = (int64_t)blockIdx.y * 32, j0 = (int64_t)blockIdx.x * 32;
  for (int dy = threadIdx.y; dy < 32; dy += blockDim.y) {
    const int64_t r = r0 + dy, j = j0 + threadIdx.x;
    if (r < p && j < p) tile[dy][threadIdx.x] = v[r * p + j];
  }
  __syncthreads();
  for (int dy = threadIdx.y; dy < 32; dy += blockDim.y) {
    const int64_t j = j0 + dy, r = r0 + threadIdx.x;
    if (r < p && j < p) a[j * p + r] = tile[threadIdx.x][dy];
  }
}

// out[r*p + i] = E[cols[i]*p + r]: the columns of E in the order cols, as a
// row-major matrix (mod.rs:480-490 permute_eigenvectors).
__global__ void gather_columns_kernel(const double* __restrict__ e, int64_t p,
                                      const int* __restrict__ cols, double* __restrict__ out) {
  __shared__ double tile[32][33];
  const int64_t i0 = (int64_t)blockIdx.x * 32, r0 = (int64_t)blockIdx.y * 32;
  for (int di = threadIdx.y; di < 32; di += blockDim.y) {
    const int64_t i = i0 + di, r = r0 + threadIdx.x;
    if (i < p && r < p) tile[di][threadIdx.x] = e[(int64_t)cols[i] * p + r];
  }
  __syncthreads();
  for (int dr = threadIdx.y; dr < 32; dr += blockDim.y) {
    const int64_t r = r0 + dr, i = i0 + threadIdx.x;
    if (i < p && r < p) out[r * p + i] = tile[threadIdx.x][dr];
  }
}

// mod.rs:78-108: Sigma[r][c] = d delta_rc + sum_t scales[t] V[r,t] V[c,t]
// over the k active columns, in the reference's order; thread (r, c >= r)
// writes both triangles.
__global__ void spiked_reconstruct_kernel(const double* __restrict__ e, int64_t p,
                                          const int* __restrict__ cols,
                                          const double* __restrict__ scales, int k, double d,
                                          double* __restrict__ out) {
  const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t r = blockIdx.y;
  if (c >= p || c < r) return;
  if (c == r) {
    double diag = d;
    for (int t = 0; t < k; ++t) {
      const double vr = e[(int64_t)cols[t] * p + r];
      diag += scales[t] * vr * vr;
    }
    out[r * p + r] = diag;
  } else {
    double val = 0.0;
    for (int t = 0; t < k; ++t) {
      const double* col = e + (int64_t)cols[t] * p;
      val += scales[t] * col[r] * col[c];
    }
    out[r * p + c] = val;
    out[c * p + r] = val;
  }
}

// G[t*p + r] = E[cols[t]*p + r] and B[t*p + r] = scales[t] * G[t*p + r]: the
// k active columns and their scaled copies, operands of the rank-k update.
__global__ void gather_scaled_kernel(const double* __restrict__ e, int64_t p,
                                     const int* __restrict__ cols,
                                     const double* __restrict__ scales, double* __restrict__ g,
                                     double* __restrict__ b) {
  const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t t = blockIdx.y;
  if (r >= p) return;
  const double v = e[(int64_t)cols[t] * p + r];
  g[t * p + r] = v;
  b[t * p + r] = scales[t] * v;
}

// After Sigma = B G^T: copy the upper triangle over the lower one and add d
// to the diagonal (d + sum_t s_t v_t^2, as the reference's diagonal).
__global__ void finish_spiked_kernel(double* __restrict__ m, int64_t p, double d) {
  const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t r = blockIdx.y;
  if (c >= p) return;
  if (c < r) m[r * p + c] = m[c * p + r];
  else if (c == r) m[r * p + r] = d + m[r * p + r];
}

// mod.rs:331-341: sc[i] = 1/sqrt(S[i][i]); *bad set when a diagonal entry is
// not positive (the matrix is then returned unchanged).
__global__ void diag_scales_kernel(const double* __restrict__ s, int64_t p, double* __restrict__ sc,
                                   int* __restrict__ bad) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= p) return;
  const double d = s[i * p + i];
  if (d <= 0.0) atomicExch(bad, 1);
  sc[i] = 1.0 / sqrt(d);
}

__global__ void renormalize_kernel(const double* __restrict__ s, int64_t p,
                                   const double* __restrict__ sc, const int* __restrict__ bad,
                                   double* __restrict__ out) {
  const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t i = blockIdx.y;
  if (j >= p) return;
  const double v = s[i * p + j];
  out[i * p + j] = *bad ? v : v * sc[i] * sc[j];
}

// B[j*p + r] = w[j] * E[j*p + r]  (the operand of U diag(w) U^T).
__global__ void scale_columns_kernel(const double* __restrict__ e, int64_t p,
                                     const double* __restrict__ w, double* __restrict__ b) {
  const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t j = blockIdx.y;
  if (r < p) b[j * p + r] = w[j] * e[j * p + r];
}

// Copies the upper triangle over the lower one (exact symmetry, as the
// reference's loop writes both from one value).
__global__ void symmetrize_kernel(double* __restrict__ m, int64_t p) {
  const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t r = blockIdx.y;
  if (c < r) m[r * p + c] = m[c * p + r];
}

dim3 rows_grid(int64_t p, int t) { return dim3(nblocks(p, t), (unsigned)p); }
dim3 tiles_grid(int64_t p) { return dim3(nblocks(p, 32), nblocks(p, 32)); }

// Eigendecomposition of the symmetric matrix in slot SLOT_E (its lower
// triangle; overwritten by the eigenvectors, column-major, column j for the
// j-th smallest eigenvalue); ascending eigenvalues to the host (eigh.cu).
shrk_status eigh_sorted_slot(int64_t p, std::vector<double>& w_host, cudaStream_t s) {
  void* a = nullptr;
  SHRK_TRY(scratch_get(SLOT_E, sizeof(double) * p * p, &a));
  return eigh_device((double*)a, p, w_host, s);
}

shrk_status einval_matrix(const char* what) {
  set_error(what);
  return SHRK_EINVAL;
}

shrk_status check_matrix_args(const void* m, size_t p, double c) {
  if (!m || p == 0) {
    set_error("matrix must be non-empty");
    return SHRK_EINVAL;
  }
  if (p > 46340) {  // p*p must fit the 32-bit sizes of the eigensolver
    set_error("matrix dimension p must be at most 46340");
    return SHRK_EINVAL;
  }
  if (!(std::isfinite(c) && c > 0.0)) {
    set_error("c (concentration ratio) must be a positive finite number");
    return SHRK_EINVAL;
  }
  return SHRK_OK;
}

// Descending order of the caller's eigenvalues (a stable sort; the
// reference's unstable sort orders ties arbitrarily).
std::vector<int> descending(const double* ev, size_t p) {
  std::vector<int> idx(p);
  std::iota(idx.begin(), idx.end(), 0);
  std::stable_sort(idx.begin(), idx.end(), [&](int a, int b) { return ev[b] < ev[a]; });
  return idx;
}

// Uploads the caller's row-major eigenvector matrix into SLOT_E, column-major.
shrk_status upload_eigenvectors(const double* v, int64_t p, cudaStream_t s) {
  void *a = nullptr, *t = nullptr;
  SHRK_TRY(scratch_get(SLOT_E, sizeof(double) * p * p, &a));
  SHRK_TRY(scratch_get(SLOT_TMP, sizeof(double) * p * p, &t));
  SHRK_CUDA(cudaMemcpyAsync(t, v, sizeof(double) * p * p, cudaMemcpyHostToDevice, s));
  transpose_kernel<<<tiles_grid(p), dim3(32, 8), 0, s>>>((const double*)t, p, (double*)a);
  SHRK_CUDA(cudaGetLastError());
  add_launches(1);
  return SHRK_OK;
}

// Downloads the columns `cols` of SLOT_E as a row-major matrix (dev_out:
// gathered straight into the caller's device matrix).
shrk_status download_columns(const std::vector<int>& cols, int64_t p, double* out,
                             cudaStream_t s, bool dev_out = false) {
  void *a = nullptr, *idx = nullptr, *o = nullptr;
  SHRK_TRY(scratch_get(SLOT_E, sizeof(double) * p * p, &a));
  SHRK_TRY(scratch_get(SLOT_IDX, sizeof(int) * p + 256, &idx));
  if (dev_out) o = out;
  else SHRK_TRY(scratch_get(SLOT_OUT2, sizeof(double) * p * p, &o));
  SHRK_CUDA(cudaMemcpyAsync(idx, cols.data(), sizeof(int) * p, cudaMemcpyHostToDevice, s));
  gather_columns_kernel<<<tiles_grid(p), dim3(32, 8), 0, s>>>((const double*)a, p,
                                                              (const int*)idx, (double*)o);
  SHRK_CUDA(cudaGetLastError());
  add_launches(1);
  if (!dev_out)
    SHRK_CUDA(cudaMemcpyAsync(out, o, sizeof(double) * p * p, cudaMemcpyDeviceToHost, s));
  SHRK_CUDA(cudaStreamSynchronize(s));
  return SHRK_OK;
}

// Copies p values from the host into a caller's device array (or a host
// array, when the outputs are on the host).
shrk_status put_vector(double* dst, const std::vector<double>& v, bool dev_out, cudaStream_t s) {
  if (!dst) return SHRK_OK;
  if (!dev_out) {
    std::copy(v.begin(), v.end(), dst);
    return SHRK_OK;
  }
  SHRK_CUDA(cudaMemcpyAsync(dst, v.data(), sizeof(double) * v.size(), cudaMemcpyHostToDevice, s));
  SHRK_CUDA(cudaStreamSynchronize(s));  // v is a local of the caller
  return SHRK_OK;
}

// mod.rs:197-242 from the eigenvectors in SLOT_E (column cols[i] belongs to
// the i-th largest eigenvalue sorted[i]).  The library lock is NOT held on
// entry: the RIE call takes it itself.
shrk_status clean_sorted(const std::vector<int>& cols, const std::vector<double>& sorted, double c,
                         int renorm, double* cov, double* evecs, double* l_rie, double* overlaps,
                         double* sigma2, bool dev_out = false) {
  const size_t p = sorted.size();
  std::vector<double> xi(p), a2(p, 0.0);
  // RmtConfig::new(c): Blocked, Sequential, no cutoff, eta = 0.4/sqrt(p)
  SHRK_TRY(shrk_rie_shrinkage(sorted.data(), p, c, SHRK_M_BLOCKED, SHRK_PREC_F64,
                              SHRK_PAR_SEQUENTIAL, xi.data()));
  // detection.rs:97-117 estimate_bulk_noise on the (descending) list
  const double med = (p % 2 == 0) ? (sorted[p / 2 - 1] + sorted[p / 2]) / 2.0 : sorted[p / 2];
  const double s2 = med / shrk_mp_median_factor(c);
  // overlaps.rs:26-46
  for (size_t i = 0; i < p; ++i) {
    const double diff = xi[i] - s2;
    if (diff > 1e-12) {
      const double num = 1.0 - (c * (s2 * s2)) / (diff * diff);
      const double den = 1.0 + (c * s2) / diff;
      if (num > 0.0) a2[i] = std::min(num / den, 1.0 - 1e-15);
    }
  }
  // mod.rs:114-129 compute_d_bulk, then the active columns and their scales
  double sum = 0.0;
  size_t count = 0;
  for (size_t i = 0; i < p; ++i)
    if (a2[i] == 0.0) {
      sum += xi[i];
      ++count;
    }
  double d_bulk = INFINITY;
  if (count > 0) {
    d_bulk = sum / (double)count;
  } else {
    for (size_t i = 0; i < p; ++i) d_bulk = std::min(d_bulk, xi[i]);
  }
  std::vector<int> act;
  std::vector<double> scales;
  for (size_t i = 0; i < p; ++i)
    if (a2[i] > 0.0) {
      act.push_back(cols[i]);
      scales.push_back(a2[i] * (xi[i] - d_bulk));
    }
  const int k = (int)act.size();
  cudaStream_t s = nullptr;
  LibScope L;
  SHRK_TRY(L.st);
  s = L.stream;
  const int64_t P = (int64_t)p;
  void *e = nullptr, *small = nullptr, *out = nullptr;
  SHRK_TRY(scratch_get(SLOT_E, sizeof(double) * P * P, &e));
  SHRK_TRY(scratch_get(SLOT_W, sizeof(double) * (2 * p + 4) + sizeof(int) * (p + 8), &small));
  SHRK_TRY(scratch_get(SLOT_OUT, sizeof(double) * P * P, &out));
  double* d_scales = (double*)small;
  double* d_sc = d_scales + p;
  int* d_flag = (int*)(d_sc + p + 4);
  int* d_cols = d_flag + 4;
  if (k > 0) {
    SHRK_CUDA(cudaMemcpyAsync(d_scales, scales.data(), sizeof(double) * k,
                              cudaMemcpyHostToDevice, s));
    SHRK_CUDA(cudaMemcpyAsync(d_cols, act.data(), sizeof(int) * k, cudaMemcpyHostToDevice, s));
  }
  if (k <= SMALL_K) {
    LaunchScope ls("matrix_reconstruct", s);
    spiked_reconstruct_kernel<<<rows_grid(P, 256), 256, 0, s>>>((const double*)e, P, d_cols,
                                                                d_scales, k, d_bulk, (double*)out);
    SHRK_CUDA(cudaGetLastError());
  } else {
    // many active directions: the rank-k update as a GEMM, Sigma = B G^T
    void* gb = nullptr;
    SHRK_TRY(scratch_get(SLOT_TMP, sizeof(double) * 2 * P * k, &gb));
    double* G = (double*)gb;
    double* B = G + P * k;
    {
      LaunchScope ls("matrix_reconstruct", s);
      gather_scaled_kernel<<<dim3(nblocks(P, 256), (unsigned)k), 256, 0, s>>>(
          (const double*)e, P, d_cols, d_scales, G, B);
      SHRK_CUDA(cudaGetLastError());
    }
    SHRK_TRY(dgemm(false, true, P, P, k, 1.0, B, P, G, P, 0.0, (double*)out, P, s));
    {
      LaunchScope ls("matrix_reconstruct", s);
      finish_spiked_kernel<<<rows_grid(P, 256), 256, 0, s>>>((double*)out, P, d_bulk);
      SHRK_CUDA(cudaGetLastError());
    }
  }
  double* result = (double*)out;
  if (renorm) {
    void* out2 = nullptr;
    SHRK_TRY(scratch_get(SLOT_OUT2, sizeof(double) * P * P, &out2));
    SHRK_CUDA(cudaMemsetAsync(d_flag, 0, sizeof(int), s));
    diag_scales_kernel<<<nblocks(P, 256), 256, 0, s>>>((const double*)out, P, d_sc, d_flag);
    SHRK_CUDA(cudaGetLastError());
    renormalize_kernel<<<rows_grid(P, 256), 256, 0, s>>>((const double*)out, P, d_sc, d_flag,
                                                         (double*)out2);
    SHRK_CUDA(cudaGetLastError());
    add_launches(2);
    result = (double*)out2;
  }
  SHRK_CUDA(cudaMemcpyAsync(cov, result, sizeof(double) * P * P,
                            dev_out ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, s));
  SHRK_CUDA(cudaStreamSynchronize(s));
  if (evecs) SHRK_TRY(download_columns(cols, P, evecs, s, dev_out));
  SHRK_TRY(put_vector(l_rie, xi, dev_out, s));
  SHRK_TRY(put_vector(overlaps, a2, dev_out, s));
  if (sigma2) *sigma2 = s2;
  return check_device_error(s);
}

// mod.rs:409-464 from the eigenvectors in SLOT_E; lock not held on entry.
shrk_status precision_sorted(const std::vector<int>& cols, const std::vector<double>& sorted,
                             double c, int method, double* prec, double* evecs, double* prec_ev,
                             double* cov_ev, double* smoothing, bool dev_out = false) {
  const size_t p = sorted.size();
  std::vector<double> pe(p), ce(p);
  double h = 0.0;
  SHRK_TRY(shrk_inverse_nonlinear_shrinkage(sorted.data(), p, c, method, pe.data(), ce.data(), &h,
                                            nullptr, nullptr));
  std::vector<double> w_col(p);
  for (size_t i = 0; i < p; ++i) w_col[cols[i]] = pe[i];
  LibScope L;
  SHRK_TRY(L.st);
  cudaStream_t s = L.stream;
  const int64_t P = (int64_t)p;
  void *e = nullptr, *small = nullptr, *b = nullptr, *out = nullptr;
  SHRK_TRY(scratch_get(SLOT_E, sizeof(double) * P * P, &e));
  SHRK_TRY(scratch_get(SLOT_W, sizeof(double) * (p + 4), &small));
  SHRK_TRY(scratch_get(SLOT_TMP, sizeof(double) * P * P, &b));
  SHRK_TRY(scratch_get(SLOT_OUT, sizeof(double) * P * P, &out));
  SHRK_CUDA(cudaMemcpyAsync(small, w_col.data(), sizeof(double) * p, cudaMemcpyHostToDevice, s));
  {
    LaunchScope ls("matrix_reconstruct", s);
    scale_columns_kernel<<<rows_grid(P, 256), 256, 0, s>>>((const double*)e, P,
                                                           (const double*)small, (double*)b);
    SHRK_CUDA(cudaGetLastError());
  }
  // Omega = B E^T (column-major; symmetric, so also the row-major result)
  SHRK_TRY(dgemm(false, true, P, P, P, 1.0, (const double*)b, P, (const double*)e, P, 0.0,
                 (double*)out, P, s));
  {
    LaunchScope ls("matrix_reconstruct", s);
    symmetrize_kernel<<<rows_grid(P, 256), 256, 0, s>>>((double*)out, P);
    SHRK_CUDA(cudaGetLastError());
  }
  SHRK_CUDA(cudaMemcpyAsync(prec, out, sizeof(double) * P * P,
                            dev_out ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, s));
  SHRK_CUDA(cudaStreamSynchronize(s));
  if (evecs) SHRK_TRY(download_columns(cols, P, evecs, s, dev_out));
  SHRK_TRY(put_vector(prec_ev, pe, dev_out, s));
  SHRK_TRY(put_vector(cov_ev, ce, dev_out, s));
  if (smoothing) *smoothing = h;
  return check_device_error(s);
}

// Eigendecomposition of a caller matrix into SLOT_E; descending eigenvalues
// and, for each, its column of SLOT_E.
shrk_status eigh_sorted(const double* m, int64_t p, std::vector<int>& cols,
                        std::vector<double>& sorted, bool dev_in = false) {
  LibScope L;
  SHRK_TRY(L.st);
  cudaStream_t s = L.stream;
  void* a = nullptr;
  SHRK_TRY(scratch_get(SLOT_E, sizeof(double) * p * p, &a));
  SHRK_CUDA(cudaMemcpyAsync(a, m, sizeof(double) * p * p,
                            dev_in ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, s));
  std::vector<double> w;
  SHRK_TRY(eigh_sorted_slot(p, w, s));
  cols.resize(p);
  sorted.resize(p);
  for (int64_t i = 0; i < p; ++i) {  // ascending: reverse it
    cols[i] = (int)(p - 1 - i);
    sorted[i] = w[p - 1 - i];
  }
  return SHRK_OK;
}

}  // namespace
}  // namespace shrk

using namespace shrk;

extern "C" {

shrk_status shrk_symmetric_eigh(const double* matrix, size_t p, double* eigenvalues,
                                double* eigenvectors) {
  SHRK_TRY(check_matrix_args(matrix, p, 1.0));
  std::vector<int> cols;
  std::vector<double> sorted;
  SHRK_TRY(eigh_sorted(matrix, (int64_t)p, cols, sorted));
  for (size_t i = 0; i < p; ++i) eigenvalues[i] = sorted[p - 1 - i];
  if (!eigenvectors) return SHRK_OK;
  std::vector<int> asc(p);
  std::iota(asc.begin(), asc.end(), 0);
  LibScope L;
  SHRK_TRY(L.st);
  SHRK_TRY(download_columns(asc, (int64_t)p, eigenvectors, L.stream));
  return check_device_error(L.stream);
}

shrk_status shrk_clean_eigensystem(const double* eigenvectors, const double* eigenvalues,
                                   size_t p, double c, double* covariance,
                                   double* sorted_eigenvectors, double* rie_eigenvalues,
                                   double* overlaps, double* sigma2) {
  SHRK_TRY(check_matrix_args(eigenvectors, p, c));
  std::vector<int> cols = descending(eigenvalues, p);
  std::vector<double> sorted(p);
  for (size_t i = 0; i < p; ++i) sorted[i] = eigenvalues[cols[i]];
  {
    LibScope L;
    SHRK_TRY(L.st);
    SHRK_TRY(upload_eigenvectors(eigenvectors, (int64_t)p, L.stream));
  }
  return clean_sorted(cols, sorted, c, 0, covariance, sorted_eigenvectors, rie_eigenvalues,
                      overlaps, sigma2);
}

shrk_status shrk_clean_covariance_matrix(const double* matrix, size_t p, double c,
                                         int renormalize, double* covariance,
                                         double* eigenvectors, double* rie_eigenvalues,
                                         double* overlaps, double* sigma2) {
  SHRK_TRY(check_matrix_args(matrix, p, c));
  std::vector<int> cols;
  std::vector<double> sorted;
  SHRK_TRY(eigh_sorted(matrix, (int64_t)p, cols, sorted));
  return clean_sorted(cols, sorted, c, renormalize, covariance, eigenvectors, rie_eigenvalues,
                      overlaps, sigma2);
}

shrk_status shrk_renormalize_to_unit_diagonal(const double* matrix, size_t p, double* out) {
  SHRK_TRY(check_matrix_args(matrix, p, 1.0));
  LibScope L;
  SHRK_TRY(L.st);
  cudaStream_t s = L.stream;
  const int64_t P = (int64_t)p;
  void *in = nullptr, *o = nullptr, *small = nullptr;
  SHRK_TRY(scratch_get(SLOT_OUT, sizeof(double) * P * P, &in));
  SHRK_TRY(scratch_get(SLOT_OUT2, sizeof(double) * P * P, &o));
  SHRK_TRY(scratch_get(SLOT_W, sizeof(double) * (p + 4) + 16, &small));
  double* d_sc = (double*)small;
  int* d_flag = (int*)(d_sc + p + 2);
  SHRK_CUDA(cudaMemcpyAsync(in, matrix, sizeof(double) * P * P, cudaMemcpyHostToDevice, s));
  SHRK_CUDA(cudaMemsetAsync(d_flag, 0, sizeof(int), s));
  diag_scales_kernel<<<nblocks(P, 256), 256, 0, s>>>((const double*)in, P, d_sc, d_flag);
  SHRK_CUDA(cudaGetLastError());
  renormalize_kernel<<<rows_grid(P, 256), 256, 0, s>>>((const double*)in, P, d_sc, d_flag,
                                                       (double*)o);
  SHRK_CUDA(cudaGetLastError());
  add_launches(2);
  SHRK_CUDA(cudaMemcpyAsync(out, o, sizeof(double) * P * P, cudaMemcpyDeviceToHost, s));
  SHRK_CUDA(cudaStreamSynchronize(s));
  return check_device_error(s);
}

shrk_status shrk_precision_from_eigensystem(const double* eigenvectors, const double* eigenvalues,
                                            size_t p, double c, int method, double* precision,
                                            double* sorted_eigenvectors, double* precision_ev,
                                            double* covariance_ev, double* smoothing) {
  SHRK_TRY(check_matrix_args(eigenvectors, p, c));
  std::vector<int> cols = descending(eigenvalues, p);
  std::vector<double> sorted(p);
  for (size_t i = 0; i < p; ++i) sorted[i] = eigenvalues[cols[i]];
  {
    LibScope L;
    SHRK_TRY(L.st);
    SHRK_TRY(upload_eigenvectors(eigenvectors, (int64_t)p, L.stream));
  }
  return precision_sorted(cols, sorted, c, method, precision, sorted_eigenvectors, precision_ev,
                          covariance_ev, smoothing);
}

shrk_status shrk_estimate_precision_matrix(const double* matrix, size_t p, double c, int method,
                                           double* precision, double* eigenvectors,
                                           double* precision_ev, double* covariance_ev,
                                           double* smoothing) {
  SHRK_TRY(check_matrix_args(matrix, p, c));
  std::vector<int> cols;
  std::vector<double> sorted;
  SHRK_TRY(eigh_sorted(matrix, (int64_t)p, cols, sorted));
  return precision_sorted(cols, sorted, c, method, precision, eigenvectors, precision_ev,
                          covariance_ev, smoothing);
}

// Device-pointer forms.  The library runs them on its own stream for the
// calling thread (the steps between the kernels are host arithmetic that
// needs the spectrum on the host); they wait for the work already queued on
// the caller's stream before reading its matrix, and the caller's stream
// waits for their outputs.
namespace {
struct StreamJoin {
  cudaStream_t caller;
  shrk_status st = SHRK_OK;
  explicit StreamJoin(void* stream) : caller((cudaStream_t)stream) {
    LibScope L;
    st = L.st;
    if (st != SHRK_OK) return;
    st = join(caller, L.stream);
  }
  // `after` waits for everything queued on `before` so far
  static shrk_status join(cudaStream_t before, cudaStream_t after) {
    if (before == after) return SHRK_OK;
    cudaEvent_t ev;
    SHRK_CUDA(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
    cudaError_t e = cudaEventRecord(ev, before);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(after, ev, 0);
    cudaEventDestroy(ev);
    if (e != cudaSuccess) {
      set_error(std::string("CUDA: ") + cudaGetErrorString(e));
      return SHRK_ECUDA;
    }
    return SHRK_OK;
  }
  shrk_status finish(shrk_status r) {
    if (r != SHRK_OK) return r;
    LibScope L;
    SHRK_TRY(L.st);
    return join(L.stream, caller);
  }
};
}  // namespace

shrk_status shrk_symmetric_eigh_dev(const double* d_matrix, size_t p, double* d_eigenvalues,
                                    double* d_eigenvectors, void* stream) {
  SHRK_TRY(check_matrix_args(d_matrix, p, 1.0));
  if (!d_eigenvalues) return einval_matrix("null eigenvalue output");
  StreamJoin J(stream);
  SHRK_TRY(J.st);
  std::vector<int> cols;
  std::vector<double> sorted;
  SHRK_TRY(eigh_sorted(d_matrix, (int64_t)p, cols, sorted, true));
  std::vector<double> asc(sorted.rbegin(), sorted.rend());
  shrk_status r = SHRK_OK;
  {
    LibScope L;
    SHRK_TRY(L.st);
    SHRK_TRY(put_vector(d_eigenvalues, asc, true, L.stream));
    if (d_eigenvectors) {
      std::vector<int> idx(p);
      std::iota(idx.begin(), idx.end(), 0);
      SHRK_TRY(download_columns(idx, (int64_t)p, d_eigenvectors, L.stream, true));
    }
    r = check_device_error(L.stream);
  }
  return J.finish(r);
}

shrk_status shrk_clean_covariance_matrix_dev(const double* d_matrix, size_t p, double c,
                                             int renormalize, double* d_covariance,
                                             double* d_eigenvectors, double* d_rie_eigenvalues,
                                             double* d_overlaps, double* sigma2, void* stream) {
  SHRK_TRY(check_matrix_args(d_matrix, p, c));
  if (!d_covariance) return einval_matrix("null covariance output");
  StreamJoin J(stream);
  SHRK_TRY(J.st);
  std::vector<int> cols;
  std::vector<double> sorted;
  SHRK_TRY(eigh_sorted(d_matrix, (int64_t)p, cols, sorted, true));
  return J.finish(clean_sorted(cols, sorted, c, renormalize, d_covariance, d_eigenvectors,
                               d_rie_eigenvalues, d_overlaps, sigma2, true));
}

shrk_status shrk_estimate_precision_matrix_dev(const double* d_matrix, size_t p, double c,
                                               int method, double* d_precision,
                                               double* d_eigenvectors, double* d_precision_ev,
                                               double* d_covariance_ev, double* smoothing,
                                               void* stream) {
  SHRK_TRY(check_matrix_args(d_matrix, p, c));
  if (!d_precision) return einval_matrix("null precision output");
  StreamJoin J(stream);
  SHRK_TRY(J.st);
  std::vector<int> cols;
  std::vector<double> sorted;
  SHRK_TRY(eigh_sorted(d_matrix, (int64_t)p, cols, sorted, true));
  return J.finish(precision_sorted(cols, sorted, c, method, d_precision, d_eigenvectors,
                                   d_precision_ev, d_covariance_ev, smoothing, true));
}

}  // extern "C"
