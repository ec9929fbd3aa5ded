// Internal (C++) interfaces between the C-ABI layer and the kernel files.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>
#include <vector>

#include "../../include/shrinkers_b200.h"

namespace shrk {

// What the FP64 reduction epilogue of the pair-sum kernels writes.
enum EpilogueMode : int {
  EPI_SUMS = 0,    // out_re/out_im = raw sums * scale
  EPI_LW = 1,      // out_re = shrinkage_factor(x, c, re*scale, im*scale)
  EPI_MP = 2,      // El Karoui inversion on a grid: 6 arrays (see exact.cu)
  EPI_DERIV = 3,   // value + derivative (4 arrays), E7
};

struct Epilogue {
  int mode = EPI_SUMS;
  double scale = 1.0;      // 1/p for the all-points convention
  double c = 0.0;          // concentration ratio (LW, MP)
  double eta = 0.0;        // imaginary part of z (MP)
  double* out_re = nullptr;
  double* out_im = nullptr;
  double* out[6] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
};

// Exact O(nt * ns) pair sums S(x_t) = sum_j 1/((x_t - s_j) - i eta), on the
// device, with the epilogue fused into the deterministic split reduction.
// precision: SHRK_PREC_F64 or SHRK_PREC_MIXED.
shrk_status exact_pair_sums(const double* d_tgt, int64_t nt, const double* d_src, int64_t ns,
                            double eta, int precision, const Epilogue& epi, cudaStream_t s);

// The same raw sums (no epilogue) with every temporary in caller-provided
// device memory and no library state touched: `part` holds part_capacity
// (re, im) split partials (>= nt), `bounds` ns/256 + 2 double2 (MIXED only),
// `err` a device int the caller has zeroed on stream s.  If a bounded wait
// gives up, every output is NaN.  sms = multiprocessor count of the device.
shrk_status exact_pair_sums_fixed(const double* d_tgt, int64_t nt, const double* d_src,
                                  int64_t ns, double eta, int precision, double* d_re,
                                  double* d_im, double* part, int64_t part_capacity,
                                  double2* bounds, int* err, int sms, cudaStream_t s);

// Windowed sums: only pairs with |x_t - s_j| <= window are included (sorted
// sources).  which: bit 0 = real part, bit 1 = imaginary part.
shrk_status windowed_sums(const double* d_tgt, int64_t nt, const double* d_src, int64_t ns,
                          double eta, double window, double scale, double* d_re, double* d_im,
                          cudaStream_t s);

// E7: raw value + derivative at every source point.
shrk_status with_deriv(const double* d_ev, int64_t p, double eta, double* d_re, double* d_im,
                       double* d_dre, double* d_dim, cudaStream_t s);

// mod.rs:304-319: RAW sums at z_t = ev_t (1 + i scale) (eta_t = scale ev_t).
shrk_status scaled_ray_sums(const double* d_ev, int64_t p, double scale, double* d_re,
                            double* d_im, cudaStream_t s);

// E6: FP32 full-square sums scaled by 1/p in FP32.
shrk_status all_f32(const float* d_ev, int64_t p, float eta, float* d_re, float* d_im,
                    cudaStream_t s);

// Adjoint of the all-points transform (see shrk_stieltjes_adjoint).
shrk_status adjoint(const double* d_ev, int64_t p, double eta, const double* d_gre,
                    const double* d_gim, int precision, double* d_grad, cudaStream_t s);

// Batched uneven spectra (batched.cu).  h_offsets may be null (then the
// offsets and etas are read back from the device to build the plan).
shrk_status batched(const double* d_ev, const int64_t* d_offsets, const int64_t* h_offsets,
                    int64_t n_spectra, const double* d_eta, int precision, double* d_re,
                    double* d_im, cudaStream_t s);
// Runs the batched autotuner for `precision` on the current device (if it has
// not run yet, or if force) and writes (R, SL) for the 8 p-buckets into
// table[16] (may be null).
shrk_status batched_tune(int precision, bool force, int* table, cudaStream_t s);
// Installs a table of the same layout (e.g. one saved from an earlier
// process) for `precision` on the current device.
shrk_status batched_set_tune(int precision, const int* table);

// Epilogue over precomputed raw sums (n targets), same arithmetic as the
// fused reduction of exact_pair_sums.
shrk_status apply_epilogue(const double* d_tgt, const double* d_raw_re, const double* d_raw_im,
                           int64_t n, const Epilogue& epi, cudaStream_t s);

// Coarse-grid NUFFT at nq points, epilogue fused into the interpolation.
// d_sorted_src holds the sources in ascending order; lo_raw/hi_raw are the
// first and last source values IN THE CALLER'S ORDER (the reference takes
// the grid bounds from the first and last entries, nufft.rs:139-146).
shrk_status nufft_points(const double* d_q, int64_t nq, const double* d_sorted_src, int64_t ns,
                         double lo_raw, double hi_raw, double eta, const Epilogue& epi,
                         cudaStream_t s);
size_t nufft_grid_size(double raw_range, double eta);
// The NUFFT grid (m cells from lo, spacing dx) of a spectrum whose first and
// last entries in the caller's order are lo_raw / hi_raw.
void nufft_geometry(double lo_raw, double hi_raw, double eta, int64_t* m, double* lo,
                    double* dx);
// The NUFFT's two stages apart: the order-4 splat of ns ascending sources
// into d_density[m] (linear in the sources), and the convolution of a
// density with the kernel pair plus interpolation at nq queries.
shrk_status nufft_density(const double* d_sorted_src, int64_t ns, int64_t m, double lo, double dx,
                          double* d_density, cudaStream_t s);
shrk_status nufft_eval(const double* d_density, int64_t m, double lo, double dx, double eta,
                       const double* d_q, int64_t nq, const Epilogue& epi, cudaStream_t s);

// fft5.rs:213-249 Fft5Options: stencil nodes (2/4/6/8), forced grid size
// (0 = the adaptive rule dx <= eta/8, m >= 8p), padding multipliers.
struct Fft5Opts {
  int order = 8;
  size_t m_override = 0;
  double pad_eta_mult = 1000.0;
  double pad_range_frac = 0.75;
};
// fft5 grid convolution at nq points (same source contract as nufft_points);
// SHRK_ENOTIMPL when the grid is larger than 2^22 cells (2^21 when the size
// is not a power of two).
shrk_status fft5_points(const double* d_q, int64_t nq, const double* d_sorted_src, int64_t ns,
                        double lo_raw, double hi_raw, double eta, const Fft5Opts& o,
                        const Epilogue& epi, cudaStream_t s);
size_t fft5_grid_size(double lo_raw, double hi_raw, size_t p, double eta, double pad_eta_mult,
                      double pad_range_frac);

// Chebyshev treecode at nq points, epilogue fused into the evaluation.
struct ChebParams { double theta; int n; int leaf_cap; bool f32; };
bool cheb_preset(int method, ChebParams* out);
size_t grid_leaf_cap(size_t n, size_t p, size_t nq, size_t preset_leaf);
shrk_status chebcode_points(const double* d_q, int64_t nq, const double* d_sorted_src, int64_t ns,
                            double eta, const ChebParams& prm, const Epilogue& epi,
                            cudaStream_t s);

// Sources in ascending order on the device (d_src itself when already
// sorted, else a sorted copy in library scratch) and the first / last entry
// of d_src in the caller's order (sources.cu).
shrk_status sorted_sources(const double* d_src, int64_t ns, const double** d_sorted,
                           double* first, double* last, cudaStream_t s);
// The same, plus the permutation: d_sorted[i] = d_src[perm[i]]; *d_perm is
// null when d_src is already sorted (the identity).  With lo / hi given,
// also the smallest and largest source (no extra read-back for sorted
// input).
shrk_status sorted_sources_perm(const double* d_src, int64_t ns, const double** d_sorted,
                                const int** d_perm, cudaStream_t s, double* lo = nullptr,
                                double* hi = nullptr);

// Treecode adjoint (chebcode.cu): the gradient of shrk_stieltjes_adjoint
// with every source sum evaluated by the ChebCode tree of preset `prm`.
shrk_status chebcode_adjoint(const double* d_ev, int64_t p, double eta, const double* d_gre,
                             const double* d_gim, const ChebParams& prm, double* d_grad,
                             cudaStream_t s);

// chebcode.rs:1312-1361 ChebCodeBatch::evaluate_many on the GPU: RAW sums at
// every eigenvalue for each of n_eta etas (device array), [n_eta][p].
shrk_status chebcode_evaluate_many(const double* d_ev, int64_t p, const double* d_etas,
                                   int64_t n_eta, const ChebParams& prm, double* d_re,
                                   double* d_im, cudaStream_t s);

// The library lock for code outside the C-ABI file: serialises library
// calls and selects the calling thread's device state (scratch, stream) for
// the scope's lifetime.  Not re-entrant: release it before calling a C-ABI
// entry point.
shrk_status lib_enter(cudaStream_t* stream);
void lib_exit();
struct LibScope {
  shrk_status st;
  cudaStream_t stream = nullptr;
  LibScope() { st = lib_enter(&stream); }
  ~LibScope() { lib_exit(); }
  LibScope(const LibScope&) = delete;
  LibScope& operator=(const LibScope&) = delete;
};

// Dyadic Chebyshev FMM (fmm.cu): S(ev_t)/p at every eigenvalue, in the
// caller's order, expansion order n in [4, 16]; m2l_tc: M2L on the tensor
// cores (TF32 x3) instead of FP64.
shrk_status fmm_all(const double* d_ev, int64_t p, double eta, int n, int m2l_tc, double* d_re,
                    double* d_im, cudaStream_t s);

// FP64 GEMM (eigh.cu): C = alpha op(A) op(B) + beta C, column-major,
// op = transpose when ta / tb.
shrk_status dgemm(bool ta, bool tb, int64_t m, int64_t n, int64_t k, double alpha, const double* A,
                  int64_t lda, const double* B, int64_t ldb, double beta, double* C, int64_t ldc,
                  cudaStream_t s, const char* family = "dgemm", bool lower = false);
// Symmetric eigendecomposition of A (p x p column-major, lower triangle
// read; overwritten by the eigenvectors, column j for the j-th smallest
// eigenvalue); the eigenvalues ascending to w_host.  Synchronises s.
shrk_status eigh_device(double* A, int64_t p, std::vector<double>& w_host, cudaStream_t s);

double mixed_near_k();
// Sets the bulk-copy wait budget of the exact pair kernels (cycles; negative
// = the default) and returns the previous one.
long long set_wait_cycles(long long cycles);
shrk_status measure_pipe_rates(double* fp32, double* fp64);
shrk_status measure_rcp_bias(double* uniform_mean, double* log_mean);

}  // namespace shrk
