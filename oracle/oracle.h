// TEST INFRASTRUCTURE ONLY.
//
// CPU restatement of the shrinkers crate's Stieltjes-transform algorithms,
// used as the parity checker for the CUDA path and as the timed CPU
// baseline.  Nothing in the product (shrinkers_b200/) links or loads it;
// only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg do.
//
// Arithmetic follows the reference's x86-64 semantics:
//   * `f64::mul_add` / `f32::mul_add` are fused  -> std::fma / std::fmaf
//   * lane `fma` of the SIMD wrappers is UNFUSED -> a + b*c
//     (src/stieltjes/simd.rs:176-185, 457-470 on non-aarch64)
//   * `recip` / `recip_fast` are true divisions   (simd.rs:194-236, 512-532)
//   * `hsum` is l0+l1 and (l0+l1)+(l2+l3)          (simd.rs:238-247, 534-543)
// The sources are compiled with -ffp-contract=off so that no other product
// is contracted into an FMA behind our back.
#pragma once
#include <cstddef>
#include <cstdint>
#include <vector>

namespace orc {

// Method identifiers, in the declaration order of StieltjesMethod
// (src/config.rs:19-89).
enum Method : int {
  NAIVE = 0, AUTOVEC, BLOCKED, BLOCKED_AUTOVEC, BLOCKED_TILED, BLOCKED_WINDOWED,
  BLOCKED_HYBRID, ADAPTIVE, FFT5, FFT3, FFT2, NUFFT, TREECODE, CHEBCODE,
  CHEBCODE_FAST, CHEBCODE_XTREME, CHEBCODE_BALANCED, EWALD, DST, AUTO, HODLR,
  SPEED_AUTO, ACCURACY_AUTO
};

bool is_auto(int m);
int resolve_auto_method(int m, bool parallel, size_t p);
int grid_appropriate(int m, size_t p, size_t nq);
bool is_sorted_ascending(const double* v, size_t n);

// Exact family (raw sums unless noted).
void autovec_sum(double x, const double* ev, size_t p, double eta, double* re, double* im);
void naive_sum(double x, const double* ev, size_t p, double eta, double* re, double* im);
void sum_cutoff(double x, const double* ev, size_t p, double eta, double cutoff, double* re, double* im);
void symmetric_sweep(const double* ev, size_t p, double eta, double* re, double* im);
void tiled_span_no_cutoff(const double* targets, size_t nt, const double* ev, size_t p,
                          size_t bs, double eta, double* re, double* im);
void tiled_one_target_pub(double t, const double* ev, size_t p, double eta, double eta_sq,
                          double* r, double* i);
void tiled_parallel(const double* ev, size_t p, double eta, double* re, double* im);
void tiled_blocks_parallel(const double* targets, size_t nt, const double* ev, size_t p,
                           double eta, double* re, double* im);
void blocked_at_points(const double* q, size_t nq, const double* ev, size_t p, double eta,
                       double cutoff, double* re, double* im);
void windowed(const double* ev, size_t p, double eta, double cut, double* re, double* im);
void windowed_parallel(const double* ev, size_t p, double eta, double cut, double* re, double* im);

// Dispatchers.  compute_all returns SCALED (1/p) values; at_points RAW sums.
// Return 0 on success, 4 when the method is outside the restated set.
int compute_all(const double* ev, size_t p, double eta, int method, double cutoff,
                bool parallel, double* re, double* im);
int compute_at_points(const double* q, size_t nq, const double* ev, size_t p, double eta,
                      int method, double cutoff, bool parallel, double* re, double* im);

// ChebCode (src/stieltjes/chebcode.rs).
struct ChebPreset { double theta; int n; int leaf_cap; bool f32; };
bool cheb_preset(int method, ChebPreset* out);
void chebcode_points(const double* q, size_t nq, const double* ev, size_t p, double eta,
                     double theta, int n, int leaf_cap, bool f32, bool parallel,
                     double* re, double* im);
size_t grid_leaf_cap(size_t n, size_t p, size_t nq, size_t preset_leaf);

// NUFFT (src/stieltjes/nufft.rs + fft5.rs).
size_t nufft_grid_size(double raw_range, double eta);
void nufft_points(const double* q, size_t nq, const double* sorted_ev, size_t p, double eta,
                  bool parallel, double* re, double* im);

// fft5 grid convolution (src/stieltjes/fft5.rs), raw sums.  order = stencil
// nodes (2/4/6/8), m_override 0 = the adaptive grid rule.  Returns 4 when the
// grid size is not a power of two.
size_t fft5_grid_size(double lo_raw, double hi_raw, size_t p, double eta, double pad_eta_mult,
                      double pad_range_frac);
int fft5_points(const double* q, size_t nq, const double* ev, size_t p, double eta, int order,
                size_t m_override, double pad_eta_mult, double pad_range_frac, double* re,
                double* im);

}  // namespace orc
