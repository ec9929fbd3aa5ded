/*
 * shrinkers_b200 -- diagnostics and measurement entry points.
 *
 * Not part of the drop-in boundary (include/shrinkers_b200.h): these have no
 * counterpart in the shrinkers crate.  They serve the benchmark (per-kernel
 * timing, launch counts, the measured pipe rates that are the roofline
 * denominators), the reciprocal-bias check of the mixed kernel, and the test
 * of the timeout path.  Same conventions as the main header: plain pointers,
 * status codes, no aborts.
 */
#ifndef SHRINKERS_B200_DIAG_H
#define SHRINKERS_B200_DIAG_H

#include <stdint.h>

#include "shrinkers_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Per-kernel CUDA-event timing of the library's own launches (off by
 * default).  shrk_timing_read returns the number of launches of the kernel
 * family `name` since the last reset and their summed duration (ms). */
void shrk_timing_enable(int on);
void shrk_timing_reset(void);
shrk_status shrk_timing_read(const char* name, int64_t* launches, double* total_ms);
/* Number of kernels the library launched since the last reset. */
int64_t shrk_launch_count(void);
/* Measured FMA issue rates of the current device (lane-operations per
 * second, one FMA = one op) for FP32 and FP64: the roofline denominators of
 * the exact kernels.  Runs two short probe kernels. */
shrk_status shrk_measure_pipe_rates(double* fp32_ops_per_s, double* fp64_ops_per_s);
/* Mean relative error of the FP32 MUFU reciprocal (rcp.approx.ftz.f32) of
 * the current device over every mantissa of [1, 2): plain and weighted 1/m
 * (log-uniform).  The mixed-precision pair kernel removes the log-uniform
 * mean from its FP32 far-field partials; this probe re-measures it. */
shrk_status shrk_measure_rcp_bias(double* uniform_mean, double* log_mean);
/* Budget, in GPU clock cycles, of every bulk-copy wait of the exact pair
 * kernels launched after this call (shrk_stieltjes_all / _at_points with an
 * exact method, their _dev forms, shrk_stieltjes_at_points_noalloc); returns
 * the previous budget.  Negative restores the default (2e9 cycles, about a
 * second).  Zero makes every such wait give up at once, which exercises the
 * timeout path without a fault: the kernels record the timeout, wait for
 * their own copies in flight and return; host-pointer calls then return
 * SHRK_ETIMEOUT and the allocation-free call writes NaN to every output.
 * Process-wide; meant for tests. */
long long shrk_diag_set_wait_limit(long long cycles);
/* The library's FP64 GEMM on device pointers (column-major, as BLAS dgemm):
 * C = alpha op(A) op(B) + beta C with op = transpose when ta / tb != 0; the
 * kernel the eigensolver's back-transform and the matrix reconstructions
 * use, exported to time it on its own. */
shrk_status shrk_diag_dgemm(int ta, int tb, int64_t m, int64_t n, int64_t k, double alpha,
                            const double* d_a, int64_t lda, const double* d_b, int64_t ldb,
                            double beta, double* d_c, int64_t ldc, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* SHRINKERS_B200_DIAG_H */
