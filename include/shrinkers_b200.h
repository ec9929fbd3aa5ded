/*
 * shrinkers_b200 -- C ABI of the B200 Stieltjes-transform hot path.
 *
 * Drop-in boundary for the `stieltjes` dispatcher of the shrinkers crate
 * (alexisrosuel/shrinkers).  Every entry point below names the reference
 * function it replaces (path:line inside the crate).  Plain pointers and
 * sizes only; no allocation is visible to the caller (device scratch is
 * cached per device and stream inside the library); every function returns
 * a status code and never aborts.  Host-pointer entry points copy the inputs
 * to the device, run on a library-owned stream of the calling thread and
 * copy the outputs back; `_dev` entry points take device pointers and a
 * cudaStream_t (as void*; NULL = the legacy default stream) and are
 * stream-ordered (no host synchronisation unless stated).
 *
 * Conventions (identical to the reference):
 *   raw sum   S(x) = sum_j 1/((x - ev_j) - i*eta)       (src/stieltjes/term.rs:26-31)
 *             Re = sum d/(d^2+eta^2), Im = sum eta/(d^2+eta^2) > 0, d = x - ev_j;
 *   all-points entry points return S(ev_i)/p (mod.rs:601-790 scale_soa/aos);
 *   at-points entry points return raw sums (mod.rs:394-494).
 *   The diagonal term i = j is included (it contributes i/eta).
 */
#ifndef SHRINKERS_B200_H
#define SHRINKERS_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------ status -- */
typedef enum {
  SHRK_OK = 0,
  SHRK_EINVAL = 1,   /* invalid argument (message via shrk_last_error)        */
  SHRK_ECUDA = 2,    /* CUDA runtime error or no usable device                */
  SHRK_ETIMEOUT = 3, /* a bounded device-side wait gave up                    */
  SHRK_ENOTIMPL = 4, /* method outside the GPU path (see shrk_method)         */
  SHRK_ENOMEM = 5    /* device allocation failed                              */
} shrk_status;

/* Method identifiers: same names and order as StieltjesMethod
 * (src/config.rs:19-89).  Exact family (NAIVE .. BLOCKED_HYBRID) -> GPU exact
 * kernels; CHEBCODE* -> GPU treecode with the same ChebPreset; NUFFT -> GPU
 * coarse-grid NUFFT; FFT5/3/2 -> GPU fft5 grid convolution; ADAPTIVE / DST ->
 * its real part with the windowed (or exact) imaginary part;
 * AUTO/SPEED_AUTO/ACCURACY_AUTO -> resolved exactly as
 * config::resolve_auto_method.  At all points TREECODE ("fmm") runs the
 * dyadic Chebyshev FMM (order 16, M2L on the tensor cores, ~1e-6 relative;
 * the reference's multipole treecode is pinned at 1e-3, treecode.rs:357-393),
 * EWALD and HODLR return SHRK_ENOTIMPL (no CPU fallback); at query points
 * all three are the exact per-point sum, as in the reference
 * (mod.rs:265-287). */
typedef enum {
  SHRK_M_NAIVE = 0, SHRK_M_AUTOVEC, SHRK_M_BLOCKED, SHRK_M_BLOCKED_AUTOVEC,
  SHRK_M_BLOCKED_TILED, SHRK_M_BLOCKED_WINDOWED, SHRK_M_BLOCKED_HYBRID,
  SHRK_M_ADAPTIVE, SHRK_M_FFT5, SHRK_M_FFT3, SHRK_M_FFT2, SHRK_M_NUFFT,
  SHRK_M_TREECODE, SHRK_M_CHEBCODE, SHRK_M_CHEBCODE_FAST, SHRK_M_CHEBCODE_XTREME,
  SHRK_M_CHEBCODE_BALANCED, SHRK_M_EWALD, SHRK_M_DST, SHRK_M_AUTO, SHRK_M_HODLR,
  SHRK_M_SPEED_AUTO, SHRK_M_ACCURACY_AUTO
} shrk_method;

/* Arithmetic of the exact kernels.  F64: every pair in FP64.  MIXED: pairs
 * farther apart than shrk_mixed_near_k()*eta in FP32 with compensated
 * accumulation, nearer pairs and all reductions in FP64.  (The reference's
 * own `precision="f32"` path is shrk_stieltjes_all_f32.) */
typedef enum { SHRK_PREC_F64 = 0, SHRK_PREC_MIXED = 1 } shrk_precision;

/* Parallelism of the reference (config.rs:200-226).  The GPU computes the
 * same sums whatever the value; it only selects which reference route the
 * auto policy and the parity tests follow. */
typedef enum { SHRK_PAR_SEQUENTIAL = 0, SHRK_PAR_PARALLEL = 1, SHRK_PAR_AUTO = 2 } shrk_parallelism;

/* ------------------------------------------------------- diagnostics -- */
/* Copies the last error message of the calling thread (NUL-terminated). */
size_t shrk_last_error(char* buf, size_t len);
/* Library version string, e.g. "0.1.0". */
const char* shrk_version(void);
/* Number of visible CUDA devices (0 when none); never fails. */
int shrk_device_count(void);

/* ------------------------------------------------ streams and state -- */
/* Concurrency: calls are thread-safe.  Host-pointer entry points run on a
 * stream of the calling host thread's own; `_dev` entry points on the
 * stream they are given.  The library keeps its device scratch per (device,
 * stream) -- per (device, host thread) for host-pointer calls -- so calls on
 * different streams, from one host thread or several, run concurrently on
 * the GPU; calls on one stream share scratch and run in stream order (the
 * library serialises their host-side setup).
 *
 * shrk_stream_check: waits for `stream` (NULL = the legacy default stream)
 * and reads and clears the device-side error word of the calls issued on
 * it: SHRK_ETIMEOUT if a bounded device-side wait of an earlier `_dev` call
 * on that stream gave up (its outputs are then unspecified), else SHRK_OK.
 * Host-pointer entry points do this themselves before returning. */
shrk_status shrk_stream_check(void* stream);
/* Frees the device scratch and caches the library holds for calls on
 * `stream` on the current device (after waiting for the stream); call it
 * before destroying a stream the library was used with.  A later call on
 * the stream allocates afresh. */
shrk_status shrk_stream_release(void* stream);

/* ---------------------------------------------------- method policy -- */
/* python.rs:321-350 parse_method (all aliases).  SHRK_EINVAL on unknown. */
shrk_status shrk_parse_method(const char* name, int* method_out);
/* config.rs:92-118 StieltjesMethod::name. */
const char* shrk_method_name(int method);
/* config.rs:543-555 resolve_auto_method (+ pareto_autogen.rs:22-86). */
int shrk_resolve_auto_method(int method, int parallel, size_t p);
/* config.rs:565-585 grid_appropriate. */
int shrk_grid_appropriate(int method, size_t p, size_t nq);
/* Near-field radius (in units of eta) of the MIXED exact kernel. */
double shrk_mixed_near_k(void);

/* ------------------------------------------------------ transforms -- */
/* mod.rs:601-790 compute_all_stieltjes: S(ev_i)/p for every i.
 * cutoff_ratio: NaN = CutoffConfig::Disabled, else Enabled{ratio}. */
shrk_status shrk_stieltjes_all(const double* ev, size_t p, double eta, int method,
                               int precision, double cutoff_ratio, int parallelism,
                               double* out_re, double* out_im);
/* Device-pointer form of shrk_stieltjes_all (ev, out_* on the device). */
shrk_status shrk_stieltjes_all_dev(const double* d_ev, size_t p, double eta, int method,
                                   int precision, double cutoff_ratio, int parallelism,
                                   double* d_re, double* d_im, void* stream);
/* mod.rs:805-848 compute_all_stieltjes_f32 (precision="f32",
 * python.rs:820-829): FP32 full-square sum scaled by 1/p in FP32. */
shrk_status shrk_stieltjes_all_f32(const float* ev, size_t p, float eta, int method,
                                   double cutoff_ratio, float* out_re, float* out_im);
/* mod.rs:394-494 compute_stieltjes_at_points: RAW sums at nq query points. */
shrk_status shrk_stieltjes_at_points(const double* q, size_t nq, const double* ev, size_t p,
                                     double eta, int method, int precision, double cutoff_ratio,
                                     int parallelism, double* raw_re, double* raw_im);
shrk_status shrk_stieltjes_at_points_dev(const double* d_q, size_t nq, const double* d_ev,
                                         size_t p, double eta, int method, int precision,
                                         double cutoff_ratio, int parallelism, double* d_re,
                                         double* d_im, void* stream);
/* A target shard of shrk_stieltjes_all_dev (all_points = 1) or of
 * shrk_stieltjes_at_points_dev (all_points = 0), for a call split over
 * several GPUs by targets with the spectrum replicated: the values at
 * d_tgt[0..nt) computed with the policies of the whole call.  all_points:
 * d_tgt points into d_ev (a slice of the spectrum), nq_total = p, outputs
 * S/p.  At points: nq_total = the whole call's query count, which sets the
 * treecode's grid leaf capacity (mod.rs:475-489) and the auto method's grid
 * rule, so every shard uses the tree of the whole call; raw sums.  The
 * treecode and grid methods evaluate each target independently of the
 * others, so the shards assemble into the single call's values bit for bit;
 * the exact methods' split reductions depend on the launch shape (1e-13).
 * The "treecode" method's all-points form (the FMM) evaluates every point
 * and keeps the slice. */
shrk_status shrk_stieltjes_shard_dev(const double* d_tgt, size_t nt, size_t nq_total,
                                     int all_points, const double* d_ev, size_t p, double eta,
                                     int method, int precision, double cutoff_ratio,
                                     int parallelism, double* d_re, double* d_im, void* stream);
/* Allocation-free form of shrk_stieltjes_at_points_dev for the exact method
 * (no counterpart in the reference): the same RAW sums, FP64 or MIXED, with
 * every device temporary taken from one static array of
 * SHRK_NOALLOC_SCRATCH_BYTES inside the library, for callers that cannot let
 * a library allocate or free device memory (a framework holding the device
 * in its own pool, latency-bound loops, fixed-footprint services).
 *   - Limits: nq <= SHRK_NOALLOC_MAX_POINTS, p <= SHRK_NOALLOC_MAX_EIGS;
 *     larger sizes return SHRK_EINVAL with a message naming the limit.
 *   - The first call on each device does a one-time setup (it looks up the
 *     array's device address, which may also load the module onto the
 *     device); make that first call before any stream capture.  The address
 *     is kept for the life of the process: do not use this entry point on a
 *     device after cudaDeviceReset (the module may then load elsewhere).
 *   - Every call on a device shares the array.  Calls that overlap -- on
 *     different streams, or enqueued concurrently from several host threads
 *     -- race on it and corrupt each other's results; serialise them (for
 *     instance one stream, one thread at a time).
 *   - Stream-ordered, no host synchronisation: if a bounded device-side wait
 *     gives up, every output of that call is NaN. */
#define SHRK_NOALLOC_SCRATCH_BYTES (8u << 20)
#define SHRK_NOALLOC_MAX_POINTS 262144
#define SHRK_NOALLOC_MAX_EIGS 16777216
shrk_status shrk_stieltjes_at_points_noalloc(const double* d_q, size_t nq, const double* d_ev,
                                             size_t p, double eta, int precision, double* d_re,
                                             double* d_im, void* stream);
/* autovec.rs:38-77 compute_all_stieltjes_with_deriv (python.rs:758-781):
 * RAW value and derivative w.r.t. the query point at every eigenvalue. */
shrk_status shrk_stieltjes_with_deriv(const double* ev, size_t p, double eta, double* re,
                                      double* im, double* dre, double* dim);

/* Batched uneven spectra (no reference counterpart; replaces a host loop of
 * compute_all_stieltjes calls): spectrum s is ev[offsets[s] .. offsets[s+1]),
 * evaluated at its own eta[s]; outputs are scaled by 1/p_s and laid out like
 * the input.  One persistent launch pulls (spectrum, target tile, source
 * split) items from a device queue. */
shrk_status shrk_stieltjes_batched(const double* ev, const int64_t* offsets, size_t n_spectra,
                                   const double* eta, int precision, double* out_re,
                                   double* out_im);
shrk_status shrk_stieltjes_batched_dev(const double* d_ev, const int64_t* d_offsets,
                                       size_t n_spectra, const double* d_eta, int precision,
                                       double* d_re, double* d_im, void* stream);
/* Autotuner of the batched launch (no reference counterpart).  For each
 * p-bucket [2^8,2^9), ..., [2^14,2^15), [2^15,inf) it times every candidate
 * (targets per thread R in {2,4}, source split SL in {1024,...,8192}) on a
 * synthetic batch of that bucket and keeps the fastest; table receives
 * (R, SL) per bucket, 16 ints.  Batched calls plan with a table the
 * autotuner chose on a B200 until this runs (with force != 0, or force == 0
 * before any batched call on the device) or shrk_batched_set_tune installs
 * another; with the environment variable SHRK_BATCHED_AUTOTUNE=1 the first
 * batched call tunes instead.  With force == 0 on a device that already has
 * a table, table receives it without tuning.  Spectra of the batched entry
 * points hold at most 16 777 216 values each. */
shrk_status shrk_batched_autotune(int precision, int force, int32_t* table);
/* Installs a (R, SL) table of the layout shrk_batched_autotune returns, for
 * `precision` on the current device, e.g. one saved from an earlier process
 * so that no call pays for tuning; R in {2, 4}, SL in {1024, 2048, 4096,
 * 8192}, else SHRK_EINVAL.  Later batched calls plan with it. */
shrk_status shrk_batched_set_tune(int precision, const int32_t* table);

/* Adjoint of m(z_j) = (1/p) sum_i 1/(ev_i - z_j), z_j = ev_j + i*eta (the
 * -conj(S)/p convention; no reference counterpart).  Given cotangents
 * g_j = g_re[j] + i g_im[j] of L = sum_j Re(conj(g_j) m_j), writes
 * grad[k] = dL/d ev_k including the dependence of z_k on ev_k. */
shrk_status shrk_stieltjes_adjoint(const double* ev, size_t p, double eta, const double* g_re,
                                   const double* g_im, int precision, double* grad);
shrk_status shrk_stieltjes_adjoint_dev(const double* d_ev, size_t p, double eta,
                                       const double* d_g_re, const double* d_g_im, int precision,
                                       double* d_grad, void* stream);
/* The same gradient with every source sum evaluated by the ChebCode tree of
 * `method` (CHEBCODE, CHEBCODE_FAST, CHEBCODE_XTREME, CHEBCODE_BALANCED:
 * the presets of chebcode.rs:926-998; no reference counterpart): leaves are
 * summed exactly, accepted nodes through Chebyshev node weights of the
 * charges 1, g_re and g_im.  FP64 throughout. */
shrk_status shrk_stieltjes_adjoint_treecode(const double* ev, size_t p, double eta,
                                            const double* g_re, const double* g_im, int method,
                                            double* grad);
shrk_status shrk_stieltjes_adjoint_treecode_dev(const double* d_ev, size_t p, double eta,
                                                const double* d_g_re, const double* d_g_im,
                                                int method, double* d_grad, void* stream);

/* chebcode.rs:1312-1361 ChebCodeBatch::evaluate_many (gamma sweeps): one tree
 * built for the preset `method` (CHEBCODE*: its theta, order and leaf
 * capacity; the far field is FP64 whatever the preset), then RAW sums at
 * every eigenvalue for each of the n_eta etas, evaluated two etas per
 * traversal (chebcode.rs:836-915: a node is accepted only when both etas
 * accept it).  out_re / out_im: n_eta x p, row-major, input order; etas must
 * be positive and finite. */
shrk_status shrk_chebcode_evaluate_many(const double* ev, size_t p, const double* etas,
                                        size_t n_eta, int method, double* out_re,
                                        double* out_im);
shrk_status shrk_chebcode_evaluate_many_dev(const double* d_ev, size_t p, const double* d_etas,
                                            size_t n_eta, int method, double* d_re, double* d_im,
                                            void* stream);

/* mod.rs:304-319 compute_stieltjes_scaled_ray: RAW sums at z_i = ev_i(1 + i*scale),
 * i.e. every point has its own eta_i = scale*ev_i.  Exact FP64 pair sums (the
 * reference takes the exact per-point route for every method here). */
shrk_status shrk_stieltjes_scaled_ray(const double* ev, size_t p, double scale, double* raw_re,
                                      double* raw_im);
shrk_status shrk_stieltjes_scaled_ray_dev(const double* d_ev, size_t p, double scale,
                                          double* d_re, double* d_im, void* stream);

/* Dyadic Chebyshev FMM (no reference counterpart: the crate's ChebCode is a
 * treecode, reproduced by the chebcode methods): S(ev_i)/p at every
 * eigenvalue, input order, from P2M / M2M / M2L / L2L / L2P on a dyadic tree
 * with leaves of at most 48 eigenvalues and the leaf plus its neighbours
 * summed directly in FP64.  order = Chebyshev points per box, 4..16; the
 * error vs the exact sums falls from ~1e-9 (10) to FP64 round-off (16).
 * m2l = 0: every stage in FP64; m2l = 1: the M2L stage on the tensor cores
 * (tcgen05, TF32 x3 products accumulated in FP32, ~1e-7 relative). */
shrk_status shrk_stieltjes_fmm(const double* ev, size_t p, double eta, int order, int m2l,
                               double* out_re, double* out_im);
shrk_status shrk_stieltjes_fmm_dev(const double* d_ev, size_t p, double eta, int order, int m2l,
                                   double* d_re, double* d_im, void* stream);

/* fft5.rs:568-590 compute_all_stieltjes_fft5_with_options: RAW sums (not
 * scaled by 1/p) at every eigenvalue from the fft5 grid convolution with the
 * Fft5Options knobs (fft5.rs:213-249): order = stencil nodes, 2/4/6/8 for
 * Linear/Cubic/Quintic/Heptic (the methods "fft5"/"fft3"/"fft2" use 8);
 * m_override = forced grid size, 0 for the rule dx <= eta/8, m >= 8p, at
 * most 2^20; pad = max(pad_eta_mult*eta, pad_range_frac*raw_range) (defaults
 * 1000 and 0.75).  The first and last entries bound the grid, as in the
 * reference (ascending input expected).  Any grid size up to 2^21, or a power
 * of two up to 2^22 (rustfft plans any length, fftplan.rs:21-28; here a size
 * that is not a power of two runs Bluestein's chirp-z form over the
 * power-of-two transform); SHRK_ENOTIMPL above that. */
shrk_status shrk_stieltjes_fft5_with_options(const double* ev, size_t p, double eta, int order,
                                             size_t m_override, double pad_eta_mult,
                                             double pad_range_frac, double* raw_re,
                                             double* raw_im);
shrk_status shrk_stieltjes_fft5_with_options_dev(const double* d_ev, size_t p, double eta,
                                                 int order, size_t m_override,
                                                 double pad_eta_mult, double pad_range_frac,
                                                 double* d_re, double* d_im, void* stream);

/* The NUFFT (nufft.rs:164-220) in its two stages, for a point-sharded
 * transform over several GPUs (no reference counterpart: the reference runs
 * in one process).  The splat is linear in the sources, so ranks that splat
 * disjoint shards of one spectrum onto the same grid and sum their densities
 * (one all-reduce of m <= 65 536 doubles) hold the density of the whole
 * spectrum; each then evaluates its own queries.
 *
 * shrk_nufft_grid: the grid of nufft.rs:106-126 (with the padding of
 * fft5.rs:339-361) for a spectrum whose first and last entries, in the
 * caller's order, are first / last: m cells from lo, spacing dx (negative
 * for descending input).  Host only.
 * shrk_nufft_density_dev: the order-4 density of ns sources (any order;
 * sorted on the device when needed) on the grid (m, lo, dx) into
 * d_density[m]; ns = 0 gives zeros.
 * shrk_nufft_eval_dev: the packed convolution of d_density with the kernel
 * pair, and RAW sums at nq device queries.
 * Splatting every source of a spectrum and evaluating gives the same values,
 * bit for bit, as shrk_stieltjes_at_points_dev with the nufft method. */
shrk_status shrk_nufft_grid(double first, double last, double eta, int64_t* m, double* lo,
                            double* dx);
shrk_status shrk_nufft_density_dev(const double* d_src, size_t ns, int64_t m, double lo,
                                   double dx, double* d_density, void* stream);
shrk_status shrk_nufft_eval_dev(const double* d_density, int64_t m, double lo, double dx,
                                double eta, const double* d_q, size_t nq, double* d_re,
                                double* d_im, void* stream);

/* --------------------------------------------------- matrix front-end -- */
/* Matrices are row-major p x p (p <= 46340), eigenvectors are their
 * columns.  The eigendecomposition is this library's own on the device
 * (Householder tridiagonalisation, multisection, inverse iteration; the
 * reference's symmetric_eigh, pipeline/mod.rs:502-585, is a Jacobi
 * iteration; eigenvector signs are arbitrary in both).  Output pointers
 * marked "may be NULL" are skipped when NULL. */
/* pipeline/mod.rs:502-585 symmetric_eigh: ascending eigenvalues (p) and
 * the eigenvectors as columns (p x p, may be NULL). */
shrk_status shrk_symmetric_eigh(const double* matrix, size_t p, double* eigenvalues,
                                double* eigenvectors);
/* pipeline/mod.rs:197-242 clean_eigensystem: from a sample eigensystem
 * (eigenvector columns parallel to `eigenvalues`, any order) and c: the
 * cleaned covariance (p x p), the eigenvectors with columns sorted by
 * descending eigenvalue (may be NULL), the RIE eigenvalues (descending),
 * the squared angular overlaps (overlaps.rs:26-46) and the noise level
 * sigma2 (MP-median-corrected median, detection.rs:97-104). */
shrk_status shrk_clean_eigensystem(const double* eigenvectors, const double* eigenvalues,
                                   size_t p, double c, double* covariance,
                                   double* sorted_eigenvectors, double* rie_eigenvalues,
                                   double* overlaps, double* sigma2);
/* pipeline/mod.rs:244-329 clean_covariance_matrix / clean_correlation_matrix
 * (one estimator): eigendecompose `matrix`, then clean_eigensystem;
 * renormalize != 0 rescales the result to unit diagonal
 * (python.rs:729-731). */
shrk_status shrk_clean_covariance_matrix(const double* matrix, size_t p, double c,
                                         int renormalize, double* covariance,
                                         double* eigenvectors, double* rie_eigenvalues,
                                         double* overlaps, double* sigma2);
/* pipeline/mod.rs:331-341 renormalize_to_unit_diagonal: D^-1/2 S D^-1/2, or
 * S unchanged when a diagonal entry is not positive. */
shrk_status shrk_renormalize_to_unit_diagonal(const double* matrix, size_t p, double* out);
/* pipeline/mod.rs:409-464 precision_from_eigensystem: inverse nonlinear
 * shrinkage (method 0 QIS, 1 LIS, 2 GIS) of the sorted spectrum and
 * Omega = U diag(precision_ev) U^T; eigenvalues must be strictly positive,
 * c in (0, 1].  precision_ev / covariance_ev follow the descending sample
 * eigenvalues. */
shrk_status shrk_precision_from_eigensystem(const double* eigenvectors, const double* eigenvalues,
                                            size_t p, double c, int method, double* precision,
                                            double* sorted_eigenvectors, double* precision_ev,
                                            double* covariance_ev, double* smoothing);
/* pipeline/mod.rs:466-478 estimate_precision_matrix: eigendecompose, then
 * precision_from_eigensystem. */
shrk_status shrk_estimate_precision_matrix(const double* matrix, size_t p, double c, int method,
                                           double* precision, double* eigenvectors,
                                           double* precision_ev, double* covariance_ev,
                                           double* smoothing);
/* Device-pointer forms of shrk_symmetric_eigh, shrk_clean_covariance_matrix
 * and shrk_estimate_precision_matrix: the matrix and every array output on
 * the device (the p x p outputs, and the p-vectors: eigenvalues, RIE
 * eigenvalues, overlaps, precision_ev, covariance_ev; "may be NULL" as in
 * the host forms), the scalar outputs (sigma2, smoothing) on the host.  The
 * calls wait for the work queued on `stream` before reading the matrix, and
 * `stream` waits for their outputs; they synchronise internally (the steps
 * between the kernels are host arithmetic on the spectrum). */
shrk_status shrk_symmetric_eigh_dev(const double* d_matrix, size_t p, double* d_eigenvalues,
                                    double* d_eigenvectors, void* stream);
shrk_status shrk_clean_covariance_matrix_dev(const double* d_matrix, size_t p, double c,
                                             int renormalize, double* d_covariance,
                                             double* d_eigenvectors, double* d_rie_eigenvalues,
                                             double* d_overlaps, double* sigma2, void* stream);
shrk_status shrk_estimate_precision_matrix_dev(const double* d_matrix, size_t p, double c,
                                               int method, double* d_precision,
                                               double* d_eigenvectors, double* d_precision_ev,
                                               double* d_covariance_ev, double* smoothing,
                                               void* stream);

/* ------------------------------------------------------- consumers -- */
/* deconvolution/inverse.rs:156-269 inverse_nonlinear_shrinkage (RmtConfig::new:
 * exact sums): method 0 QIS, 1 LIS, 2 GIS.  precision_ev / covariance_ev hold
 * p entries in input order; *smoothing receives the bandwidth h; theta and
 * htheta (p entries each) may be NULL.  Eigenvalues must be strictly positive
 * and c in (0, 1]. */
shrk_status shrk_inverse_nonlinear_shrinkage(const double* ev, size_t p, double c, int method,
                                             double* precision_ev, double* covariance_ev,
                                             double* smoothing, double* theta, double* htheta);
/* shrinkage.rs:22-34 shrinkage_factor (pure host arithmetic). */
double shrk_shrinkage_factor(double lambda, double c, double m_re, double m_im);
/* estimation.rs:48-56 inverse_bbp; estimation.rs:37-39 bbp_threshold. */
double shrk_inverse_bbp(double lambda_hat, double gamma, double sigma2);
double shrk_bbp_threshold(double gamma, double sigma2);
/* detection.rs:75-83 mp_median_factor. */
double shrk_mp_median_factor(double gamma);
/* detection.rs:134-153 detect_spikes_bema on an ASCENDING spectrum.
 * spike_indices must hold p entries; *k receives the count. */
shrk_status shrk_detect_spikes_bema(const double* sorted, size_t p, double gamma, double margin,
                                    size_t* k, int64_t* spike_indices, double* bulk_edge,
                                    double* sigma2);
/* estimation.rs:75-90 ledoit_wolf_shrinkage: xi_i from the GPU transform
 * with the LW map fused into the FP64 reduction epilogue.  eta NaN ->
 * 0.4/sqrt(p) (mod.rs:150-153).  Input order preserved. */
shrk_status shrk_ledoit_wolf_shrinkage(const double* ev, size_t p, double c, int method,
                                       int precision, int parallelism, double eta, double* xi);
/* shrinkage.rs:60-84 rie_shrinkage (trace-rescaled). */
shrk_status shrk_rie_shrinkage(const double* ev, size_t p, double c, int method, int precision,
                               int parallelism, double* xi);
/* deconvolution/mod.rs:116-259 spectral_deconvolution with the MP inversion
 * fused into the grid transform's epilogue.  eta/lambda_min/lambda_max NaN =
 * None.  out7 holds 7*n_points doubles: lambda_grid, density, w_re,
 * sample_stieltjes_real/imag, population_stieltjes_real/imag. */
shrk_status shrk_spectral_deconvolution(const double* ev, size_t p, double c, size_t n_points,
                                        double eta, double lambda_min, double lambda_max,
                                        int method, int precision, int parallelism,
                                        double cutoff_ratio, double* out7);
/* population.rs:72-116 estimate_population_eigenvalues (RmtConfig::new:
 * Blocked, sequential, eta = 0.4/sqrt(p_bulk)).  spikes/spike_sample hold p
 * entries (descending on return), bulk_population/bulk_sample p entries
 * (p - k written, ascending in the sample eigenvalue). */
shrk_status shrk_estimate_population_eigenvalues(const double* ev, size_t p, double c,
                                                 double margin, int precision, size_t* k,
                                                 double* spikes, double* spike_sample,
                                                 double* bulk_edge, double* sigma2,
                                                 double* bulk_population, double* bulk_sample);
/* hybrid.rs:96-138 deconvolve_spiked (eta NaN -> 0.1/sqrt(p_bulk)). */
shrk_status shrk_deconvolve_spiked(const double* ev, size_t p, double c, size_t n_points,
                                   double eta, double margin, int method, int precision,
                                   int parallelism, double cutoff_ratio, size_t* k,
                                   double* spikes, double* spike_sample, double* bulk_edge,
                                   double* sigma2, double* out7);

#ifdef __cplusplus
}
#endif

#endif /* SHRINKERS_B200_H */
