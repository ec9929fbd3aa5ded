// FFT grid convolution for the Stieltjes transform on sm_100a: the fft5
// family (fft5 / fft3 / fft2, and the real part of adaptive and dst) and the
// coarse-grid NUFFT preset over the same pipeline.
//
// Replaces the dual-convolution core of src/stieltjes/fft5.rs
// (Fft5Options 213-249, lagrange_weights 136-164, splat 175-185 / 259-318,
// fft_convolution 325-432, interp_at 191-211, interpolate_grid 440-476, entry
// points 559-625), the packing helpers of src/stieltjes/fftplan.rs:43-76 and
// the NUFFT policy of src/stieltjes/nufft.rs (33-126, entry points 164-220).
// Pipeline (all FP64), stencil width N = 2/4/6/8 a template parameter:
//
//   1. weights      one thread per source: stencil cell i0 = floor((v-lo)/dx)
//                   and the N Lagrange weights of t = pos - i0.
//   2. gather+pack  one thread per grid cell; a CTA of 256 cells finds the
//                   run of sources whose stencils touch it (two warp-wide
//                   searches), stages their cells in shared memory, and each
//                   thread adds its sources' weights in ascending source
//                   order -- the order of the reference's sequential splat,
//                   so the density is the same sums, without atomics.  Grids
//                   with more than two sources per cell (the NUFFT's coarse
//                   grid) use one warp per cell instead.  Then
//                   packed[c] = density[c] + i x_c/(x_c^2 + eta^2).
//   3. fft          four-step FFT m = m1*m2 (m1, m2 <= 2048): column FFTs of
//                   length m1 in shared memory with the inter-pass twiddle,
//                   then row FFTs of length m2.  Twiddles and the analytic
//                   even-kernel spectrum are device tables cached per grid.
//   4. spectral     unpack the two real spectra (conjugate symmetry), form
//                   Im_hat + i Re_hat = D*K_even + i D*K_odd.
//   5. fft          inverse transform.
//   6. interp       N-point interpolation at the query points, 1/m scale,
//                   fused FP64 epilogue.
#include "common.cuh"
#include "epilogue.cuh"
#include "internal.h"

#include <cmath>
#include <map>
#include <string>

namespace shrk {

namespace {

// nufft.rs:33-58
constexpr double NUFFT_PAD_ETA_MULT = 2000.0;
constexpr double NUFFT_PAD_RANGE_FRAC = 0.75;
constexpr double NUFFT_RESOLUTION = 5.0;
constexpr size_t NUFFT_MIN_GRID = 8192;
constexpr size_t NUFFT_MAX_GRID = 65536;

// fft5.rs:345-353: dx <= eta/8, m >= 8p, at most 2^20 cells.
constexpr size_t FFT5_MAX_AUTO_GRID = (size_t)1 << 20;

constexpr int FFT_MAXL = 2048;                  // longest in-shared-memory transform
constexpr int64_t FFT_MAX_M = (int64_t)FFT_MAXL * FFT_MAXL;

size_t next_pow2(size_t n) {  // mod.rs:529-535
  size_t p = 1;
  while (p < n) p <<= 1;
  return p;
}

// Rust's saturating float -> usize cast (NaN and negatives -> 0).
size_t sat_usize(double v) {
  if (!(v > 0.0)) return 0;
  if (v >= 18446744073709551616.0) return SIZE_MAX;
  return (size_t)v;
}

// fft5.rs:136-164 lagrange_weights<N>, operation order preserved.
template <int N>
__device__ __forceinline__ void lagrange(double t, double w[N]) {
  const double q = (double)(N / 2);
  double pref[N], suf[N], acc = 1.0;
#pragma unroll
  for (int j = 0; j < N; ++j) {
    pref[j] = acc;
    acc *= t - (double)j + q - 1.0;
  }
  acc = 1.0;
#pragma unroll
  for (int j = N - 1; j >= 0; --j) {
    suf[j] = acc;
    acc *= t - (double)j + q - 1.0;
  }
#pragma unroll
  for (int j = 0; j < N; ++j) {
    double den = 1.0;
#pragma unroll
    for (int l = 0; l < N; ++l)
      if (l != j) den *= (double)(j - l);
    w[j] = pref[j] * suf[j] / den;
  }
}

// floor((v - lo)/dx) as a cell index clamped to [-N - 1, m + N] (every slot
// of a source beyond that range lands on the same edge cell), and the
// fraction t = pos - floor(pos) of the unclamped position.
template <int N>
__device__ __forceinline__ int64_t cell_of(double v, double lo, double dx, int64_t m, double* t) {
  const double pos = (v - lo) / dx;
  const double fl = floor(pos);
  *t = pos - fl;
  const double c = fmin(fmax(fl, -(double)N - 1.0), (double)(m + N));
  return (int64_t)c;
}

struct GridArgs {
  const double* src;  // ascending
  int64_t ns;
  int rev;            // 1: visit the sources in descending order (dx < 0)
  double lo, dx, eta;
  int64_t m;
  int* cell;          // per visited source: stencil cell, clamped to [-N, m + N]
  double* w;          // per visited source: the N stencil weights, SoA [N][ns]
  double2* packed;
};

// Per source: stencil cell and weights (fft5.rs:175-185).  The visiting order
// makes cell[] non-decreasing.
template <int N>
__global__ void splat_weights_kernel(const GridArgs a) {
  const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= a.ns) return;
  const double v = a.rev ? a.src[a.ns - 1 - j] : a.src[j];
  double t;
  int64_t i0 = cell_of<N>(v, a.lo, a.dx, a.m, &t);
  double w[N];
  lagrange<N>(t, w);
  i0 = i0 < -N ? -N : (i0 > a.m + N ? a.m + N : i0);
  a.cell[j] = (int)i0;
#pragma unroll
  for (int k = 0; k < N; ++k) a.w[(int64_t)k * a.ns + j] = w[k];
}

// First source index j with cell[j] >= key (ns if none), cell[] non-
// decreasing: a 32-way search where every lane probes one point per round.
__device__ int64_t warp_first_ge(const int* __restrict__ cell, int64_t ns, int key, int lane) {
  int64_t lo = 0, hi = ns;  // the answer lies in [lo, hi]
  while (hi - lo > 32) {
    const int64_t step = (hi - lo + 31) / 32;
    const int64_t q = lo + (int64_t)lane * step;
    const bool less = q < hi && cell[q] < key;
    const int cnt = __popc(__ballot_sync(0xffffffffu, less));
    const int64_t nlo = cnt > 0 ? lo + (int64_t)(cnt - 1) * step + 1 : lo;
    hi = min(hi, lo + (int64_t)cnt * step);
    lo = nlo;
  }
  const int64_t q = lo + lane;
  const bool less = q < hi && cell[q] < key;
  return lo + __popc(__ballot_sync(0xffffffffu, less));
}

// First index in [lo, hi) of a non-decreasing array with value >= key.
__device__ __forceinline__ int64_t first_ge(const int* __restrict__ v, int64_t lo, int64_t hi,
                                            int key) {
  while (lo < hi) {
    const int64_t mid = (lo + hi) >> 1;
    if (v[mid] < key) lo = mid + 1;
    else hi = mid;
  }
  return lo;
}

constexpr int GATHER_T = 256;     // grid cells per CTA
constexpr int GATHER_CAP = 4096;  // source cells staged in shared memory

// Steps 1+pack: the density of cell c is the sum of weight k = c + N/2 - 1 - i0
// over the sources with i0 in [c - N/2, c + N/2 - 1] (fft5.rs:175-185), in
// ascending source order; the two edge cells also collect every clamped slot.
// Then packed[c] = density[c] + i x_c/(x_c^2 + eta^2) (fft5.rs:364-376).
template <int N>
__global__ void __launch_bounds__(GATHER_T) splat_gather_kernel(const GridArgs a) {
  constexpr int H = N / 2;
  __shared__ int s_cell[GATHER_CAP];
  __shared__ int64_t s_run[2];
  const int64_t m = a.m;
  const int64_t c0 = (int64_t)blockIdx.x * GATHER_T;
  const int64_t c = c0 + threadIdx.x;
  if (threadIdx.x < 32) {
    const int lane = threadIdx.x;
    const int64_t clast = min(c0 + GATHER_T - 1, m - 1);
    const int64_t jA = warp_first_ge(a.cell, a.ns, (int)(c0 - H), lane);
    const int64_t jB = warp_first_ge(a.cell, a.ns, (int)(clast + H), lane);
    if (lane == 0) {
      s_run[0] = jA;
      s_run[1] = jB;
    }
  }
  __syncthreads();
  const int64_t jA = s_run[0], jB = s_run[1];
  const int64_t n = jB - jA;
  const bool staged = n <= GATHER_CAP;
  if (staged)
    for (int64_t i = threadIdx.x; i < n; i += GATHER_T) s_cell[i] = a.cell[jA + i];
  __syncthreads();
  if (c >= m) return;
  double dens = 0.0;
  if (c > 0 && c < m - 1) {
    int64_t j0, j1;
    if (staged) {
      j0 = jA + first_ge(s_cell, 0, n, (int)c - H);
      j1 = jA + first_ge(s_cell, j0 - jA, n, (int)c + H);
    } else {
      j0 = first_ge(a.cell, jA, jB, (int)c - H);
      j1 = first_ge(a.cell, j0, jB, (int)c + H);
    }
    for (int64_t j = j0; j < j1; ++j) {
      const int i0 = staged ? s_cell[j - jA] : a.cell[j];
      dens += a.w[(int64_t)((int)c + H - 1 - i0) * a.ns + j];
    }
  } else {
    // edge cell: every slot whose clamped index lands here, sources then slots
    const int64_t j0 = (c == 0) ? 0 : first_ge(a.cell, 0, a.ns, (int)(m - 1 - H));
    const int64_t j1 = (c == 0) ? first_ge(a.cell, 0, a.ns, H) : a.ns;
    for (int64_t j = j0; j < j1; ++j) {
      const int i0 = a.cell[j];
#pragma unroll
      for (int k = 0; k < N; ++k) {
        int64_t cell = (int64_t)i0 - H + 1 + k;
        cell = cell < 0 ? 0 : (cell > m - 1 ? m - 1 : cell);
        if (cell == c) dens += a.w[(int64_t)k * a.ns + j];
      }
    }
  }
  const int64_t half = m / 2;
  const double sd = (c <= half) ? (double)c : (double)c - (double)m;
  const double x = sd * a.dx;
  const double denom = x * x + a.eta * a.eta;
  a.packed[c] = make_double2(dens, x / denom);
}

// The same density for grids with many sources per cell (the NUFFT's coarse
// grid): one warp per cell, lanes stride the cell's source run and a fixed
// butterfly adds the lane sums (deterministic; the addition order is not the
// sequential one).
template <int N>
__global__ void splat_gather_warp_kernel(const GridArgs a) {
  constexpr int H = N / 2;
  const int64_t c = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (c >= a.m) return;  // whole warps exit together
  const int64_t m = a.m;
  double dens = 0.0;
  if (c > 0 && c < m - 1) {
    const int64_t j0 = warp_first_ge(a.cell, a.ns, (int)c - H, lane);
    const int64_t j1 = warp_first_ge(a.cell, a.ns, (int)c + H, lane);
    for (int64_t j = j0 + lane; j < j1; j += 32) {
      const int k = (int)c + H - 1 - a.cell[j];
      dens += a.w[(int64_t)k * a.ns + j];
    }
  } else {
    const int64_t j0 = (c == 0) ? 0 : warp_first_ge(a.cell, a.ns, (int)(m - 1 - H), lane);
    const int64_t j1 = (c == 0) ? warp_first_ge(a.cell, a.ns, H, lane) : a.ns;
    for (int64_t j = j0 + lane; j < j1; j += 32) {
      const int i0 = a.cell[j];
#pragma unroll
      for (int k = 0; k < N; ++k) {
        int64_t cell = (int64_t)i0 - H + 1 + k;
        cell = cell < 0 ? 0 : (cell > m - 1 ? m - 1 : cell);
        if (cell == c) dens += a.w[(int64_t)k * a.ns + j];
      }
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) dens += __shfl_xor_sync(0xffffffffu, dens, o);
  if (lane == 0) {
    const int64_t half = m / 2;
    const double sd = (c <= half) ? (double)c : (double)c - (double)m;
    const double x = sd * a.dx;
    const double denom = x * x + a.eta * a.eta;
    a.packed[c] = make_double2(dens, x / denom);
  }
}

// ---------------------------------------------------------------- FFT --
__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

__device__ __forceinline__ unsigned bitrev(unsigned v, int bits) {
  return bits == 0 ? 0u : (__brev(v) >> (32 - bits));
}

// Transforms per CTA for length L: G*L <= FFT_MAXL.
__host__ __device__ __forceinline__ int fft_group(int L) {
  return L <= 512 ? 4 : (L <= 1024 ? 2 : 1);
}

// Radix-2 decimation-in-time transform of G rows of length L in shared
// memory (rows already in bit-reversed order).  tw: table of
// (cos 2 pi j/m, sin 2 pi j/m), sign -1 forward, +1 inverse.
__device__ void smem_fft(double2* buf, int G, int L, int64_t m, const double2* tw, double sign) {
  for (int len = 2; len <= L; len <<= 1) {
    const int half = len >> 1;
    const int64_t step = m / len;
    const int nb = G * (L >> 1);
    for (int b = threadIdx.x; b < nb; b += blockDim.x) {
      const int g = b / (L >> 1);
      const int r = b % (L >> 1);
      const int grp = r / half, k = r % half;
      const int i = g * L + grp * len + k;
      const double2 t = tw[(int64_t)k * step];
      const double2 w = make_double2(t.x, sign * t.y);
      const double2 u = buf[i];
      const double2 v = cmul(buf[i + half], w);
      buf[i] = make_double2(u.x + v.x, u.y + v.y);
      buf[i + half] = make_double2(u.x - v.x, u.y - v.y);
    }
    __syncthreads();
  }
}

// Pass 1: Y[k1*m2 + n2] = W_m^{n2 k1} * sum_n1 x[m2 n1 + n2] W_m1^{n1 k1}.
__global__ void __launch_bounds__(256) fft_pass1(const double2* __restrict__ x,
                                                 double2* __restrict__ y, int m1, int b1, int m2,
                                                 int64_t m, const double2* __restrict__ tw,
                                                 double sign) {
  __shared__ double2 buf[FFT_MAXL];
  const int G = fft_group(m1);
  const int n2_0 = blockIdx.x * G;
  for (int e = threadIdx.x; e < G * m1; e += blockDim.x) {
    const int n1 = e / G, g = e % G;
    if (n2_0 + g < m2) buf[g * m1 + bitrev((unsigned)n1, b1)] = x[(int64_t)m2 * n1 + n2_0 + g];
  }
  __syncthreads();
  smem_fft(buf, G, m1, m, tw, sign);
  for (int e = threadIdx.x; e < G * m1; e += blockDim.x) {
    const int k1 = e / G, g = e % G;
    const int n2 = n2_0 + g;
    if (n2 >= m2) continue;
    const double2 t = tw[((int64_t)n2 * k1) % m];
    y[(int64_t)k1 * m2 + n2] = cmul(buf[g * m1 + k1], make_double2(t.x, sign * t.y));
  }
}

// Pass 2: X[k1 + m1 k2] = sum_n2 Y[k1*m2 + n2] W_m2^{n2 k2}.
__global__ void __launch_bounds__(256) fft_pass2(const double2* __restrict__ y,
                                                 double2* __restrict__ x, int m1, int m2, int b2,
                                                 int64_t m, const double2* __restrict__ tw,
                                                 double sign) {
  __shared__ double2 buf[FFT_MAXL];
  const int G = fft_group(m2);
  const int k1_0 = blockIdx.x * G;
  for (int e = threadIdx.x; e < G * m2; e += blockDim.x) {
    const int g = e / m2, n2 = e % m2;
    if (k1_0 + g < m1) buf[g * m2 + bitrev((unsigned)n2, b2)] = y[(int64_t)(k1_0 + g) * m2 + n2];
  }
  __syncthreads();
  smem_fft(buf, G, m2, m, tw, sign);
  for (int e = threadIdx.x; e < G * m2; e += blockDim.x) {
    const int k2 = e / G, g = e % G;
    if (k1_0 + g >= m1) continue;
    x[(int64_t)(k1_0 + g) + (int64_t)m1 * k2] = buf[g * m2 + k2];
  }
}

// fftplan.rs:43-76: unpack D (density) and K (odd kernel) from the packed
// forward transform, multiply, repack as Im_hat + i Re_hat.
__global__ void spectral_kernel(const double2* __restrict__ C, const double* __restrict__ ke,
                                double2* __restrict__ out, int64_t m) {
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= m) return;
  const double2 ck = C[k];
  const double2 cn = C[(m - k) % m];
  const double2 cnc = make_double2(cn.x, -cn.y);
  const double2 s = make_double2(ck.x + cnc.x, ck.y + cnc.y);
  const double2 df = make_double2(ck.x - cnc.x, ck.y - cnc.y);
  const double2 D = make_double2(0.5 * s.x, 0.5 * s.y);
  const double2 K = make_double2(0.5 * df.y, -0.5 * df.x);  // (-0.5 i) * df
  const double ih_re = D.x * ke[k], ih_im = D.y * ke[k];
  const double2 rh = cmul(D, K);
  out[k] = make_double2(ih_re - rh.y, ih_im + rh.x);
}

struct InterpArgs {
  const double* q;
  int64_t nq;
  const double2* grid;
  int64_t m;
  double lo, dx, inv_m;
  Epilogue epi;
};

// fft5.rs:191-211 interp_at<N> + 440-476: re <- .im, im <- .re, times 1/m.
template <int N>
__global__ void interp_kernel(const InterpArgs a) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= a.nq) return;
  const double qv = a.q[t];
  double tt;
  const int64_t i0 = cell_of<N>(qv, a.lo, a.dx, a.m, &tt);
  double w[N];
  lagrange<N>(tt, w);
  double ra = 0.0, ia = 0.0;
#pragma unroll
  for (int j = 0; j < N; ++j) {
    int64_t cell = i0 - N / 2 + 1 + j;
    cell = cell < 0 ? 0 : (cell > a.m - 1 ? a.m - 1 : cell);
    const double2 g = a.grid[cell];
    ia += g.x * w[j];
    ra += g.y * w[j];
  }
  epi_store(a.epi, t, qv, ra * a.inv_m, ia * a.inv_m);
}

// Twiddles (cos 2 pi j/m, sin 2 pi j/m) for j < m.
__global__ void twiddle_kernel(double2* tw, int64_t m) {
  const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= m) return;
  double s, c;
  sincospi(2.0 * (double)j / (double)m, &s, &c);
  tw[j] = make_double2(c, s);
}

// fft5.rs:404-416: K_even[k] = (pi/dx) r^|k|, |k| = min(k, m - k),
// r = exp(-2 pi eta/(m dx)).  The power is evaluated directly, not by the
// reference's running product (the two differ by that product's rounding,
// at most |k| ulp).
__global__ void even_kernel_spectrum(double* ke, int64_t m, double ke0, double r) {
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= m) return;
  const int64_t half = m / 2;
  const int64_t kk = k <= half ? k : m - k;
  ke[k] = ke0 * pow(r, (double)kk);
}

// Constant tables, cached per (device, m) and (device, m, dx, eta).
struct Tables {
  double2* tw = nullptr;
  int64_t tw_m = 0;
  double* ke = nullptr;
  int64_t ke_cap = 0;
  int64_t ke_m = 0;
  double ke_dx = 0.0, ke_eta = 0.0;
};
std::map<int, Tables> g_tables;

unsigned blocks_for(int64_t n, int t) { return (unsigned)((n + t - 1) / t); }

shrk_status ensure_tables(int64_t m, double dx, double eta, cudaStream_t s, Tables** out) {
  int dev = 0;
  SHRK_CUDA(cudaGetDevice(&dev));
  Tables& T = g_tables[dev];
  bool made = false;
  if (T.tw_m != m) {
    if (T.tw) SHRK_CUDA(cudaFree(T.tw));
    T.tw = nullptr;
    T.tw_m = 0;
    SHRK_CUDA(cudaMalloc(&T.tw, sizeof(double2) * m));
    twiddle_kernel<<<blocks_for(m, 256), 256, 0, s>>>(T.tw, m);
    SHRK_CUDA(cudaGetLastError());
    T.tw_m = m;
    made = true;
  }
  if (T.ke_m != m || T.ke_dx != dx || T.ke_eta != eta) {
    if (T.ke_cap < m) {
      if (T.ke) SHRK_CUDA(cudaFree(T.ke));
      T.ke = nullptr;
      T.ke_cap = 0;
      SHRK_CUDA(cudaMalloc(&T.ke, sizeof(double) * m));
      T.ke_cap = m;
    }
    const double r = std::exp(-2.0 * M_PI * eta / ((double)m * dx));
    even_kernel_spectrum<<<blocks_for(m, 256), 256, 0, s>>>(T.ke, m, M_PI / dx, r);
    SHRK_CUDA(cudaGetLastError());
    T.ke_m = m;
    T.ke_dx = dx;
    T.ke_eta = eta;
    made = true;
  }
  // Tables may be read later from another stream.
  if (made) SHRK_CUDA(cudaStreamSynchronize(s));
  *out = &T;
  return SHRK_OK;
}

int ilog2(int64_t v) {
  int b = 0;
  while ((int64_t(1) << b) < v) ++b;
  return b;
}

shrk_status fft(double2* buf, double2* tmp, int64_t m, const double2* tw, double sign,
                const char* family, cudaStream_t s) {
  const int bits = ilog2(m);
  const int b1 = (bits + 1) / 2, b2 = bits / 2;
  const int m1 = 1 << b1, m2 = 1 << b2;
  {
    LaunchScope ls(family, s);
    fft_pass1<<<blocks_for(m2, fft_group(m1)), 256, 0, s>>>(buf, tmp, m1, b1, m2, m, tw, sign);
    SHRK_CUDA(cudaGetLastError());
  }
  {
    LaunchScope ls(family, s);
    fft_pass2<<<blocks_for(m1, fft_group(m2)), 256, 0, s>>>(tmp, buf, m1, m2, b2, m, tw, sign);
    SHRK_CUDA(cudaGetLastError());
  }
  return SHRK_OK;
}

// One grid: stencil width, size, origin and spacing, and the launch families
// its kernels are timed under.
struct GridPlan {
  int order;
  int64_t m;
  double lo, dx;
  const char* fam_splat;
  const char* fam_fft;
  const char* fam_spectral;
  const char* fam_interp;
};

template <int N>
shrk_status run_grid(const double* d_q, int64_t nq, const double* d_src, int64_t ns, double eta,
                     const GridPlan& g, const Epilogue& epi, cudaStream_t s) {
  const int64_t m = g.m;
  Tables* T = nullptr;
  SHRK_TRY(ensure_tables(m, g.dx, eta, s, &T));
  void* w = nullptr;
  SHRK_TRY(scratch_get(11, sizeof(double2) * 3 * (size_t)m, &w));
  double2* A = (double2*)w;
  double2* B = A + m;
  double2* Tmp = B + m;
  void* sw = nullptr;
  SHRK_TRY(scratch_get(24, (sizeof(int) + N * sizeof(double)) * (size_t)ns + 256, &sw));
  double* wts = (double*)sw;
  int* cell = (int*)(wts + (int64_t)N * ns);
  GridArgs ga{d_src, ns, g.dx < 0.0 ? 1 : 0, g.lo, g.dx, eta, m, cell, wts, A};
  {
    LaunchScope ls(g.fam_splat, s);
    splat_weights_kernel<N><<<blocks_for(ns, 256), 256, 0, s>>>(ga);
    SHRK_CUDA(cudaGetLastError());
  }
  {
    LaunchScope ls(g.fam_splat, s);
    if (ns > 2 * m)
      splat_gather_warp_kernel<N><<<blocks_for(m * 32, 256), 256, 0, s>>>(ga);
    else
      splat_gather_kernel<N><<<blocks_for(m, GATHER_T), GATHER_T, 0, s>>>(ga);
    SHRK_CUDA(cudaGetLastError());
  }
  SHRK_TRY(fft(A, Tmp, m, T->tw, -1.0, g.fam_fft, s));
  {
    LaunchScope ls(g.fam_spectral, s);
    spectral_kernel<<<blocks_for(m, 256), 256, 0, s>>>(A, T->ke, B, m);
    SHRK_CUDA(cudaGetLastError());
  }
  SHRK_TRY(fft(B, Tmp, m, T->tw, +1.0, g.fam_fft, s));
  InterpArgs ia{d_q, nq, B, m, g.lo, g.dx, 1.0 / (double)m, epi};
  {
    LaunchScope ls(g.fam_interp, s);
    interp_kernel<N><<<blocks_for(nq, 256), 256, 0, s>>>(ia);
    SHRK_CUDA(cudaGetLastError());
  }
  return SHRK_OK;
}

shrk_status run_grid_order(const double* d_q, int64_t nq, const double* d_src, int64_t ns,
                           double eta, const GridPlan& g, const Epilogue& epi, cudaStream_t s) {
  switch (g.order) {
    case 2: return run_grid<2>(d_q, nq, d_src, ns, eta, g, epi, s);
    case 4: return run_grid<4>(d_q, nq, d_src, ns, eta, g, epi, s);
    case 6: return run_grid<6>(d_q, nq, d_src, ns, eta, g, epi, s);
    case 8: return run_grid<8>(d_q, nq, d_src, ns, eta, g, epi, s);
    default:
      set_error("fft5: the stencil order must be 2, 4, 6 or 8 nodes");
      return SHRK_EINVAL;
  }
}

}  // namespace

// nufft.rs:106-126 grid_size_for_range.
size_t nufft_grid_size(double raw_range, double eta) {
  double pad = std::max(NUFFT_PAD_ETA_MULT * eta, NUFFT_PAD_RANGE_FRAC * raw_range);
  double range = raw_range + 2.0 * pad;
  size_t max_grid = std::max(std::max(NUFFT_MAX_GRID, NUFFT_MIN_GRID), (size_t)2);
  double target = NUFFT_RESOLUTION * range / eta;
  target = std::isfinite(target) ? std::min(target, (double)max_grid) : (double)max_grid;
  return std::min(next_pow2(std::max((size_t)std::ceil(target), NUFFT_MIN_GRID)), max_grid);
}

// fft5.rs:339-361: pad = max(pad_eta_mult eta, pad_range_frac raw_range),
// m = next_pow2(min(max(ceil(8 range/eta), 8p), 2^20)), at least 2.
size_t fft5_grid_size(double lo_raw, double hi_raw, size_t p, double eta, double pad_eta_mult,
                      double pad_range_frac) {
  const double raw_range = hi_raw - lo_raw;
  const double pad = std::max(pad_eta_mult * eta, pad_range_frac * raw_range);
  const double lo = lo_raw - pad, hi = hi_raw + pad;
  const double range = hi - lo;
  size_t min_grid = sat_usize(std::ceil(8.0 * range / eta));
  const size_t p8 = p > SIZE_MAX / 8 ? SIZE_MAX : 8 * p;
  min_grid = std::min(std::max(min_grid, p8), FFT5_MAX_AUTO_GRID);
  return std::max(next_pow2(min_grid), (size_t)2);
}

shrk_status nufft_points(const double* d_q, int64_t nq, const double* d_src, int64_t ns,
                         double lo_raw, double hi_raw, double eta, const Epilogue& epi,
                         cudaStream_t s) {
  if (nq <= 0 || ns <= 0) return SHRK_OK;
  // fft5.rs:339-361 with the NUFFT options (m fixed by the policy).
  const double raw_range = hi_raw - lo_raw;
  const int64_t m = (int64_t)std::max(nufft_grid_size(raw_range, eta), (size_t)2);
  const double pad = std::max(NUFFT_PAD_ETA_MULT * eta, NUFFT_PAD_RANGE_FRAC * raw_range);
  const double lo = lo_raw - pad, hi = hi_raw + pad;
  const double range = hi - lo;
  GridPlan g{4, m, lo, range / (double)m, "nufft_splat", "nufft_fft", "nufft_spectral",
             "nufft_interp"};
  return run_grid_order(d_q, nq, d_src, ns, eta, g, epi, s);
}

shrk_status fft5_points(const double* d_q, int64_t nq, const double* d_src, int64_t ns,
                        double lo_raw, double hi_raw, double eta, const Fft5Opts& o,
                        const Epilogue& epi, cudaStream_t s) {
  if (nq <= 0 || ns <= 0) return SHRK_OK;
  const size_t m = o.m_override ? std::max(o.m_override, (size_t)2)
                                : fft5_grid_size(lo_raw, hi_raw, (size_t)ns, eta, o.pad_eta_mult,
                                                 o.pad_range_frac);
  if ((m & (m - 1)) != 0 || m > (size_t)FFT_MAX_M) {
    set_error("fft5: the grid size must be a power of two no larger than 2^22 (got " +
              std::to_string(m) + ")");
    return SHRK_ENOTIMPL;
  }
  const double raw_range = hi_raw - lo_raw;
  const double pad = std::max(o.pad_eta_mult * eta, o.pad_range_frac * raw_range);
  const double lo = lo_raw - pad, hi = hi_raw + pad;
  const double range = hi - lo;
  GridPlan g{o.order, (int64_t)m, lo, range / (double)m, "fft5_splat", "fft5_fft",
             "fft5_spectral", "fft5_interp"};
  return run_grid_order(d_q, nq, d_src, ns, eta, g, epi, s);
}

}  // namespace shrk
