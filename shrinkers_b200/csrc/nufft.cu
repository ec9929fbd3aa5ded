// Coarse-grid NUFFT for the Stieltjes transform on sm_100a.
//
// Replaces src/stieltjes/nufft.rs (grid policy 33-126, entry points 164-220)
// and the dual-convolution core of src/stieltjes/fft5.rs (splat 175-185 /
// 259-318, fft_convolution 325-432, interpolate_grid 440-476) with the
// packing helpers of src/stieltjes/fftplan.rs:43-76.  Pipeline (8 kernels,
// all FP64):
//
//   1. splat        one thread per source computes its stencil cell and
//                   4-point Cubic Lagrange weights; then one warp per grid
//                   cell GATHERS the weights of the sources whose stencil
//                   covers it (sources ascending, so they are one contiguous
//                   run, found by a 32-way search) and writes packed[c] =
//                   density[c] + i * x_c/(x_c^2 + eta^2).  Fixed-order warp
//                   sums: deterministic, no atomics (the reference's
//                   sequential and per-worker splats differ from each other
//                   by rounding; its tests pin the NUFFT by tolerance).
//   2. fft (x2)     four-step FFT m = m1*m2 (m1, m2 <= 256): column FFTs of
//                   length m1 in shared memory with the inter-pass twiddle,
//                   then row FFTs of length m2.  Twiddles and the analytic
//                   even-kernel spectrum are tables computed on the host
//                   exactly as the reference computes them.
//   3. spectral     unpack the two real spectra (conjugate symmetry), form
//                   Im_hat + i Re_hat = D*K_even + i D*K_odd.
//   4. fft (x2)     inverse transform.
//   5. interp       4-point interpolation at the query points, 1/m scale,
//                   fused FP64 epilogue.
#include "common.cuh"
#include "epilogue.cuh"
#include "internal.h"

#include <cmath>
#include <map>
#include <vector>

namespace shrk {

namespace {

// nufft.rs:33-58
constexpr double PAD_ETA_MULT = 2000.0;
constexpr double PAD_RANGE_FRAC = 0.75;
constexpr double RESOLUTION = 5.0;
constexpr size_t MIN_GRID = 8192;
constexpr size_t MAX_GRID = 65536;

size_t next_pow2(size_t n) {  // mod.rs:529-535
  size_t p = 1;
  while (p < n) p <<= 1;
  return p;
}

// fft5.rs:136-164 lagrange_weights<4>, operation order preserved.
__device__ __forceinline__ void lagrange4(double t, double w[4]) {
  const double q = 2.0;
  double pref[4], suf[4], acc = 1.0;
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    pref[j] = acc;
    acc *= t - (double)j + q - 1.0;
  }
  acc = 1.0;
#pragma unroll
  for (int j = 3; j >= 0; --j) {
    suf[j] = acc;
    acc *= t - (double)j + q - 1.0;
  }
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    double den = 1.0;
#pragma unroll
    for (int l = 0; l < 4; ++l)
      if (l != j) den *= (double)(j - l);
    w[j] = pref[j] * suf[j] / den;
  }
}

struct GridArgs {
  const double* src;  // ascending
  int64_t ns;
  double lo, dx, eta;
  int64_t m;
  int* cell;          // per source: floor((src - lo)/dx), clamped to [-4, m + 4]
  double* w;          // per source: the 4 stencil weights, SoA [4][ns]
  double2* packed;
};

__device__ __forceinline__ int64_t cell0_of(double v, double lo, double dx, double* t) {
  const double pos = (v - lo) / dx;
  const double fl = floor(pos);
  *t = pos - fl;  // pos - (i0 as f64), i0 = floor(pos)
  return (int64_t)fl;
}

// Per source: stencil cell i0 = floor((v - lo)/dx) and the 4-point Cubic
// Lagrange weights of t = pos - i0 (fft5.rs:175-185).  Clamping i0 to
// [-4, m + 4] keeps the edge-cell mapping (every slot of such a source lands
// on the same edge cell) and the order of the sorted sources.
__global__ void splat_weights_kernel(const GridArgs a) {
  const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= a.ns) return;
  double t;
  const int64_t i0 = cell0_of(a.src[j], a.lo, a.dx, &t);
  double w[4];
  lagrange4(t, w);
  a.cell[j] = (int)(i0 < -4 ? -4 : (i0 > a.m + 4 ? a.m + 4 : i0));
#pragma unroll
  for (int k = 0; k < 4; ++k) a.w[(int64_t)k * a.ns + j] = w[k];
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

// Steps 1+pack: one warp per grid cell gathers the stencil weights of the
// sources covering it (fft5.rs:259-318), then packed[c] = density[c] +
// i x_c/(x_c^2 + eta^2) (fft5.rs:364-376).  Lanes stride the cell's source
// run and a fixed butterfly adds the lane sums: deterministic, no atomics.
__global__ void splat_pack_kernel(const GridArgs a) {
  const int64_t c = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (c >= a.m) return;  // whole warps exit together
  const int64_t m = a.m;
  double dens = 0.0;
  if (c > 0 && c < m - 1) {
    // interior cell: exactly one stencil slot k = c + 1 - i0 per source
    const int64_t j0 = warp_first_ge(a.cell, a.ns, (int)c - 2, lane);
    const int64_t j1 = warp_first_ge(a.cell, a.ns, (int)c + 2, lane);
    for (int64_t j = j0 + lane; j < j1; j += 32) {
      const int k = (int)c + 1 - a.cell[j];
      dens += a.w[(int64_t)k * a.ns + j];
    }
  } else {
    // edge cell: every slot whose clamped index lands here
    const int64_t j0 = (c == 0) ? 0 : warp_first_ge(a.cell, a.ns, (int)m - 3, lane);
    const int64_t j1 = (c == 0) ? warp_first_ge(a.cell, a.ns, 2, lane) : a.ns;
    for (int64_t j = j0 + lane; j < j1; j += 32) {
      const int i0 = a.cell[j];
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        int64_t cell = (int64_t)i0 - 1 + k;
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
constexpr int FFT_G = 4;        // transforms per CTA
constexpr int FFT_MAXL = 256;   // longest in-shared-memory transform

__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

__device__ __forceinline__ unsigned bitrev(unsigned v, int bits) {
  return __brev(v) >> (32 - bits);
}

// Radix-2 decimation-in-time transform of G rows of length L in shared
// memory (rows already in bit-reversed order).  tw: table of
// (cos 2 pi j/m, sin 2 pi j/m), sign -1 forward, +1 inverse.
__device__ void smem_fft(double2 (*buf)[FFT_MAXL], int L, int lbits, int64_t m, const double2* tw,
                         double sign) {
  for (int len = 2; len <= L; len <<= 1) {
    const int half = len >> 1;
    const int64_t step = m / len;
    const int nb = FFT_G * (L >> 1);
    for (int b = threadIdx.x; b < nb; b += blockDim.x) {
      const int g = b / (L >> 1);
      const int r = b % (L >> 1);
      const int grp = r / half, k = r % half;
      const int i = grp * len + k;
      const double2 t = tw[(int64_t)k * step];
      const double2 w = make_double2(t.x, sign * t.y);
      const double2 u = buf[g][i];
      const double2 v = cmul(buf[g][i + half], w);
      buf[g][i] = make_double2(u.x + v.x, u.y + v.y);
      buf[g][i + half] = make_double2(u.x - v.x, u.y - v.y);
    }
    __syncthreads();
  }
  (void)lbits;
}

// Pass 1: Y[k1*m2 + n2] = W_m^{n2 k1} * sum_n1 x[m2 n1 + n2] W_m1^{n1 k1}.
__global__ void __launch_bounds__(256) fft_pass1(const double2* __restrict__ x,
                                                 double2* __restrict__ y, int m1, int b1, int m2,
                                                 int64_t m, const double2* __restrict__ tw,
                                                 double sign) {
  __shared__ double2 buf[FFT_G][FFT_MAXL];
  const int n2_0 = blockIdx.x * FFT_G;
  for (int e = threadIdx.x; e < FFT_G * m1; e += blockDim.x) {
    const int n1 = e / FFT_G, g = e % FFT_G;
    buf[g][bitrev((unsigned)n1, b1)] = x[(int64_t)m2 * n1 + n2_0 + g];
  }
  __syncthreads();
  smem_fft(buf, m1, b1, m, tw, sign);
  for (int e = threadIdx.x; e < FFT_G * m1; e += blockDim.x) {
    const int k1 = e / FFT_G, g = e % FFT_G;
    const int n2 = n2_0 + g;
    const double2 t = tw[((int64_t)n2 * k1) % m];
    y[(int64_t)k1 * m2 + n2] = cmul(buf[g][k1], make_double2(t.x, sign * t.y));
  }
}

// Pass 2: X[k1 + m1 k2] = sum_n2 Y[k1*m2 + n2] W_m2^{n2 k2}.
__global__ void __launch_bounds__(256) fft_pass2(const double2* __restrict__ y,
                                                 double2* __restrict__ x, int m1, int m2, int b2,
                                                 int64_t m, const double2* __restrict__ tw,
                                                 double sign) {
  __shared__ double2 buf[FFT_G][FFT_MAXL];
  const int k1_0 = blockIdx.x * FFT_G;
  for (int e = threadIdx.x; e < FFT_G * m2; e += blockDim.x) {
    const int g = e / m2, n2 = e % m2;
    buf[g][bitrev((unsigned)n2, b2)] = y[(int64_t)(k1_0 + g) * m2 + n2];
  }
  __syncthreads();
  smem_fft(buf, m2, b2, m, tw, sign);
  for (int e = threadIdx.x; e < FFT_G * m2; e += blockDim.x) {
    const int k2 = e / FFT_G, g = e % FFT_G;
    x[(int64_t)(k1_0 + g) + (int64_t)m1 * k2] = buf[g][k2];
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

// fft5.rs:191-211 interp_at<4> + 440-476: re <- .im, im <- .re, times 1/m.
__global__ void interp_kernel(const InterpArgs a) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= a.nq) return;
  const double qv = a.q[t];
  double tt;
  const int64_t i0 = cell0_of(qv, a.lo, a.dx, &tt);
  double w[4];
  lagrange4(tt, w);
  double ra = 0.0, ia = 0.0;
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    int64_t cell = i0 - 1 + j;
    cell = cell < 0 ? 0 : (cell > a.m - 1 ? a.m - 1 : cell);
    const double2 g = a.grid[cell];
    ia += g.x * w[j];
    ra += g.y * w[j];
  }
  epi_store(a.epi, t, qv, ra * a.inv_m, ia * a.inv_m);
}

// Host-side constant tables, cached per (device, m) and (device, m, dx, eta).
struct Tables {
  double2* tw = nullptr;
  int64_t tw_m = 0;
  double* ke = nullptr;
  int64_t ke_m = 0;
  double ke_dx = 0.0, ke_eta = 0.0;
};
std::map<int, Tables> g_tables;

shrk_status ensure_tables(int64_t m, double dx, double eta, cudaStream_t s, Tables** out) {
  int dev = 0;
  SHRK_CUDA(cudaGetDevice(&dev));
  Tables& T = g_tables[dev];
  if (T.tw_m != m) {
    std::vector<double2> h(m);
    for (int64_t j = 0; j < m; ++j) {
      const double ang = 2.0 * M_PI * (double)j / (double)m;
      h[j] = make_double2(std::cos(ang), std::sin(ang));
    }
    if (T.tw) SHRK_CUDA(cudaFree(T.tw));
    T.tw = nullptr;
    T.tw_m = 0;
    SHRK_CUDA(cudaMalloc(&T.tw, sizeof(double2) * m));
    SHRK_CUDA(cudaMemcpyAsync(T.tw, h.data(), sizeof(double2) * m, cudaMemcpyHostToDevice, s));
    SHRK_CUDA(cudaStreamSynchronize(s));
    T.tw_m = m;
  }
  if (T.ke_m != m || T.ke_dx != dx || T.ke_eta != eta) {
    // fft5.rs:404-416: K_even[k] = (pi/dx) r^|k| by recurrence.
    std::vector<double> h(m);
    const int64_t half = m / 2;
    const double r = std::exp(-2.0 * M_PI * eta / ((double)m * dx));
    const double ke0 = M_PI / dx;
    double pw = 1.0;
    for (int64_t k = 0; k <= half; ++k) {
      h[k] = ke0 * pw;
      pw *= r;
    }
    pw = r;
    for (int64_t k = m - 1; k > half; --k) {
      h[k] = ke0 * pw;
      pw *= r;
    }
    if (T.ke_m != m) {
      if (T.ke) SHRK_CUDA(cudaFree(T.ke));
      T.ke = nullptr;
      T.ke_m = 0;
      SHRK_CUDA(cudaMalloc(&T.ke, sizeof(double) * m));
    }
    SHRK_CUDA(cudaMemcpyAsync(T.ke, h.data(), sizeof(double) * m, cudaMemcpyHostToDevice, s));
    SHRK_CUDA(cudaStreamSynchronize(s));
    T.ke_m = m;
    T.ke_dx = dx;
    T.ke_eta = eta;
  }
  *out = &T;
  return SHRK_OK;
}

int ilog2(int64_t v) {
  int b = 0;
  while ((int64_t(1) << b) < v) ++b;
  return b;
}

shrk_status fft(double2* buf, double2* tmp, int64_t m, const double2* tw, double sign,
                cudaStream_t s) {
  const int bits = ilog2(m);
  const int b1 = (bits + 1) / 2, b2 = bits / 2;
  const int m1 = 1 << b1, m2 = 1 << b2;
  {
    LaunchScope ls("nufft_fft", s);
    fft_pass1<<<m2 / FFT_G, 256, 0, s>>>(buf, tmp, m1, b1, m2, m, tw, sign);
    SHRK_CUDA(cudaGetLastError());
  }
  {
    LaunchScope ls("nufft_fft", s);
    fft_pass2<<<m1 / FFT_G, 256, 0, s>>>(tmp, buf, m1, m2, b2, m, tw, sign);
    SHRK_CUDA(cudaGetLastError());
  }
  return SHRK_OK;
}

}  // namespace

// nufft.rs:106-126 grid_size_for_range.
size_t nufft_grid_size(double raw_range, double eta) {
  double pad = std::max(PAD_ETA_MULT * eta, PAD_RANGE_FRAC * raw_range);
  double range = raw_range + 2.0 * pad;
  size_t max_grid = std::max(std::max(MAX_GRID, MIN_GRID), (size_t)2);
  double target = RESOLUTION * range / eta;
  target = std::isfinite(target) ? std::min(target, (double)max_grid) : (double)max_grid;
  return std::min(next_pow2(std::max((size_t)std::ceil(target), MIN_GRID)), max_grid);
}

shrk_status nufft_points(const double* d_q, int64_t nq, const double* d_src, int64_t ns,
                         double lo_raw, double hi_raw, double eta, const Epilogue& epi,
                         cudaStream_t s) {
  if (nq <= 0 || ns <= 0) return SHRK_OK;
  // fft5.rs:339-361 with the NUFFT options (m fixed by the policy).
  const double raw_range = hi_raw - lo_raw;
  const int64_t m = (int64_t)std::max(nufft_grid_size(raw_range, eta), (size_t)2);
  if ((m & (m - 1)) != 0 || m > (int64_t)FFT_MAXL * FFT_MAXL || m < 16) {
    set_error("nufft: grid size must be a power of two in [16, 65536]");
    return SHRK_ENOTIMPL;
  }
  const double pad = std::max(PAD_ETA_MULT * eta, PAD_RANGE_FRAC * raw_range);
  const double lo = lo_raw - pad, hi = hi_raw + pad;
  const double range = hi - lo;
  const double dx = range / (double)m;
  Tables* T = nullptr;
  SHRK_TRY(ensure_tables(m, dx, eta, s, &T));
  void* w = nullptr;
  SHRK_TRY(scratch_get(11, sizeof(double2) * 3 * m, &w));
  double2* A = (double2*)w;
  double2* B = A + m;
  double2* Tmp = B + m;
  void* sw = nullptr;
  SHRK_TRY(scratch_get(24, (sizeof(int) + 4 * sizeof(double)) * (size_t)ns + 256, &sw));
  double* wts = (double*)sw;
  int* cell = (int*)(wts + 4 * ns);
  GridArgs ga{d_src, ns, lo, dx, eta, m, cell, wts, A};
  {
    LaunchScope ls("nufft_splat", s);
    splat_weights_kernel<<<(unsigned)((ns + 255) / 256), 256, 0, s>>>(ga);
    SHRK_CUDA(cudaGetLastError());
  }
  {
    LaunchScope ls("nufft_splat", s);
    splat_pack_kernel<<<(unsigned)((m * 32 + 255) / 256), 256, 0, s>>>(ga);
    SHRK_CUDA(cudaGetLastError());
  }
  SHRK_TRY(fft(A, Tmp, m, T->tw, -1.0, s));
  {
    LaunchScope ls("nufft_spectral", s);
    spectral_kernel<<<(unsigned)((m + 255) / 256), 256, 0, s>>>(A, T->ke, B, m);
    SHRK_CUDA(cudaGetLastError());
  }
  SHRK_TRY(fft(B, Tmp, m, T->tw, +1.0, s));
  InterpArgs ia{d_q, nq, B, m, lo, dx, 1.0 / (double)m, epi};
  {
    LaunchScope ls("nufft_interp", s);
    interp_kernel<<<(unsigned)((nq + 255) / 256), 256, 0, s>>>(ia);
    SHRK_CUDA(cudaGetLastError());
  }
  return SHRK_OK;
}

}  // namespace shrk
