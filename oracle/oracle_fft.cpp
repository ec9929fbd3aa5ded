// TEST INFRASTRUCTURE ONLY (see oracle.h): restatement of the FFT grid
// convolution of src/stieltjes/fft5.rs (Fft5Options 213-249, lagrange_weights
// 136-164, splat 175-185, splat_chunk 295-318, fft_convolution 325-432,
// interp_at 191-211, interpolate_grid 440-476, entry points 559-625) with the
// packing helpers of src/stieltjes/fftplan.rs:43-76, and of the coarse-grid
// NUFFT policy over it (src/stieltjes/nufft.rs: grid policy 33-126, entry
// points 164-220).
//
// The reference's transforms come from rustfft 6.4.1 (Cargo.lock), which is
// not vendored.  Its published contract -- unnormalised DFT, forward sign
// e^{-2 pi i jk/m}, inverse e^{+2 pi i jk/m} -- is restated here with an
// iterative radix-2 decimation-in-time FFT of our own; the rounding of
// rustfft's mixed-radix plans is not reproduced, so FFT-level parity with the
// reference is by tolerance only.
#include "oracle.h"

#include <algorithm>
#include <cmath>
#include <complex>
#include <vector>
#include <omp.h>

namespace orc {

typedef std::complex<double> cplx;

// nufft.rs:33-58
static const double PAD_ETA_MULT = 2000.0, PAD_RANGE_FRAC = 0.75, RESOLUTION = 5.0;
static const size_t MIN_GRID = 8192, MAX_GRID = 65536;

static size_t next_pow2(size_t n) {  // mod.rs:529-535
  size_t p = 1;
  while (p < n) p <<= 1;
  return p;
}

// nufft.rs:106-126 grid_size_for_range.
size_t nufft_grid_size(double raw_range, double eta) {
  double pad = std::max(PAD_ETA_MULT * eta, PAD_RANGE_FRAC * raw_range);
  double range = raw_range + 2.0 * pad;
  size_t max_grid = std::max(std::max(MAX_GRID, MIN_GRID), (size_t)2);
  double target = RESOLUTION * range / eta;
  target = std::isfinite(target) ? std::min(target, (double)max_grid) : (double)max_grid;
  return std::min(next_pow2(std::max((size_t)std::ceil(target), MIN_GRID)), max_grid);
}

// fft5.rs:136-164 lagrange_weights<N>.
template <int N>
static inline void lagrange_weights(double t, double* w) {
  const double q = (double)(N / 2);
  double pref[N], suf[N], acc = 1.0;
  for (int j = 0; j < N; ++j) {
    pref[j] = acc;
    acc *= t - (double)j + q - 1.0;
  }
  acc = 1.0;
  for (int j = N - 1; j >= 0; --j) {
    suf[j] = acc;
    acc *= t - (double)j + q - 1.0;
  }
  for (int j = 0; j < N; ++j) {
    double den = 1.0;
    for (int l = 0; l < N; ++l)
      if (l != j) den *= (double)(j - l);
    w[j] = pref[j] * suf[j] / den;
  }
}

// fft5.rs:175-185 splat<N>: one unit mass at grid position pos.
template <int N>
static inline void splat(double* density, size_t m, double pos) {
  double fl = std::floor(pos);
  long i0 = (long)fl;
  double t = pos - (double)i0;
  double w[N];
  lagrange_weights<N>(t, w);
  const long off0 = -N / 2 + 1;
  for (int j = 0; j < N; ++j) {
    long cell = std::min(std::max(i0 + off0 + j, 0L), (long)m - 1);
    density[cell] += w[j];
  }
}

// fft5.rs:295-318 splat_chunk: dispatch on the stencil width.
static void splat_chunk(const double* ev, size_t a, size_t b, double* density, size_t m,
                        double lo, double dx, int order) {
  for (size_t k = a; k < b; ++k) {
    const double pos = (ev[k] - lo) / dx;
    switch (order) {
      case 2: splat<2>(density, m, pos); break;
      case 4: splat<4>(density, m, pos); break;
      case 6: splat<6>(density, m, pos); break;
      default: splat<8>(density, m, pos); break;
    }
  }
}

// Radix-2 iterative DFT, unnormalised; sign = -1 forward, +1 inverse.
void fft_radix2(cplx* a, size_t m, int sign) {
  for (size_t i = 1, j = 0; i < m; ++i) {
    size_t bit = m >> 1;
    for (; j & bit; bit >>= 1) j ^= bit;
    j ^= bit;
    if (i < j) std::swap(a[i], a[j]);
  }
  std::vector<cplx> tw(m / 2);
  for (size_t k = 0; k < m / 2; ++k) {
    double ang = 2.0 * M_PI * (double)k / (double)m;
    tw[k] = cplx(std::cos(ang), sign * std::sin(ang));
  }
  for (size_t len = 2; len <= m; len <<= 1) {
    size_t step = m / len;
    for (size_t i = 0; i < m; i += len) {
      for (size_t k = 0; k < len / 2; ++k) {
        cplx u = a[i + k], v = a[i + k + len / 2] * tw[k * step];
        a[i + k] = u + v;
        a[i + k + len / 2] = u - v;
      }
    }
  }
}

// Any-length DFT for grids that are not a power of two (rustfft plans any
// length, fftplan.rs:21-28): the direct sum, one output per iteration, with
// the twiddle index n k reduced modulo m exactly in integers so that every
// factor is a correctly rounded cos/sin of 2 pi j/m.  Every output is one
// sequential sum, so the threads do not change the result.  O(m^2): the
// grids the tests force this way are at most a few 10^4 points.
void dft_any(cplx* a, size_t m, int sign) {
  if ((m & (m - 1)) == 0) {
    fft_radix2(a, m, sign);
    return;
  }
  std::vector<cplx> tw(m), out(m);
  for (size_t j = 0; j < m; ++j) {
    const double ang = 2.0 * M_PI * (double)j / (double)m;
    tw[j] = cplx(std::cos(ang), sign * std::sin(ang));
  }
#pragma omp parallel for schedule(static)
  for (long long k = 0; k < (long long)m; ++k) {
    cplx acc(0.0, 0.0);
    size_t idx = 0;
    for (size_t n = 0; n < m; ++n) {
      acc += a[n] * tw[idx];
      idx += (size_t)k;
      if (idx >= m) idx -= m;
    }
    out[(size_t)k] = acc;
  }
  std::copy(out.begin(), out.end(), a);
}

struct Grid { std::vector<cplx> out; double lo, dx; size_t m; };

// fft5.rs:213-249 Fft5Options.
struct Opts {
  int order;          // stencil nodes: 2, 4, 6 or 8
  size_t m_override;  // 0 = the adaptive rule
  double pad_eta_mult, pad_range_frac;
};

// Rust's saturating float -> usize cast (NaN -> 0, negative -> 0).
static size_t sat_usize(double v) {
  if (!(v > 0.0)) return 0;
  if (v >= 18446744073709551616.0) return SIZE_MAX;
  return (size_t)v;
}

// fft5.rs:339-361: the fft5 grid rule dx <= eta/8 and m >= 8p, capped at 2^20.
size_t fft5_grid_size(double lo_raw, double hi_raw, size_t p, double eta, double pad_eta_mult,
                      double pad_range_frac) {
  const double raw_range = hi_raw - lo_raw;
  const double pad = std::max(pad_eta_mult * eta, pad_range_frac * raw_range);
  const double lo = lo_raw - pad, hi = hi_raw + pad;
  const double range = hi - lo;
  size_t min_grid = sat_usize(std::ceil(8.0 * range / eta));
  min_grid = std::min(std::max(min_grid, 8 * p), (size_t)1024 * 1024);
  return std::max(next_pow2(min_grid), (size_t)2);
}

static void convolve_density(const double* density, size_t m, double lo, double dx, double eta,
                             Grid& G);

// fft5.rs:325-432 fft_convolution: grid (lo, dx, m) from the first/last
// entries, order-N splat, packed forward FFT, analytic even kernel, packed
// product, inverse FFT (radix-2 for powers of two, the direct DFT otherwise).
static void convolution(const double* ev, size_t p, double eta, const Opts& o, size_t m,
                        bool parallel, Grid& G) {
  double lo_raw = ev[0], hi_raw = ev[p - 1];
  double raw_range = hi_raw - lo_raw;
  double pad = std::max(o.pad_eta_mult * eta, o.pad_range_frac * raw_range);
  double lo = lo_raw - pad, hi = hi_raw + pad;
  double range = hi - lo;
  double dx = range / (double)m;

  std::vector<double> density(m, 0.0);
  if (parallel && p >= 4096) {  // fft5.rs:259-292 per-worker buffers + reduce
    int nt = omp_get_max_threads();
    std::vector<std::vector<double>> bufs(nt, std::vector<double>(m, 0.0));
    size_t chunk = (p + nt - 1) / nt;
#pragma omp parallel num_threads(nt)
    {
      int t = omp_get_thread_num();
      size_t a = std::min(p, (size_t)t * chunk), b = std::min(p, a + chunk);
      splat_chunk(ev, a, b, bufs[t].data(), m, lo, dx, o.order);
    }
    for (int t = 0; t < nt; ++t)
      for (size_t i = 0; i < m; ++i) density[i] += bufs[t][i];
  } else {
    splat_chunk(ev, 0, p, density.data(), m, lo, dx, o.order);
  }

  convolve_density(density.data(), m, lo, dx, eta, G);
}

// fft5.rs:364-432: the density packed with the odd kernel, forward FFT,
// analytic even kernel, packed product, inverse FFT, on the grid (m, lo, dx).
static void convolve_density(const double* density, size_t m, double lo, double dx, double eta,
                             Grid& G) {
  const size_t half = m / 2;
  std::vector<cplx> packed(m);
  const double mf = (double)m;
  for (size_t i = 0; i < m; ++i) {
    double sd = (i <= half) ? (double)i : (double)i - mf;
    double x = sd * dx;
    double denom = x * x + eta * eta;
    packed[i] = cplx(density[i], x / denom);
  }
  dft_any(packed.data(), m, -1);
  // fftplan.rs:43-54 unpack_packed_real_pair
  std::vector<cplx> D(m), K(m);
  for (size_t k = 0; k < m; ++k) {
    cplx ck = packed[k], cnk = std::conj(packed[(m - k) % m]);
    cplx s = ck + cnk, df = ck - cnk;
    D[k] = cplx(0.5 * s.real(), 0.5 * s.imag());
    // (-0.5 i) * df
    K[k] = cplx(0.5 * df.imag(), -0.5 * df.real());
  }
  // fft5.rs:404-416 analytic even kernel
  double r = std::exp(-2.0 * M_PI * eta / ((double)m * dx));
  double ke0 = M_PI / dx;
  std::vector<double> ke(m);
  double pw = 1.0;
  for (size_t k = 0; k <= half; ++k) { ke[k] = ke0 * pw; pw *= r; }
  pw = r;
  for (size_t k = m - 1; k > half; --k) { ke[k] = ke0 * pw; pw *= r; }
  // fftplan.rs:62-76 pack_dual_product
  G.out.resize(m);
  for (size_t k = 0; k < m; ++k) {
    cplx d = D[k];
    double ih_re = d.real() * ke[k], ih_im = d.imag() * ke[k];
    cplx rh = d * K[k];
    G.out[k] = cplx(ih_re - rh.imag(), ih_im + rh.real());
  }
  dft_any(G.out.data(), m, +1);
  G.lo = lo;
  G.dx = dx;
  G.m = m;
}

// fft5.rs:191-211 interp_at<N>: re <- .im, im <- .re, times 1/m.
template <int N>
static inline void interp_at(const Grid& G, double q, double inv_m, double* re, double* im) {
  double pos = (q - G.lo) / G.dx;
  long i0 = (long)std::floor(pos);
  double t = pos - (double)i0, w[N];
  lagrange_weights<N>(t, w);
  const long off0 = -N / 2 + 1;
  double ra = 0.0, ia = 0.0;
  for (int j = 0; j < N; ++j) {
    long cell = std::min(std::max(i0 + off0 + j, 0L), (long)G.m - 1);
    ia += G.out[cell].real() * w[j];
    ra += G.out[cell].imag() * w[j];
  }
  *re = ra * inv_m;
  *im = ia * inv_m;
}

// fft5.rs:440-476 interpolate_grid.
static void interpolate(const Grid& G, const double* q, size_t nq, int order, bool parallel,
                        double* re, double* im) {
  const double inv_m = 1.0 / (double)G.m;
#pragma omp parallel for schedule(static) if (parallel && nq >= 4096)
  for (long k = 0; k < (long)nq; ++k) {
    switch (order) {
      case 2: interp_at<2>(G, q[k], inv_m, &re[k], &im[k]); break;
      case 4: interp_at<4>(G, q[k], inv_m, &re[k], &im[k]); break;
      case 6: interp_at<6>(G, q[k], inv_m, &re[k], &im[k]); break;
      default: interp_at<8>(G, q[k], inv_m, &re[k], &im[k]); break;
    }
  }
}

static Opts nufft_opts() { return Opts{4, 0, PAD_ETA_MULT, PAD_RANGE_FRAC}; }

// nufft.rs:164-220 (raw sums; the first/last entries bound the spectrum).
void nufft_points(const double* q, size_t nq, const double* ev, size_t p, double eta,
                  bool parallel, double* re, double* im) {
  if (p == 0 || nq == 0) return;
  Grid G;
  const size_t m = std::max(nufft_grid_size(ev[p - 1] - ev[0], eta), (size_t)2);
  convolution(ev, p, eta, nufft_opts(), m, parallel, G);
  interpolate(G, q, nq, 4, parallel, re, im);
}

// fft5.rs:559-625 compute_all_stieltjes_fft5_with_options /
// compute_stieltjes_fft_at_points (raw sums, sequential splat and
// interpolation).  Returns 0.
int fft5_points(const double* q, size_t nq, const double* ev, size_t p, double eta, int order,
                size_t m_override, double pad_eta_mult, double pad_range_frac, double* re,
                double* im) {
  if (p == 0 || nq == 0) return 0;
  const Opts o{order, m_override, pad_eta_mult, pad_range_frac};
  const size_t m = m_override ? std::max(m_override, (size_t)2)
                              : fft5_grid_size(ev[0], ev[p - 1], p, eta, pad_eta_mult,
                                               pad_range_frac);
  Grid G;
  convolution(ev, p, eta, o, m, false, G);
  interpolate(G, q, nq, order, false, re, im);
  return 0;
}

}  // namespace orc

using namespace orc;

extern "C" {

size_t orc_nufft_grid_size(double raw_range, double eta) { return nufft_grid_size(raw_range, eta); }

void orc_nufft_points(const double* q, size_t nq, const double* ev, size_t p, double eta,
                      int parallel, double* re, double* im) {
  nufft_points(q, nq, ev, p, eta, parallel != 0, re, im);
}

// Grid-level export for kernel-by-kernel parity: density after the splat
// (m doubles) and the packed grid after the inverse FFT (2m doubles,
// interleaved re/im, before the 1/m scaling).  Returns m.
size_t orc_nufft_grid(const double* ev, size_t p, double eta, double* density_out,
                      double* packed_out, double* lo_out, double* dx_out) {
  Grid G;
  const size_t m = std::max(nufft_grid_size(ev[p - 1] - ev[0], eta), (size_t)2);
  convolution(ev, p, eta, nufft_opts(), m, false, G);
  if (density_out) {
    std::fill(density_out, density_out + G.m, 0.0);
    splat_chunk(ev, 0, p, density_out, G.m, G.lo, G.dx, 4);
  }
  if (packed_out)
    for (size_t k = 0; k < G.m; ++k) {
      packed_out[2 * k] = G.out[k].real();
      packed_out[2 * k + 1] = G.out[k].imag();
    }
  if (lo_out) *lo_out = G.lo;
  if (dx_out) *dx_out = G.dx;
  return G.m;
}

// The NUFFT grid of a spectrum with first/last entries first/last
// (nufft.rs:106-126 with the padding of fft5.rs:339-361).
void orc_nufft_geometry(double first, double last, double eta, size_t* m, double* lo,
                        double* dx) {
  const double raw_range = last - first;
  *m = std::max(nufft_grid_size(raw_range, eta), (size_t)2);
  const double pad = std::max(PAD_ETA_MULT * eta, PAD_RANGE_FRAC * raw_range);
  *lo = first - pad;
  *dx = ((last + pad) - *lo) / (double)*m;
}

// The two stages of the grid convolution apart, on a given grid: the
// sequential order-N splat of p sources (fft5.rs:295-318), and the
// convolution of a density plus interpolation at nq points (raw sums).
void orc_grid_density(const double* ev, size_t p, size_t m, double lo, double dx, int order,
                      double* density) {
  std::fill(density, density + m, 0.0);
  splat_chunk(ev, 0, p, density, m, lo, dx, order);
}

void orc_grid_eval(const double* density, size_t m, double lo, double dx, double eta, int order,
                   const double* q, size_t nq, double* re, double* im) {
  Grid G;
  convolve_density(density, m, lo, dx, eta, G);
  interpolate(G, q, nq, order, false, re, im);
}

void orc_fft(double* interleaved, size_t m, int sign) {
  dft_any(reinterpret_cast<std::complex<double>*>(interleaved), m, sign);
}

void orc_lagrange4(double t, double* w) { lagrange_weights<4>(t, w); }

// Lagrange weights of an n-node stencil (n = 2, 4, 6, 8).
void orc_lagrange(int n, double t, double* w) {
  switch (n) {
    case 2: lagrange_weights<2>(t, w); break;
    case 4: lagrange_weights<4>(t, w); break;
    case 6: lagrange_weights<6>(t, w); break;
    default: lagrange_weights<8>(t, w); break;
  }
}

size_t orc_fft5_grid_size(double lo_raw, double hi_raw, size_t p, double eta, double pad_eta_mult,
                          double pad_range_frac) {
  return fft5_grid_size(lo_raw, hi_raw, p, eta, pad_eta_mult, pad_range_frac);
}

int orc_fft5_points(const double* q, size_t nq, const double* ev, size_t p, double eta, int order,
                    size_t m_override, double pad_eta_mult, double pad_range_frac, double* re,
                    double* im) {
  return fft5_points(q, nq, ev, p, eta, order, m_override, pad_eta_mult, pad_range_frac, re, im);
}

}  // extern "C"
