// Device helpers shared by the exact pair-sum kernels (forward and adjoint):
// FP64 / FP32 pair arithmetic, the FP32 separation scheme of the MIXED
// kernels, packed f32x2 operations, and small reductions.
#pragma once

#include "common.cuh"

namespace shrk {

typedef unsigned long long u64;

// Near-field radius (units of eta) below which MIXED kernels stay in FP64.
#ifndef SHRK_NEAR_K
#define SHRK_NEAR_K 32.0
#endif

constexpr int SUB = 256;  // sources per near/far classification block

__device__ __forceinline__ double warp_max(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}
__device__ __forceinline__ double warp_min(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmin(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

// FP64 pair: re += d/(d^2+eta^2), iv += 1/(d^2+eta^2).
__device__ __forceinline__ void pair64(double x, double s, double eta2, double& re, double& iv) {
  const double d = x - s;
  const double inv = rcp_f64(fma(d, d, eta2));
  re = fma(d, inv, re);
  iv = iv + inv;
}

// ---------------------------------------------- FP32 separation scheme --
// Targets and sources are split around a centre c: x - c = xh + xl and
// s - c = mh + ml, with xh a multiple of a power of two u >= ulp(max|s-c|).
// Then mh - xh is exact (or rounds on the source's own bits) and the final
// rounding of (mh - xh) + (ml - xl) depends on the source's low bits ml, so
// the separation errors of different pairs are independent.  Rounding a
// FIXED target offset onto each source's float grid instead would shift the
// target coherently by up to half an ulp of d -- a systematic error (~7e-9
// relative at p = 1e6) that no accumulation scheme removes.

// Power of two u >= ulp_float(M) (IEEE-754 exponent field of M, minus the
// 23 fraction bits).
__device__ __forceinline__ double snap_unit(double M) {
  const long long bits = __double_as_longlong(M) & 0x7FF0000000000000LL;
  return __longlong_as_double(bits) * 0x1p-23;
}

// x - c = xh + xl with xh a multiple of u (exact in float while
// |x - c| < 2^23 u, which the callers guarantee).
__device__ __forceinline__ void split_target(double x, double c, double u, float& xh, float& xl) {
  const double xo = x - c;
  const double h = rint(xo / u) * u;
  xh = (float)h;
  xl = (float)(xo - h);
}

// Scalar separation d = x - s from the split parts.
__device__ __forceinline__ float sep32(float xh, float xl, float mh, float ml) {
  return (xh - mh) + (xl - ml);
}

__device__ __forceinline__ void split_source(double s, double c, float& mh, float& ml) {
  const double so = s - c;
  mh = (float)so;
  ml = (float)(so - (double)mh);
}

// Unbiased FP32 reciprocal: the MUFU seed's error has a nonzero mean (a
// few 1e-9 relative, measured), which would add coherently over a far
// field of ~1e6 same-signed terms; one Newton step removes it.
__device__ __forceinline__ float rcp32_unbiased(float a) {
  const float r = rcp_f32(a);
  return fmaf(r, fmaf(-a, r, 1.0f), r);
}

// ------------------------------------------------------ packed f32x2 --
// sm_100 packed FP32 pairs: one issue slot drives two FP32 lanes.
__device__ __forceinline__ u64 pk2(float lo, float hi) {
  u64 r;
  asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(lo), "f"(hi));
  return r;
}
__device__ __forceinline__ void upk2(u64 v, float& lo, float& hi) {
  asm("mov.b64 {%0, %1}, %2;" : "=f"(lo), "=f"(hi) : "l"(v));
}
__device__ __forceinline__ u64 ffma2(u64 a, u64 b, u64 c) {
  u64 d;
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
  return d;
}
__device__ __forceinline__ u64 fadd2(u64 a, u64 b) {
  u64 d;
  asm("add.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
  return d;
}
__device__ __forceinline__ u64 fsub2(u64 a, u64 b) {
  u64 d;
  asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
  return d;
}

__device__ __forceinline__ u64 fmul2(u64 a, u64 b) {
  u64 d;
  asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
  return d;
}

// Mean relative error of the MUFU reciprocal (rcp.approx.ftz.f32) on
// sm_100, measured over every mantissa of [1, 2) with the log-uniform weight
// 1/m (shrk_measure_rcp_bias): r_mufu = (1/a)(1 + RCP32_BIAS) on average.
// A far field of ~1e6 terms of one sign would carry this offset coherently,
// so the FP64 fold scales each FP32 partial by (1 - RCP32_BIAS) instead of
// refining every reciprocal with a Newton step (two packed FMAs per four
// pairs); the remaining error of a seed (<= 1 ulp, zero mean) averages out
// over the sum like the rounding of a refined reciprocal.
constexpr double RCP32_BIAS = 3.7e-9;

// Four FP32 far-field pairs: two targets (the packed lanes) x two sources
// s1, s2 of one 256-source block with centre cb.
//   TH + TL = x - cb   (TH = float(x - cb), TL = the rounding remainder)
//   SM      = float(s1 - cb),  DL = float(s1 - s2)
//   d1 = TH - (SM - TL) = x - s1,   d2 = d1 + DL = x - s2
// The remainder TL keeps the block-wide target offset exact.  It must enter
// through SM, whose ulp is far finer than TH's: (TH - SM) + TL would round
// TL away (TH - SM already sits on TH's ulp grid) and leave a coherent
// offset of up to half an ulp on every pair of the block.  In this order the
// one rounding at ulp(d) depends on each source's low bits, so the
// separation errors of different pairs are independent.
// One reciprocal serves both sources:
//   e_k = d_k^2 + eta^2,  r = 1/(e1 e2) (MUFU, its mean error removed at the
//   fold: RCP32_BIAS),
//   d1/e1 + d2/e2 = (d1 e2 + d2 e1) r,   1/e1 + 1/e2 = (e1 + e2) r.
// r is carried negated (NR = -r) so the packed pipe needs no negation:
// RE and IVN accumulate -sum d/e and -sum 1/e.  The caller keeps e1 e2
// inside the FP32 normal range (block span <= 1e9, gap >= 1e-9).
__device__ __forceinline__ void pairs32x4(u64 SM, u64 DL, u64 TH, u64 TL, u64 ETA2, u64& RE,
                                          u64& IVN) {
  const u64 D1 = fsub2(TH, fsub2(SM, TL));
  const u64 D2 = fadd2(D1, DL);
  const u64 E1 = ffma2(D1, D1, ETA2);
  const u64 E2 = ffma2(D2, D2, ETA2);
  const u64 P = fmul2(E1, E2);
  float a0, a1;
  upk2(P, a0, a1);
  const u64 NR = pk2(rcp_f32(-a0), rcp_f32(-a1));
  const u64 NUM = ffma2(D1, E2, fmul2(D2, E1));
  RE = ffma2(NUM, NR, RE);
  IVN = ffma2(fadd2(E1, E2), NR, IVN);
}

// Host: (min, max) of every SUB-block of d_src into bounds[0..nblocks) and the
// global (min, max) into bounds[nblocks] (two small kernels on stream s).
shrk_status source_bounds(const double* d_src, int64_t ns, int64_t nblocks, double2* bounds,
                          cudaStream_t s);

// Host: work decomposition of an (nt targets) x (ns sources) pair sum into
// tiles of `tile` targets and source splits that are multiples of `chunk`.
struct SplitPlan {
  int64_t n_tiles;
  int n_splits;
  int64_t split_len;
  int grid;
};
SplitPlan plan_splits(int64_t nt, int64_t ns, int tile, int chunk, int ctas_per_sm);

}  // namespace shrk
