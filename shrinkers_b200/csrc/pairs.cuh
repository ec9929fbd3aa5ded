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

// Two FP32 far-field pairs (two targets, one source) in packed form.  All
// quantities are carried negated so no negation is needed on the packed
// pipe: ND = s - x, NR = -1/(d^2+eta^2) refined by one Newton step.
//   re += d * r   ==  RE += ND * NR
//   iv += r       ==  IVN += NR          (IVN accumulates -iv)
__device__ __forceinline__ void pair32x2(u64 MH, u64 ML, u64 XH, u64 XL, u64 ETA2, u64 ONE,
                                         u64& RE, u64& IVN) {
  const u64 ND = fadd2(fsub2(MH, XH), fsub2(ML, XL));
  const u64 DEN = ffma2(ND, ND, ETA2);
  float a0, a1;
  upk2(DEN, a0, a1);
  const u64 NR0 = pk2(rcp_f32(-a0), rcp_f32(-a1));
  const u64 E = ffma2(DEN, NR0, ONE);  // 1 - den * r
  const u64 NR = ffma2(NR0, E, NR0);   // -(r + r e)
  RE = ffma2(ND, NR, RE);
  IVN = fadd2(IVN, NR);
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
