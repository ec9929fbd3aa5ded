// FP64 epilogues applied to raw Stieltjes sums, shared by every method's
// final kernel (exact split reduction, NUFFT interpolation, treecode
// evaluation).  The arithmetic is written operation by operation as in the
// reference; the library is compiled without FMA contraction.
#pragma once

#include "internal.h"

namespace shrk {

// x: the target abscissa (eigenvalue or grid point); re/im: raw sums.
__device__ __forceinline__ void epi_store(const Epilogue& e, int64_t t, double x, double re,
                                          double im) {
  if (e.mode == EPI_SUMS) {
    e.out_re[t] = re * e.scale;
    e.out_im[t] = im * e.scale;
  } else if (e.mode == EPI_LW) {
    // shrinkage.rs:22-34 on the scaled pair (mod.rs:216-237 map_stieltjes)
    const double li = x, c = e.c;
    const double mr = re * e.scale, mi = im * e.scale;
    const double tr = c * li * mr, ti = c * li * mi;
    const double dr = 1.0 - c + tr, di = ti;
    const double n2 = dr * dr + di * di;
    e.out_re[t] = n2 > 0.0 ? li / n2 : li;
  } else if (e.mode == EPI_MP) {
    // deconvolution/mod.rs:206-248 on the raw grid sums
    const double zr = x, zi = e.eta, c = e.c, inv_p = e.scale;
    const double gr = -re * inv_p, gi = im * inv_p;
    const double zgr = zr * gr - zi * gi, zgi = zr * gi + zi * gr;
    const double ar = 1.0 - c - c * zgr, ai = -c * zgi;
    const double an = ar * ar + ai * ai;
    const double wr = an > 0.0 ? (zr * ar + zi * ai) / an : zr;
    const double mr = ar * gr - ai * gi, mi = ar * gi + ai * gr;
    e.out[0][t] = mi / 3.141592653589793;
    e.out[1][t] = wr;
    e.out[2][t] = gr;
    e.out[3][t] = gi;
    e.out[4][t] = mr;
    e.out[5][t] = mi;
  }
}

}  // namespace shrk
