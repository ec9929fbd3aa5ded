"""The dyadic Chebyshev FMM (shrk_stieltjes_fmm) against the exact sums.

No reference counterpart exists (the crate's ChebCode is a treecode,
reproduced bit for bit by the chebcode methods), so each expansion order has
an accuracy class, measured against the oracle's exact sums (or its
double-double truth on a sample at large p) and set here with a margin:
order 10 ~1e-9, 12 ~5e-11, 16 at FP64 round-off (median relative error of
the complex value).
"""
import ctypes as C
import math

import numpy as np
import pytest

from shrinkers_b200 import _native, spectra

pytestmark = pytest.mark.gpu
_D = C.POINTER(C.c_double)
BARS = {10: 1e-8, 12: 5e-10, 16: 1e-12}


def fmm(ev, eta, order, m2l=0):
    L = _native.load()
    ev = np.ascontiguousarray(ev, dtype=np.float64)
    re, im = np.empty(ev.size), np.empty(ev.size)
    _native.check(L.shrk_stieltjes_fmm(ev.ctypes.data_as(_D), ev.size, eta, order, m2l,
                                       re.ctypes.data_as(_D), im.ctypes.data_as(_D)))
    return re, im


def rel(re, im, ore, oim):
    return np.hypot(re - ore, im - oim) / np.hypot(ore, oim)


@pytest.mark.parametrize("p", [1000, 20000])
@pytest.mark.parametrize("order", [10, 12, 16])
def test_accuracy_class_vs_exact(oracle, p, order):
    ev = spectra.config5(p)
    eta = 1.0 / math.sqrt(p)
    re, im = fmm(ev, eta, order)
    ore, oim = oracle.compute_all(ev, eta, "blocked", parallel=True)
    err = rel(re, im, ore, oim)
    assert np.median(err) < BARS[order], np.median(err)
    assert err.max() < 100 * BARS[order], err.max()


@pytest.mark.parametrize("eta_kind", ["1/sqrtp", "1e-4"])
def test_full_size_spiked(oracle, eta_kind):
    """p = 1e6 MP(c=0.1) + 20 spikes in [3, 50] at both etas of the workload:
    order 16 against the double-double truth on a sample of targets."""
    p = 1_000_000
    ev = spectra.config3(p)
    eta = 1.0 / math.sqrt(p) if eta_kind == "1/sqrtp" else 1e-4
    re, im = fmm(ev, eta, 16)
    idx = np.random.default_rng(4).choice(p, 48, replace=False)
    t_re, t_im = oracle.truth_points(ev[idx], ev, eta)
    err = rel(re[idx] * p, im[idx] * p, t_re, t_im)
    assert np.median(err) < 1e-11, np.median(err)
    assert np.all(np.isfinite(re)) and np.all(np.isfinite(im))


@pytest.mark.parametrize("p", [1, 2, 3, 47, 48, 49, 300])
def test_small_and_degenerate(oracle, p):
    ev = np.sort(np.random.default_rng(p).uniform(0.5, 2.5, p))
    eta = 0.05
    re, im = fmm(ev, eta, 16)
    ore, oim = oracle.compute_all(ev, eta, "naive")
    assert np.max(rel(re, im, ore, oim)) < 1e-12
    # repeated values: every source in one leaf at the deepest level
    ev = np.full(200, 1.25)
    ev[::7] = 0.75
    re, im = fmm(ev, eta, 12)
    ore, oim = oracle.compute_all(ev, eta, "naive")
    assert np.max(rel(re, im, ore, oim)) < 1e-12


def test_unsorted_input_and_python_api(rk, oracle):
    p = 30000
    ev = spectra.config5(p)
    perm = np.random.default_rng(9).permutation(p)
    evs = np.ascontiguousarray(ev[perm])
    eta = 1.0 / math.sqrt(p)
    re, im = fmm(ev, eta, 14)
    re2, im2 = fmm(evs, eta, 14)
    np.testing.assert_array_equal(re2, re[perm])
    np.testing.assert_array_equal(im2, im[perm])
    out = rk.stieltjes_fmm(ev, eta=eta, order=14)
    np.testing.assert_array_equal(out["real"], re)
    with pytest.raises(ValueError, match="order"):
        rk.stieltjes_fmm(ev, eta=eta, order=3)


@pytest.mark.parametrize("order", [10, 12])
def test_tensor_core_m2l_lower_orders(order):
    """The tensor-core M2L with its L2L epilogue at orders below 16 (padded
    operands, n x n side matrices): the same ~1e-6 class against the FP64
    M2L of the same order."""
    p = 50_000
    ev = spectra.config5(p)
    eta = 1.0 / math.sqrt(p)
    r64, i64 = fmm(ev, eta, order)
    rtc, itc = fmm(ev, eta, order, m2l=1)
    err = rel(rtc, itc, r64, i64)
    assert np.all(np.isfinite(rtc)) and np.all(np.isfinite(itc))
    assert np.median(err) < 2e-6, np.median(err)
    assert err.max() < 5e-6, err.max()  # measured 1.2-1.5e-6


@pytest.mark.parametrize("p", [20_000, 200_000])
def test_tensor_core_m2l(oracle, p):
    """M2L on the tensor cores (TF32 x3, FP32 accumulation): the same
    expansions, error ~1e-6 against the FP64 M2L.  Levels of at most 128
    boxes take the FP64 top-of-tree kernel in both modes, so both sizes are
    deep enough to reach the tensor-core launches."""
    ev = spectra.config5(p)
    eta = 1.0 / math.sqrt(p)
    r64, i64 = fmm(ev, eta, 16)
    L = _native.load()
    L.shrk_timing_enable(1)
    L.shrk_timing_reset()
    try:
        rtc, itc = fmm(ev, eta, 16, m2l=1)
        n_tc, ms = C.c_int64(), C.c_double()
        _native.check(L.shrk_timing_read(b"fmm_m2l_tc", C.byref(n_tc), C.byref(ms)))
    finally:
        L.shrk_timing_enable(0)
        L.shrk_timing_reset()
    assert n_tc.value >= 1  # the tcgen05 kernel ran
    err = rel(rtc, itc, r64, i64)
    assert np.all(np.isfinite(rtc)) and np.all(np.isfinite(itc))
    assert np.median(err) < 2e-6, np.median(err)
    assert err.max() < 5e-6, err.max()  # measured 1.2-1.5e-6
    if p <= 20_000:
        ore, oim = oracle.compute_all(ev, eta, "blocked", parallel=True)
        assert np.median(rel(rtc, itc, ore, oim)) < 2e-6
