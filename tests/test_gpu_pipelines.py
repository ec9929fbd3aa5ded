"""The estimators that consume m, end to end through the Python API (GPU),
against the oracle's restatement of the reference pipelines.

Workload: the Wishart case n=4000, p=1000 (c=0.25), population
diag(12, 7, 4, 1, ..., 1), eigenvalues of X^T X / n, seed 0.
BEMA spike counts and ranks are host arithmetic and must match bit for bit;
transform-derived outputs match within 1e-12 relative (exact method) or bit
for bit (treecode presets)."""
import math

import numpy as np
import pytest

from shrinkers_b200 import spectra

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def c1():
    return spectra.config1()


def test_estimate_population_eigenvalues_c1(rk, oracle, c1):
    got = rk.estimate_population_eigenvalues(c1, c=0.25)
    ref = oracle.estimate_population_eigenvalues(c1, 0.25)
    assert got["k"] == ref["k"] == 3
    np.testing.assert_array_equal(got["spikes"], ref["spikes"])
    np.testing.assert_array_equal(got["spike_sample"], ref["spike_sample"])
    assert got["bulk_edge"] == ref["bulk_edge"] and got["sigma2"] == ref["sigma2"]
    np.testing.assert_array_equal(got["bulk_sample"], ref["bulk_sample"])
    np.testing.assert_allclose(got["bulk_population"], ref["bulk_population"], rtol=1e-12)


@pytest.mark.parametrize("method", ["blocked", "auto", "chebcode", "chebcode_fast", "nufft"])
def test_deconvolve_spiked_c1(rk, oracle, c1, method):
    got = rk.deconvolve_spiked(c1, c=0.25, method=method)
    ref = oracle.deconvolve_spiked(c1, 0.25, method=method)
    assert got["k"] == ref["k"] == 3
    np.testing.assert_array_equal(got["spikes"], ref["spikes"])
    np.testing.assert_array_equal(got["bulk"]["lambda_grid"], ref["bulk"]["lambda_grid"])
    for key in ["density", "w_re", "sample_stieltjes_real", "sample_stieltjes_imag",
                "population_stieltjes_real", "population_stieltjes_imag"]:
        a, b = got["bulk"][key], ref["bulk"][key]
        if method.startswith("cheb") or method == "auto":
            np.testing.assert_array_equal(a, b, err_msg=key)
        else:
            np.testing.assert_allclose(a, b, rtol=1e-10, atol=1e-12 * np.max(np.abs(b)),
                                       err_msg=key)


def test_deconvolve_spiked_pinned_eta(rk, oracle, c1):
    """The workload's explicit eta = 1/sqrt(p_bulk)."""
    eta = 1.0 / math.sqrt(997)
    got = rk.deconvolve_spiked(c1, c=0.25, eta=eta, method="blocked")
    ref = oracle.deconvolve_spiked(c1, 0.25, eta=eta, method="blocked")
    np.testing.assert_allclose(got["bulk"]["density"], ref["bulk"]["density"], rtol=1e-10,
                               atol=1e-13)


def test_ledoit_wolf_and_rie(rk, oracle, c1):
    lw = rk.ledoit_wolf_shrinkage(c1, c=0.25)
    np.testing.assert_allclose(lw, oracle.ledoit_wolf(c1, 0.25), rtol=1e-12)
    for method in ["blocked", "autovec", "chebcode_fast"]:
        got = rk.shrink_eigenvalues(c1, c=0.25, method=method)
        ref = oracle.rie(c1, 0.25, method=method)
        np.testing.assert_allclose(got, ref, rtol=1e-11)
    np.testing.assert_allclose(rk.shrink_eigenvalues(c1, c=0.25).sum(), c1.sum(), rtol=1e-10)


def test_stieltjes_transform_c1_all_methods(rk, oracle, c1):
    eta = 1.0 / math.sqrt(1000)
    for method in ["blocked", "blocked_tiled", "naive", "chebcode", "chebcode_fast",
                   "chebcode_xtreme", "chebcode_balanced", "nufft", "auto", "accuracy_auto"]:
        got = rk.stieltjes_transform(c1, eta=eta, method=method)
        ore, oim = oracle.compute_all(c1, eta, method)
        if method.startswith("cheb") or method == "auto":
            np.testing.assert_array_equal(got["real"], ore, err_msg=method)
            np.testing.assert_array_equal(got["imag"], oim, err_msg=method)
        else:
            scale = np.maximum(np.abs(ore), np.abs(oim))
            assert np.max((np.abs(got["real"] - ore) + np.abs(got["imag"] - oim)) / scale) < 1e-10


def test_mixed_precision_c1(rk, oracle, c1):
    eta = 1.0 / math.sqrt(1000)
    got = rk.stieltjes_transform(c1, eta=eta, precision="mixed")
    t_re, t_im = oracle.truth_points(c1, c1, eta)
    err = np.hypot(got["real"] - t_re / 1000, got["imag"] - t_im / 1000) / np.hypot(t_re, t_im) * 1000
    assert np.median(err) < 1e-9


def test_out_of_scope_methods_fail_loudly(rk, c1):
    """All-points methods without a GPU kernel raise instead of falling back
    to the CPU (at query points they are the exact per-point sum)."""
    for method in ["ewald", "hodlr"]:
        with pytest.raises(NotImplementedError, match="no GPU implementation"):
            rk.stieltjes_transform(c1, method=method)


def test_treecode_method_runs_the_fmm(rk, oracle):
    """method "fmm" / "treecode" (StieltjesMethod::TreeCode) at all points is
    the GPU's dyadic Chebyshev FMM.  The reference's own tests of its
    multipole treecode, restated: treecode.rs:303-329 (p = 1500 log spectrum,
    eta = 0.15, raw sums within 0.5 of autovec) and treecode.rs:357-393
    (p = 512, eta = 0.1/sqrt(p), max relative error of each part below
    1e-3, floor 1e-12); plus the FMM's own class at a size whose levels
    reach the tensor-core M2L (p = 2e4: median below 2e-6 of |S|)."""
    p = 1500
    ev = spectra.log_spectrum(p)
    a = rk.stieltjes_transform(ev, eta=0.15, method="fmm")
    b = rk.stieltjes_transform(ev, eta=0.15, method="treecode")
    np.testing.assert_array_equal(a["real"], b["real"])
    for i in range(100):
        r, m = oracle.autovec_sum(ev[i], ev, 0.15)
        assert abs(a["real"][i] * p - r) < 0.5 and abs(a["imag"][i] * p - m) < 0.5
    p = 512
    ev = spectra.log_spectrum(p)
    eta = 0.1 / math.sqrt(p)
    t = rk.stieltjes_transform(ev, eta=eta, method="fmm")
    e_re, e_im = oracle.compute_at_points(ev, ev, eta, "naive")
    err_r = np.abs(t["real"] * p - e_re) / np.maximum(np.abs(e_re), 1e-12)
    err_i = np.abs(t["imag"] * p - e_im) / np.maximum(np.abs(e_im), 1e-12)
    assert err_r.max() < 1e-3 and err_i.max() < 1e-3
    p = 20000
    ev = spectra.config5(p)
    eta = 1.0 / math.sqrt(p)
    t = rk.stieltjes_transform(ev, eta=eta, method="fmm")
    o_re, o_im = oracle.compute_all(ev, eta, "blocked", parallel=True)
    err = np.hypot(t["real"] - o_re, t["imag"] - o_im) / np.hypot(o_re, o_im)
    assert np.median(err) < 2e-6 and err.max() < 5e-6
