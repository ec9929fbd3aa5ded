"""Scaled-ray transform and inverse nonlinear shrinkage on the GPU.

The ray sums (every point with its own eta_i = h lambda_i) are checked
against the oracle's restatement of compute_stieltjes_scaled_ray within the
exact kernels' FP64 bar (1e-12 relative per point, floor scale
max(|re|, |im|, 1e-12)); the estimator outputs within 1e-10 relative (the
reference compares its own exact kernels to each other at 1e-9 and to a
NumPy implementation at 1e-10, inverse.rs:393-423, test_python_api.py:355).
"""
import math

import numpy as np
import pytest

import shrinkers_b200 as rk
from shrinkers_b200 import spectra

pytestmark = pytest.mark.gpu


def _spectra():
    g = 0.4 + (np.arange(61) + 1.0) * 0.05            # inverse.rs test spectrum
    mp = spectra.mp_spectrum(2000, 0.4, seed=3)
    big = spectra.config5(20000, seed=8)
    perm = np.random.default_rng(4).permutation(5000)
    unsorted = spectra.mp_spectrum(5000, 0.2, seed=5)[perm]
    return [(g, 0.35), (mp, 0.4), (big, 0.3), (unsorted, 0.2)]


@pytest.mark.parametrize("case", range(4))
def test_scaled_ray_matches_oracle(oracle, case):
    ev, _ = _spectra()[case]
    h = 0.05
    r = rk.stieltjes_scaled_ray(ev, h)
    o_re, o_im = oracle.scaled_ray(ev, h)
    scale = np.maximum(np.maximum(np.abs(o_re), np.abs(o_im)), 1e-12)
    err = (np.abs(r["real"] - o_re) + np.abs(r["imag"] - o_im)) / scale
    assert np.max(err) <= 1e-12, np.max(err)


@pytest.mark.parametrize("case", range(4))
@pytest.mark.parametrize("method", ["qis", "lis", "gis"])
def test_inverse_shrinkage_matches_oracle(oracle, case, method):
    ev, c = _spectra()[case]
    r = rk.inverse_nonlinear_shrinkage(ev, c, method=method)
    o = oracle.inverse_shrinkage(ev, c, method)
    assert r["smoothing"] == o["smoothing"]
    np.testing.assert_allclose(r["precision_eigenvalues"], o["precision_eigenvalues"],
                               rtol=1e-10, atol=0)
    np.testing.assert_allclose(r["covariance_eigenvalues"], o["covariance_eigenvalues"],
                               rtol=1e-10, atol=0)


def test_qis_golden_master_through_gpu(golden):
    g = golden["qis_golden"]
    sp = g["spectrum"]
    lam = sp["base"] + (np.arange(sp["p"]) + 1.0) * sp["step"]
    r = rk.inverse_nonlinear_shrinkage(lam, g["c"])
    assert abs(r["smoothing"] / g["smoothing"] - 1.0) <= 1e-12
    for i, _, prec in g["rows"]:
        assert abs(r["precision_eigenvalues"][i] / prec - 1.0) <= g["max_relative"]


def test_python_contract():
    """The reference's Python-level behaviours (test_python_api.py:341-411)."""
    ev = spectra.mp_spectrum(120, 0.3, seed=1)
    r = rk.inverse_nonlinear_shrinkage(ev, c=0.3)
    assert set(r) == {"precision_eigenvalues", "covariance_eigenvalues", "smoothing"}
    assert r["precision_eigenvalues"].shape == (120,) and r["smoothing"] > 0
    assert np.all(np.isfinite(r["precision_eigenvalues"]))
    assert np.all(r["precision_eigenvalues"] > 0)
    ev = spectra.mp_spectrum(100, 0.4, seed=2)
    q = rk.inverse_nonlinear_shrinkage(ev, c=0.4)
    np.testing.assert_allclose(q["covariance_eigenvalues"].sum(), ev.sum(), rtol=1e-12)
    for m in ("qis", "lis", "gis", "QIS", "quadratic", "geometric_inverse"):
        out = rk.inverse_nonlinear_shrinkage(spectra.mp_spectrum(90, 0.5, seed=3), c=0.5,
                                             method=m)
        assert np.all(np.isfinite(out["precision_eigenvalues"]))
        assert np.all(out["precision_eigenvalues"] > 0)
    ev = spectra.mp_spectrum(150, 0.3, seed=4)
    seq = rk.inverse_nonlinear_shrinkage(ev, c=0.3, parallel=False)
    par = rk.inverse_nonlinear_shrinkage(ev, c=0.3, parallel=True)
    np.testing.assert_allclose(seq["precision_eigenvalues"], par["precision_eigenvalues"],
                               rtol=1e-12)


def test_qis_beats_the_naive_inverse():
    """test_python_api.py:370-383: on a sample covariance with a known
    population, QIS precision eigenvalues are closer to the truth than
    1/lambda."""
    rng = np.random.default_rng(3)
    p, n = 60, 240
    pop = np.linspace(0.5, 3.0, p)
    x = rng.standard_normal((n, p)) * np.sqrt(pop)
    lam = np.linalg.eigvalsh(x.T @ x / n)
    qis = rk.inverse_nonlinear_shrinkage(np.ascontiguousarray(lam), c=p / n)["precision_eigenvalues"]
    true = 1.0 / pop

    def err(e):
        return np.linalg.norm(np.sort(e) - np.sort(true)) / np.linalg.norm(true)

    assert err(qis) < err(1.0 / lam)
