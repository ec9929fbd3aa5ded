"""The reference's Python API tests (tests/test_python_api.py of the crate),
run against shrinkers_b200 on the GPU: same calls, same expectations."""
import threading

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def sample_spectrum(p=200, seed=0):
    rng = np.random.default_rng(seed)
    return np.ascontiguousarray(np.sort(0.5 + rng.uniform(0.0, 1.5, size=p)))


def spiked_spectrum(p=300, spikes=(5.0, 7.0, 10.0), seed=1):
    bulk = sample_spectrum(p, seed)
    return np.sort(np.concatenate([bulk, np.asarray(spikes, dtype=np.float64)]))


class TestDeconvolveSpiked:
    def test_result_shape_and_keys(self, rk):
        res = rk.deconvolve_spiked(spiked_spectrum(), c=0.25, n_points=50)
        assert set(res) == {"k", "spikes", "spike_sample", "bulk_edge", "sigma2", "bulk"}
        assert isinstance(res["k"], int)
        bulk = res["bulk"]
        assert set(bulk) == {"lambda_grid", "density", "w_re", "sample_stieltjes_real",
                             "sample_stieltjes_imag", "population_stieltjes_real",
                             "population_stieltjes_imag"}
        for key in bulk:
            assert len(bulk[key]) == 50

    def test_detects_clear_spikes(self, rk):
        res = rk.deconvolve_spiked(spiked_spectrum(), c=0.25, n_points=50)
        assert res["k"] == 3
        assert res["spikes"][0] < res["spike_sample"][0]
        assert res["spikes"][0] > res["spikes"][1] > res["spikes"][2]

    def test_no_spikes_on_pure_bulk(self, rk):
        res = rk.deconvolve_spiked(sample_spectrum(), c=0.25, n_points=50)
        assert res["k"] == 0 and len(res["spikes"]) == 0

    def test_density_is_finite(self, rk):
        res = rk.deconvolve_spiked(sample_spectrum(), c=0.3, n_points=80)
        assert np.all(np.isfinite(res["bulk"]["density"]))

    def test_method_kwarg_accepted(self, rk):
        a = rk.deconvolve_spiked(sample_spectrum(120), c=0.25, n_points=40, method="blocked")
        b = rk.deconvolve_spiked(sample_spectrum(120), c=0.25, n_points=40, method="blocked_tiled")
        np.testing.assert_allclose(a["bulk"]["density"], b["bulk"]["density"], atol=1e-10)

    def test_unsorted_input_ok(self, rk):
        rng = np.random.default_rng(7)
        evals = spiked_spectrum()
        shuffled = rng.permutation(evals)
        a = rk.deconvolve_spiked(evals, c=0.25, n_points=40)
        b = rk.deconvolve_spiked(shuffled, c=0.25, n_points=40)
        assert a["k"] == b["k"]
        np.testing.assert_allclose(a["spikes"], b["spikes"], rtol=1e-12)

    def test_roundoff_negative_eigenvalues_clamped(self, rk):
        evals = sample_spectrum()
        evals[2] = -3e-15
        res = rk.deconvolve_spiked(evals, c=0.25, n_points=40)
        assert "bulk" in res

    def test_inferred_eta_is_the_bulk_default(self, rk):
        ev = spiked_spectrum()
        sentinel = rk.deconvolve_spiked(ev, c=0.25, n_points=40, eta="inferred")
        none = rk.deconvolve_spiked(ev, c=0.25, n_points=40, eta=None)
        np.testing.assert_array_equal(sentinel["bulk"]["density"], none["bulk"]["density"])


class TestStieltjesTransform:
    def test_keys_and_imag_positive_convention(self, rk):
        res = rk.stieltjes_transform(sample_spectrum(100))
        assert set(res) == {"real", "imag"}
        assert np.all(res["imag"] > 0)

    def test_exact_methods_agree(self, rk):
        evals = sample_spectrum(80)
        a = rk.stieltjes_transform(evals, method="naive")
        b = rk.stieltjes_transform(evals, method="blocked_tiled")
        np.testing.assert_allclose(a["real"], b["real"], atol=1e-11)
        np.testing.assert_allclose(a["imag"], b["imag"], atol=1e-11)

    def test_f32_dtype_and_close(self, rk):
        evals = sample_spectrum(100)
        f64 = rk.stieltjes_transform(evals, precision="f64")
        f32 = rk.stieltjes_transform(evals, precision="f32")
        assert f32["real"].dtype == np.float32
        np.testing.assert_allclose(f32["real"], f64["real"], rtol=5e-2)

    def test_parallel_matches_serial(self, rk):
        evals = sample_spectrum(150)
        serial = rk.stieltjes_transform(evals, parallel=False)
        multi = rk.stieltjes_transform(evals, parallel=True)
        auto = rk.stieltjes_transform(evals, parallel=None)
        np.testing.assert_allclose(serial["real"], multi["real"], atol=1e-12)
        np.testing.assert_allclose(serial["real"], auto["real"], atol=1e-12)

    def test_unknown_precision(self, rk):
        with pytest.raises(ValueError, match="unknown precision"):
            rk.stieltjes_transform(sample_spectrum(10), precision="f16")


class TestSpikedToolkit:
    def test_estimate_population_eigenvalues(self, rk):
        evals = spiked_spectrum()
        res = rk.estimate_population_eigenvalues(evals, c=0.25)
        assert res["k"] == 3
        assert len(res["bulk_population"]) == len(evals) - 3
        assert len(res["bulk_sample"]) == len(evals) - 3

    def test_ledoit_wolf_and_shrink_eigenvalues_lengths(self, rk):
        evals = sample_spectrum(120)
        lw = rk.ledoit_wolf_shrinkage(evals, c=0.3)
        shrunk = rk.shrink_eigenvalues(evals, c=0.3)
        assert lw.shape == (120,) and shrunk.shape == (120,)
        np.testing.assert_allclose(shrunk.sum(), evals.sum(), rtol=1e-10)

    def test_shrink_eigenvalues_method_kwarg(self, rk):
        evals = sample_spectrum(100)
        a = rk.shrink_eigenvalues(evals, c=0.3, method="autovec")
        b = rk.shrink_eigenvalues(evals, c=0.3, method="blocked_tiled", parallel=True)
        np.testing.assert_allclose(a, b, atol=1e-10)


def test_stieltjes_transform_with_deriv(rk, oracle):
    ev = sample_spectrum(300)
    eta = 0.05 / np.sqrt(300)
    res = rk.stieltjes_transform_with_deriv(ev, eta=eta)
    ref = oracle.with_deriv(ev, eta)
    for key, r in zip(["real", "imag", "deriv_real", "deriv_imag"], ref):
        np.testing.assert_allclose(res[key], r, rtol=1e-11, atol=1e-11 * np.max(np.abs(r)))


def test_gil_released_during_compute(rk):
    """test_python_api.py:635-665: the GIL is free while the kernel runs."""
    evals = sample_spectrum(20000)
    rk.stieltjes_transform(evals)  # warm the library and device state
    done = threading.Event()

    def work():
        for _ in range(20):
            rk.stieltjes_transform(evals)
        done.set()

    t = threading.Thread(target=work)
    t.start()
    spins = 0
    while not done.is_set():
        sum(range(1000))
        spins += 1
    t.join(timeout=60)
    assert not t.is_alive()
    assert spins > 50, spins


def test_nufft_matches_chebcode_fast(rk):
    """test_python_api.py:672-685."""
    p = 4000
    evals = sample_spectrum(p)
    eta = 1.0 / np.sqrt(p)
    nufft = rk.stieltjes_transform(evals, eta=eta, method="nufft")
    cheb = rk.stieltjes_transform(evals, eta=eta, method="chebcode_fast")
    num = np.linalg.norm(nufft["real"] - cheb["real"]) + np.linalg.norm(nufft["imag"] - cheb["imag"])
    den = np.linalg.norm(cheb["real"]) + np.linalg.norm(cheb["imag"])
    assert num / den < 5e-4
    alias = rk.stieltjes_transform(evals, eta=eta, method="fft_fast")
    np.testing.assert_allclose(alias["real"], nufft["real"])
