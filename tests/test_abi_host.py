"""C ABI and host logic, CPU only (no compute call reaches a GPU here).

* libshrinkers_b200.so loads and exports every function that
  include/*.h declares, and the Python binding covers them all;
* the host-side policy (parse_method, auto resolution, grid redirect) and the
  host estimators (BEMA, inverse BBP, shrinkage factor) agree with the oracle;
* the Python boundary raises the reference's errors before touching a GPU.
"""
import ctypes as C
import glob
import os
import re

import numpy as np
import pytest

from shrinkers_b200 import _native, spectra

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_functions():
    text = ""
    for h in sorted(glob.glob(os.path.join(ROOT, "include", "*.h"))):
        text += open(h).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(shrk_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    L = _native.load()
    names = header_functions()
    assert len(names) >= 30
    for n in names:
        assert hasattr(L, n), f"{n} declared but not exported"
        assert n in _native.SIGNATURES, f"{n} not bound in _native.SIGNATURES"
    for n in _native.SIGNATURES:
        assert n in names, f"{n} bound but not declared in the header"


METHOD_ALIASES = {  # python.rs:321-350
    "naive": "naive", "autovec": "autovec", "blocked": "blocked",
    "blocked_autovec": "blocked_autovec", "blocked_tiled": "blocked_tiled",
    "blocked_windowed": "blocked_windowed", "blocked_hybrid": "blocked_hybrid",
    "adaptive": "adaptive", "fft5": "fft5", "fft3": "fft3", "fft2": "fft2",
    "nufft": "nufft", "fft_fast": "nufft", "fmm": "fmm", "treecode": "fmm",
    "chebcode": "chebcode", "chebyshev": "chebcode", "chebcode_fast": "chebcode_fast",
    "chebf": "chebcode_fast", "chebcode_xtreme": "chebcode_xtreme", "chebx": "chebcode_xtreme",
    "chebcode_balanced": "chebcode_balanced", "chebb": "chebcode_balanced", "ewald": "ewald",
    "dst": "dst", "auto": "auto", "hodlr": "hodlr", "speed_auto": "speed_auto",
    "speed": "speed_auto", "accuracy_auto": "accuracy_auto", "accuracy": "accuracy_auto",
}


def test_parse_method_accepts_every_alias(rk):
    for alias, canonical in METHOD_ALIASES.items():
        assert rk.method_name(rk.parse_method(alias)) == canonical
    with pytest.raises(ValueError, match="unknown method 'warp9'"):
        rk.parse_method("warp9")


def test_auto_resolution_matches_oracle(oracle):
    L = _native.load()
    for m in ["auto", "speed_auto", "accuracy_auto", "blocked", "nufft"]:
        for par in (0, 1):
            for p in [1, 500, 1000, 1001, 1500, 4000, 9000, 15000, 30000, 50000, 50001, 200000]:
                mid = oracle.M[m]
                assert L.shrk_resolve_auto_method(mid, par, p) == \
                    oracle.lib().orc_resolve_auto_method(mid, par, p)
    for m in oracle.METHODS:
        for p, nq in [(50_000, 200), (200_000, 200), (300_000, 200), (1000, 250), (1000, 249)]:
            assert L.shrk_grid_appropriate(oracle.M[m], p, nq) == \
                oracle.lib().orc_grid_appropriate(oracle.M[m], p, nq)


def test_host_estimators_bit_exact(oracle):
    """BEMA, inverse BBP, the MP median factor and the shrinkage factor are
    host arithmetic; they must equal the oracle bit for bit."""
    L = _native.load()
    rng = np.random.default_rng(3)
    for g in np.linspace(0.01, 1.0, 23):
        assert L.shrk_mp_median_factor(g) == oracle.mp_median_factor(g)
        for lh in rng.uniform(0.5, 40.0, 10):
            assert L.shrk_inverse_bbp(lh, g, 1.3) == oracle.inverse_bbp(lh, g, 1.3)
    for _ in range(50):
        a = rng.uniform(-3, 3, 4)
        assert L.shrk_shrinkage_factor(*a) == oracle.shrinkage_factor(*a)
    ev = spectra.config1()
    for c, margin in [(0.25, 1.0), (0.25, 1.05), (0.1, 1.0), (0.9, 1.2)]:
        k = C.c_size_t()
        idx = np.empty(ev.size, np.int64)
        e, s2 = C.c_double(), C.c_double()
        L.shrk_detect_spikes_bema(ev.ctypes.data_as(C.POINTER(C.c_double)), ev.size, c, margin,
                                  C.byref(k), idx.ctypes.data_as(C.POINTER(C.c_int64)),
                                  C.byref(e), C.byref(s2))
        ref = oracle.bema(ev, c, margin)
        assert k.value == ref["k"]
        assert list(idx[:k.value]) == list(ref["spike_indices"])
        assert e.value == ref["bulk_edge"] and s2.value == ref["sigma2"]


def test_config1_bema_detects_three_spikes(oracle):
    ev = spectra.config1()
    r = oracle.bema(ev, 0.25, 1.0)
    assert r["k"] == 3
    assert list(r["spike_indices"]) == [997, 998, 999]


# ------------------------------------------------ boundary validation --
# python.rs error contract (tests/test_python_api.py:132-161, 499-569).
def sample_spectrum(p=200, seed=0):
    rng = np.random.default_rng(seed)
    return np.ascontiguousarray(np.sort(0.5 + rng.uniform(0.0, 1.5, size=p)))


def spiked_spectrum(p=300, spikes=(5.0, 7.0, 10.0), seed=1):
    return np.sort(np.concatenate([sample_spectrum(p, seed), np.asarray(spikes, dtype=np.float64)]))


def test_stieltjes_transform_validation(rk):
    with pytest.raises(ValueError, match="non-empty"):
        rk.stieltjes_transform(np.array([], dtype=np.float64))
    with pytest.raises(ValueError, match="eta"):
        rk.stieltjes_transform(sample_spectrum(50), eta=-0.1)
    with pytest.raises(TypeError):
        rk.stieltjes_transform(sample_spectrum(50), parallel="yes")
    with pytest.raises(ValueError, match="contiguous"):
        rk.stieltjes_transform(sample_spectrum(20)[::2])
    bad = sample_spectrum(20)
    bad[3] = np.nan
    with pytest.raises(ValueError, match="finite"):
        rk.stieltjes_transform(bad)
    with pytest.raises(ValueError, match="unknown method"):
        rk.stieltjes_transform(sample_spectrum(20), method="warp9")
    with pytest.raises(ValueError, match="cutoff"):
        rk.stieltjes_transform(sample_spectrum(20), cutoff=-1.0)
    with pytest.raises(ValueError, match="expected a float, None, or the string 'inferred'"):
        rk.stieltjes_transform(sample_spectrum(20), eta="sometimes")


def test_deconvolve_spiked_validation(rk):
    ev = sample_spectrum()
    bad = ev.copy()
    bad[3] = np.nan
    with pytest.raises(ValueError, match="finite"):
        rk.deconvolve_spiked(bad, c=0.25)
    bad = ev.copy()
    bad[2] = -1.0
    with pytest.raises(ValueError, match="non-negative"):
        rk.deconvolve_spiked(bad, c=0.25)
    with pytest.raises(ValueError, match="concentration"):
        rk.deconvolve_spiked(ev, c=0.0)
    with pytest.raises(ValueError, match="concentration"):
        rk.deconvolve_spiked(ev, c=1.5)
    with pytest.raises(ValueError, match="unknown method"):
        rk.deconvolve_spiked(ev, c=0.25, method="warp9")
    for bad_eta in [0.0, -0.1, float("nan"), float("inf")]:
        with pytest.raises(ValueError, match="eta"):
            rk.deconvolve_spiked(spiked_spectrum(), c=0.25, eta=bad_eta)
    with pytest.raises(ValueError, match="n_points"):
        rk.deconvolve_spiked(ev, c=0.25, n_points=0)


@pytest.mark.parametrize("margin", [0.0, -1.0, float("nan")])
def test_margin_rejected_everywhere(rk, margin):
    ev = spiked_spectrum()
    with pytest.raises(ValueError, match="margin"):
        rk.detect_spikes_bema(ev, c=0.25, margin=margin)
    with pytest.raises(ValueError, match="margin"):
        rk.estimate_population_eigenvalues(ev, c=0.25, margin=margin)
    with pytest.raises(ValueError, match="margin"):
        rk.deconvolve_spiked(ev, c=0.25, n_points=20, margin=margin)


def test_inverse_bbp_validation_and_values(rk, oracle):
    with pytest.raises(ValueError, match="lambda_hat"):
        rk.inverse_bbp(-1.0, c=0.25)
    with pytest.raises(ValueError, match="lambda_hat"):
        rk.inverse_bbp(float("nan"), c=0.25)
    ell = rk.inverse_bbp(6.0, c=0.25, sigma2=1.0)
    assert isinstance(ell, float) and ell == oracle.inverse_bbp(6.0, 0.25, 1.0)
    out = rk.inverse_bbp(np.array([6.0, 8.0]), c=0.25, sigma2=1.0)
    assert out.shape == (2,) and np.all(out < [6.0, 8.0])


def test_detect_spikes_bema_host(rk):
    res = rk.detect_spikes_bema(spiked_spectrum(), c=0.25)
    assert set(res) == {"k", "spike_indices", "bulk_edge", "sigma2"}
    assert res["k"] == 3 and res["sigma2"] > 0


def test_non_ndarray_input_is_type_error(rk):
    with pytest.raises(TypeError):
        rk.stieltjes_transform([1.0, 2.0, 3.0])
    with pytest.raises(TypeError):
        rk.stieltjes_transform(np.arange(5, dtype=np.float32))


def test_treecode_adjoint_rejects_non_treecode_methods(rk):
    """The method check runs on the host before any device work."""
    import ctypes as C
    L = _native.load()
    x = np.ones(4)
    D = C.POINTER(C.c_double)
    st = L.shrk_stieltjes_adjoint_treecode(x.ctypes.data_as(D), 4, 0.5, x.ctypes.data_as(D),
                                           x.ctypes.data_as(D), 2, x.ctypes.data_as(D))
    assert st == _native.SHRK_EINVAL
    assert "ChebCode" in _native.last_error()


def test_inverse_shrinkage_validation(rk):
    """python.rs:202-216 and 353-359 messages; checked before any device work."""
    with pytest.raises(ValueError, match="strictly positive"):
        rk.inverse_nonlinear_shrinkage(np.array([0.0, 1.0, 2.0]), c=0.3)
    with pytest.raises(ValueError, match="unknown inverse shrinkage"):
        rk.inverse_nonlinear_shrinkage(np.array([1.0, 2.0]), c=0.3, method="nope")
    with pytest.raises(ValueError):
        rk.inverse_nonlinear_shrinkage(np.array([1.0, 2.0]), c=1.5)
