"""The oracle pinned against the reference's own golden vectors, known
answers and tolerance suite (CPU only).

Fixtures come from tests/golden/reference_vectors.json (extracted from the
crate's test modules by tests/golden/make_golden.py); tolerances are the
reference's own, cited per test.
"""
import numpy as np
import pytest

from shrinkers_b200 import spectra


def rel_l2(a_re, a_im, b_re, b_im):
    num = np.sqrt(np.sum((a_re - b_re) ** 2 + (a_im - b_im) ** 2))
    return num / np.sqrt(np.sum(b_re ** 2 + b_im ** 2))


# ---------------------------------------------------------------- golden --
def test_golden_master_regression(oracle, golden):
    """deconvolution/mod.rs:281-399: El Karoui inversion at epsilon 1e-14."""
    g = golden["golden_master"]
    r = oracle.spectral_deconvolution(np.array(g["evals"]), g["c"], g["n_points"], eta=g["eta"],
                                      method="blocked")
    for key in ["density", "w_re", "sample_stieltjes_imag", "population_stieltjes_imag"]:
        np.testing.assert_allclose(r[key], g[key], rtol=0, atol=g["epsilon"])


def test_empirical_at_point_known_answer(oracle, golden):
    """deconvolution/mod.rs:646-665: Im g_A(2+0.1i) = -10.198.../3 for {1,2,3}."""
    g = golden["empirical_at_point"]
    re, im = oracle.compute_at_points([g["z"][0]], g["evals"], g["z"][1], method="naive")
    p = len(g["evals"])
    # convention A = -S/p (mod.rs:67-84)
    assert abs(-re[0] / p - g["ga_real"]) < 1e-12
    assert abs(-im[0] / p - g["ga_imag"]) < 1e-10


def test_term_basic(oracle, golden):
    """term.rs:52-57."""
    g = golden["term_basic"]
    r, i = oracle.term(*g["args"])
    assert abs(r - g["expected"][0]) < g["tol"]
    assert abs(i - g["expected"][1]) < g["tol"]


def test_symmetric_sweep_known_cases(oracle, golden):
    """cacheblock.rs:1580-1624: unsorted 7 values, p = 1, sym vs full square."""
    g = golden["symmetric_small"]
    ev = np.array(g["evals"])
    re, im = oracle.symmetric_sweep(ev, g["eta"])
    for i, li in enumerate(ev):
        r, m = oracle.autovec_sum(li, ev, g["eta"])
        assert abs(re[i] - r) < g["tol"] and abs(im[i] - m) < g["tol"]
    r1, i1 = oracle.symmetric_sweep([g["p1"]["lambda"]], g["p1"]["eta"])
    assert r1[0] == 0.0
    assert abs(i1[0] - g["p1"]["im"]) < 1e-15
    big = np.sort([((i * 7919) % 9973) / 9973.0 * 4.0 - 2.0 for i in range(g["big"]["n"])])
    sr, si = oracle.symmetric_sweep(big, g["big"]["eta"])
    pr, pi = oracle.tiled_full_square(big, g["big"]["eta"])
    scale = np.maximum(np.maximum(np.abs(sr), np.abs(si)), 1e-12)
    assert np.max((np.abs(pr - sr) + np.abs(pi - si)) / scale) < g["big"]["tol"]


def test_inverse_bbp_roundtrip(oracle, golden):
    """estimation.rs:98-108 (+ threshold 120-126)."""
    g = golden["inverse_bbp_roundtrip"]
    for ell in g["ells"]:
        lh = ell * (1.0 + g["gamma"] / (ell - 1.0))
        assert abs(oracle.inverse_bbp(lh, g["gamma"], g["sigma2"]) - ell) < g["tol"]
    t = golden["bbp_threshold"]
    assert abs(oracle.bbp_threshold(t["gamma"], t["sigma2"]) - t["expected"]) < t["tol"]
    edge = oracle.bbp_threshold(0.5, 1.0)
    assert abs(oracle.inverse_bbp(edge, 0.5, 1.0) - edge) < 1e-10


def test_bema_known_counts(oracle, golden):
    """detection.rs:286-311."""
    g = golden["bema_known"]
    b = g["bulk"]
    ev = np.sort(np.concatenate([b["start"] + b["step"] * np.arange(b["n"]), g["spikes"]]))
    r = oracle.bema(ev, g["gamma"], g["margin"])
    assert r["k"] == g["k"]
    assert 2.0 < r["bulk_edge"] < 5.0
    g = golden["bema_none"]
    b = g["bulk"]
    ev = b["start"] + b["step"] * np.arange(b["n"])
    assert oracle.bema(ev, g["gamma"], g["margin"])["k"] == g["k"]
    for gam, want, tol in golden["mp_median_factor"]["points"]:
        assert abs(oracle.mp_median_factor(gam) - want) < tol


def test_nufft_grid_pins(oracle, golden):
    """nufft.rs:229-250."""
    for raw, eta, m in golden["nufft_grid"]["cases"]:
        assert oracle.nufft_grid_size(raw, eta) == m


def test_auto_resolution_pins(oracle, golden):
    """config.rs:592-658 + at-points redirect 661-713."""
    for par, p, meth in golden["auto_resolution"]["cases"]:
        name = {"ChebCodeFast": "chebcode_fast", "Nufft": "nufft"}[meth]
        assert oracle.lib().orc_resolve_auto_method(oracle.M["auto"], int(par), p) == oracle.M[name]
    ga = oracle.lib().orc_grid_appropriate
    assert ga(oracle.M["nufft"], 200_000, 200) == oracle.M["chebcode_fast"]
    assert ga(oracle.M["nufft"], 300_000, 200) == oracle.M["nufft"]
    assert ga(oracle.M["fft5"], 50_000, 200) == oracle.M["chebcode_fast"]
    assert ga(oracle.M["chebcode"], 50_000, 200) == oracle.M["chebcode"]


# ------------------------------------------------------ tolerance suite --
def test_all_exact_methods_agree(oracle):
    """mod.rs:858-913: every exact method vs naive at p=50, 1e-13."""
    ev = np.log1p((np.arange(50) + 0.5) * 0.2)
    eta = 0.05
    ref = np.array([oracle.naive_sum(li, ev, eta) for li in ev]) / 50.0
    for m in ["naive", "autovec", "blocked", "blocked_tiled", "blocked_windowed",
              "blocked_hybrid"]:
        re, im = oracle.compute_all(ev, eta, m)
        assert np.max(np.abs(re - ref[:, 0])) < 1e-13, m
        assert np.max(np.abs(im - ref[:, 1])) < 1e-13, m


@pytest.mark.parametrize("p", [300, 2001, 2002, 2003, 4001])
def test_tiled_parallel_matches_sequential(oracle, p):
    """mod.rs:1035-1085: includes p % 4 != 0 (the remainder-bug class), 1e-12."""
    ev = spectra.log_spectrum(p)
    eta = 0.1 / np.sqrt(p)
    s_re, s_im = oracle.compute_all(ev, eta, "blocked", parallel=False)
    p_re, p_im = oracle.compute_all(ev, eta, "blocked", parallel=True)
    scale = np.maximum(np.maximum(np.abs(s_re), np.abs(s_im)), 1e-12)
    assert np.max((np.abs(p_re - s_re) + np.abs(p_im - s_im)) / scale) < 1e-12


@pytest.mark.parametrize("nt,p", [(1, 5), (31, 1001), (33, 2002), (100, 4003), (64, 4000)])
def test_tiled_block_shape_is_bit_identical(oracle, nt, p):
    """The block-shaped route (32-target blocks x source quads, the
    reference's loop shape) gives every target the same sums as one chain
    per target, in both ISA builds: ragged blocks and p % 4 tails included."""
    ev = spectra.log_spectrum(p)
    eta = 1.0 / np.sqrt(p)
    t = ev[np.linspace(0, p - 1, nt).astype(np.int64)]
    base = oracle.tiled_targets(t, ev, eta, "target", "v2")
    isas = ["v2", "v3"] if oracle.host_has_v3() else ["v2"]
    for shape in ["block", "target"]:
        for isa in isas:
            re, im = oracle.tiled_targets(t, ev, eta, shape, isa)
            assert np.array_equal(re, base[0]) and np.array_equal(im, base[1]), (shape, isa)


def test_with_deriv_matches_finite_difference(oracle):
    """autovec.rs:115-148."""
    p = 300
    ev = spectra.log_spectrum(p)
    eta = 0.05 / np.sqrt(p)
    re, im, dre, dim = oracle.with_deriv(ev, eta)
    for i in range(0, p, 37):
        r, m = oracle.autovec_sum(ev[i], ev, eta)
        assert abs(re[i] - r) < 1e-10 and abs(im[i] - m) < 1e-10
    for i in [0, 1, p // 3, p - 1]:
        h = min(1e-5, max(abs(ev[i]), 1.0) * 1e-5)
        rp, ip = oracle.autovec_sum(ev[i] + h, ev, eta)
        rm, imm = oracle.autovec_sum(ev[i] - h, ev, eta)
        fd = ((rp - rm) / (2 * h), (ip - imm) / (2 * h))
        tol = 8e-2 if i == 0 else 5e-4
        assert abs(dre[i] - fd[0]) < tol * (abs(fd[0]) + 1.0)
        assert abs(dim[i] - fd[1]) < tol * (abs(fd[1]) + 1.0)


@pytest.mark.parametrize("p", [512, 2000, 8000])
def test_chebcode_default_accuracy(oracle, p):
    """chebcode.rs:1401-1419: DEFAULT preset max rel < 1e-2."""
    ev = spectra.log_spectrum(p)
    eta = 0.1 / np.sqrt(p)
    ex_re, ex_im = oracle.compute_all(ev, eta, "blocked", parallel=True)
    cr, ci = oracle.compute_all(ev, eta, "chebcode", parallel=True)
    scale = np.maximum(np.abs(ex_re) + np.abs(ex_im), 1e-12)
    assert np.max((np.abs(cr - ex_re) + np.abs(ci - ex_im)) / scale) < 1e-2


def test_chebcode_presets_error_classes(oracle):
    """Preset error classes (chebcode.rs:939-972, RESULT.md) on an MP spectrum."""
    p = 8000
    ev = spectra.config2(p)
    eta = 1.0 / np.sqrt(p)
    ex_re, ex_im = oracle.compute_all(ev, eta, "blocked", parallel=True)
    for name, tol in [("chebcode_fast", 5e-5), ("chebcode", 5e-8), ("chebcode_balanced", 5e-8),
                      ("chebcode_xtreme", 1e-10)]:
        r, i = oracle.compute_all(ev, eta, name, parallel=True)
        assert rel_l2(r, i, ex_re, ex_im) < tol, name


def test_chebcode_unsorted_input(oracle):
    """chebcode.rs:1366-1399: shuffled input, results in input order."""
    p = 512
    ev = spectra.log_spectrum(p)
    perm = np.random.default_rng(7).permutation(p)
    r1, i1 = oracle.compute_all(ev, 0.05, "chebcode")
    r2, i2 = oracle.compute_all(ev[perm], 0.05, "chebcode")
    np.testing.assert_allclose(r2, r1[perm], rtol=0, atol=1e-12)
    np.testing.assert_allclose(i2, i1[perm], rtol=0, atol=1e-12)


def test_nufft_matches_exact_and_parallel(oracle):
    """nufft.rs:252-318: rel-L2 < 1e-4 at p=8192, eta=1/sqrt(p), seq/par < 1e-9."""
    p = 8192
    ev = spectra.log_spectrum(p)
    eta = 1.0 / np.sqrt(p)
    ex_re, ex_im = oracle.compute_all(ev, eta, "blocked", parallel=True)
    got = oracle.nufft_points(ev, ev, eta, parallel=False)
    assert rel_l2(got[0] / p, got[1] / p, ex_re, ex_im) < 1e-4
    par = oracle.nufft_points(ev, ev, eta, parallel=True)
    assert np.max(np.maximum(np.abs(got[0] - par[0]), np.abs(got[1] - par[1]))) < 1e-9
    grid = ev[0] + (ev[-1] - ev[0]) * np.arange(200) / 199.0
    eg = oracle.compute_at_points(grid, ev, eta, "blocked", parallel=True)
    gg = oracle.nufft_points(grid, ev, eta)
    assert rel_l2(gg[0], gg[1], eg[0], eg[1]) < 1e-4


def test_fft_matches_dft(oracle):
    """The oracle's own radix-2 FFT against a direct DFT (rustfft contract)."""
    rng = np.random.default_rng(0)
    x = rng.standard_normal(256) + 1j * rng.standard_normal(256)
    np.testing.assert_allclose(oracle.fft(x, -1), np.fft.fft(x), rtol=0, atol=1e-11)
    np.testing.assert_allclose(oracle.fft(x, +1), np.fft.ifft(x) * 256, rtol=0, atol=1e-11)


@pytest.mark.parametrize("m", [3, 7, 100, 3000])
def test_fft_any_length_matches_numpy(oracle, m):
    """Lengths that are not a power of two (a forced fft5 grid_size; rustfft
    plans any length): the oracle's direct DFT against numpy's FFT."""
    rng = np.random.default_rng(m)
    x = rng.standard_normal(m) + 1j * rng.standard_normal(m)
    tol = 1e-14 * m
    np.testing.assert_allclose(oracle.fft(x, -1), np.fft.fft(x), rtol=0, atol=tol)
    np.testing.assert_allclose(oracle.fft(x, +1), np.fft.ifft(x) * m, rtol=0, atol=tol)


def test_lagrange_partition_of_unity(oracle):
    """fft5.rs:774-804: every stencil width, t = s/97 for s in 0..97."""
    for t in np.linspace(0, 0.999, 17):
        assert abs(oracle.lagrange4(t).sum() - 1.0) < 1e-14
    for n in (2, 4, 6, 8):
        for s in range(97):
            w = oracle.lagrange(n, s / 97.0)
            assert abs(w.sum() - 1.0) < 1e-12
            assert np.all(np.isfinite(w)) and np.all(np.abs(w) < 10.0)


# ------------------------------------------------------------------- fft5 --
_ORDERS = {"linear": 2, "cubic": 4, "quintic": 6, "heptic": 8}


def _harness_exact(oracle, p, cache={}):
    if p not in cache:
        ev = spectra.harness_spectrum(p)
        eta = 1.0 / np.sqrt(p)
        cache[p] = (ev, eta, *oracle.compute_all(ev, eta, "blocked_tiled", parallel=True))
    return cache[p]


def test_fft5_reproduces_the_reference_order_sweep(oracle, golden):
    """The reference's own measured fft5 errors (docs/pareto/order_sweep.jsonl,
    144 rows: p in {1000, 5000, 20000}, 4 stencils, forced and adaptive grids,
    6 paddings) are reproduced by the restatement to the 4 printed digits."""
    g = golden["fft5_order_sweep"]
    worst = 0.0
    for r in g["rows"]:
        ev, eta, ere, eim = _harness_exact(oracle, r["p"])
        kw = dict(order=_ORDERS[r["order"]], m=r["m"])
        if r["kind"] == "pad":
            kw["pad_eta_mult"] = float(r["pad_mult"])
        gre, gim = oracle.fft5_points(ev, ev, eta, **kw)
        # support/mod.rs:126-135 rel_l2_scaled: raw sums times 1/len
        err = rel_l2(gre / ev.size, gim / ev.size, ere, eim)
        worst = max(worst, abs(err - r["err"]) / r["err"])
    assert worst < 1e-3, worst


def test_fft5_adaptive_grid_sizes(oracle, golden):
    """The adaptive grid (m = null rows) is the forced grid whose error it
    repeats: 32768 at p = 1000, 65536 at 5000, 262144 at 20000."""
    rows = golden["fft5_order_sweep"]["rows"]
    for p, m in [(1000, 32768), (5000, 65536), (20000, 262144)]:
        ev = spectra.harness_spectrum(p)
        assert oracle.fft5_grid_size(ev, 1.0 / np.sqrt(p)) == m
        auto = {r["order"]: r["err"] for r in rows if r["kind"] == "grid" and r["p"] == p
                and r["m"] is None}
        forced = {r["order"]: r["err"] for r in rows if r["kind"] == "grid" and r["p"] == p
                  and r["m"] == m}
        assert auto == forced


def test_fft5_pipeline_ordering(oracle, golden):
    """fft5.rs:874-925: at a forced m = 8192 the error orders heptic <= cubic
    < linear (the test's 1/p excludes the two outliers)."""
    g = golden["fft5_pipeline_ordering"]
    p, c = g["p"], g["c"]
    lo, hi = (1 - np.sqrt(c)) ** 2, (1 + np.sqrt(c)) ** 2
    ev = np.sort(np.concatenate([lo + ((np.arange(p) + 0.5) / p) * (hi - lo),
                                 [hi * 2.3, lo * 0.35]]))
    eta = 1.0 / np.sqrt(p)
    ere, eim = oracle.compute_all(ev, eta, "blocked_tiled")
    err = {}
    for n in (2, 4, 8):
        gre, gim = oracle.fft5_points(ev, ev, eta, order=n, m=g["m"])
        err[n] = rel_l2(gre / p, gim / p, ere, eim)
    assert err[4] < err[2] and err[8] <= err[4]


def test_fft_family_dispatch(oracle):
    """mod.rs:634-641 / 672-690, adaptive.rs:43-68: fft5/fft3/fft2 are one
    kernel; adaptive = fft5 real part + windowed imaginary part (ratio 10 by
    default); dst = fft5 real part + the caller's window, or the exact
    imaginary part without one; the single-point fallback of every other grid
    method is the autovec sum (mod.rs:265-287)."""
    p = 3000
    ev = spectra.log_spectrum(p)
    eta = 0.1 / np.sqrt(p)
    f5 = oracle.compute_all(ev, eta, "fft5")
    for name in ("fft3", "fft2"):
        r = oracle.compute_all(ev, eta, name)
        np.testing.assert_array_equal(r[0], f5[0])
        np.testing.assert_array_equal(r[1], f5[1])
    win = oracle.compute_all(ev, eta, "blocked_windowed", cutoff=10.0)
    ad = oracle.compute_all(ev, eta, "adaptive")
    np.testing.assert_array_equal(ad[0], f5[0])
    np.testing.assert_array_equal(ad[1], win[1])
    win7 = oracle.compute_all(ev, eta, "blocked_windowed", cutoff=7.0)
    ds = oracle.compute_all(ev, eta, "dst", cutoff=7.0)
    np.testing.assert_array_equal(ds[0], f5[0])
    np.testing.assert_array_equal(ds[1], win7[1])
    ex = oracle.compute_all(ev, eta, "blocked")
    ds0 = oracle.compute_all(ev, eta, "dst")
    np.testing.assert_array_equal(ds0[1], ex[1])
    # adaptive.rs:76-99: finite everywhere
    assert np.all(np.isfinite(ad[0])) and np.all(np.isfinite(ad[1]))
    q = np.linspace(ev[0], ev[-1], 50)
    av = oracle.compute_at_points(q, ev, eta, "autovec")
    for name in ("adaptive", "dst", "treecode", "ewald", "hodlr"):
        r = oracle.compute_at_points(q, ev, eta, name)
        np.testing.assert_array_equal(r[0], av[0])
    fq = oracle.compute_at_points(q, ev, eta, "fft5")
    fp = oracle.fft5_points(q, ev, eta)
    np.testing.assert_array_equal(fq[0], fp[0])


def test_truth_matches_exact(oracle):
    """The double-double truth agrees with the FP64 sums to ~1e-14."""
    ev = spectra.config2(2000)
    eta = 1.0 / np.sqrt(2000)
    tr, ti = oracle.truth_points(ev, ev, eta)
    er, ei = oracle.compute_all(ev, eta, "blocked")
    assert rel_l2(tr / 2000, ti / 2000, er, ei) < 1e-13


def test_adjoint_direct_matches_finite_difference(oracle):
    """FP64 direct-sum gradient vs central differences (h = 1e-6)."""
    p = 400
    ev = spectra.config5(p)
    eta = 1.0 / np.sqrt(p)
    rng = np.random.default_rng(5)
    w, v = rng.standard_normal(p), rng.standard_normal(p)
    idx = np.random.default_rng(6).choice(p, 16, replace=False)
    g = oracle.adjoint_direct(ev, eta, w, v, idx)

    def loss(x):
        # m = -conj(S)/p: Re m = -Re S/p, Im m = Im S/p (truth in double-double)
        re, im = oracle.truth_points(x, x, eta)
        return np.sum(w * (-re / p) + v * (im / p))

    h = 1e-6
    for t, k in enumerate(idx):
        xp, xm = ev.copy(), ev.copy()
        xp[k] += h
        xm[k] -= h
        fd = (loss(xp) - loss(xm)) / (2 * h)
        assert abs(fd - g[t]) < 1e-5 * max(1.0, abs(g[t])), (k, fd, g[t])


def test_lw_and_population_pipeline_shapes(oracle):
    """population.rs:126-169 and hybrid.rs:150-200 behaviours on the oracle."""
    bulk = 0.5 + 0.015 * np.arange(100)
    ev = np.concatenate([bulk, [5.0, 7.0, 10.0]])
    r = oracle.estimate_population_eigenvalues(ev, 0.25)
    assert r["k"] == 3 and len(r["bulk_population"]) == 100
    assert r["spikes"][0] > r["spikes"][1] > r["spikes"][2]
    assert np.all(r["spikes"] < r["spike_sample"])
    d = oracle.deconvolve_spiked(ev, 0.25, 100, eta=0.1, method="blocked")
    assert d["k"] == 3 and np.all(np.isfinite(d["bulk"]["density"]))
    lw = oracle.ledoit_wolf(bulk, 0.25)
    np.testing.assert_allclose(r["bulk_population"][:0], lw[:0])
    # no-spike path delegates to plain LW (population.rs:131-145)
    ev0 = 0.5 + 0.01 * np.arange(100)
    r0 = oracle.estimate_population_eigenvalues(ev0, 0.25)
    np.testing.assert_allclose(r0["bulk_population"], oracle.ledoit_wolf(ev0, 0.25), atol=1e-12)


def _qis_spectrum(g):
    sp = g["spectrum"]
    return sp["base"] + (np.arange(sp["p"]) + 1.0) * sp["step"]


def test_inverse_shrinkage_qis_golden_master(oracle, golden):
    """inverse.rs:426 qis_golden_master: smoothing, theta and precision pins."""
    g = golden["qis_golden"]
    r = oracle.inverse_shrinkage(_qis_spectrum(g), g["c"], "qis")
    assert abs(r["smoothing"] / g["smoothing"] - 1.0) <= 1e-12
    for i, theta, prec in g["rows"]:
        assert abs(r["theta"][i] / theta - 1.0) <= g["max_relative"]
        assert abs(r["precision_eigenvalues"][i] / prec - 1.0) <= g["max_relative"]


def test_scaled_ray_is_theta_by_definition(oracle, golden):
    """theta_i + i Htheta_i = lambda_i m(lambda_i (1 + i h)): the ray sums equal
    the inverse-shrinkage shrinkers written in the inverse eigenvalues
    x = 1/lambda (1e-12 absolute, as inverse.rs:308-320)."""
    g = golden["qis_golden"]
    lam = _qis_spectrum(g)
    r = oracle.inverse_shrinkage(lam, g["c"], "qis")
    h, p = r["smoothing"], lam.size
    x = 1.0 / lam
    diff = x[None, :] - x[:, None]            # x_j - x_i
    den = diff ** 2 + (x[None, :] * h) ** 2
    theta = np.sum(x[None, :] * diff / den, axis=1) / p
    htheta = np.sum(x[None, :] ** 2 * h / den, axis=1) / p
    np.testing.assert_allclose(r["theta"], theta, rtol=0, atol=1e-12)
    np.testing.assert_allclose(r["htheta"], htheta, rtol=0, atol=1e-12)


def test_inverse_shrinkage_properties(oracle, golden):
    """QIS preserves the trace; GIS is the geometric mean of QIS (unscaled)
    and LIS (inverse.rs:323-399)."""
    g = golden["qis_golden"]
    lam = _qis_spectrum(g)
    c = 0.45
    q = oracle.inverse_shrinkage(lam, c, "qis")
    np.testing.assert_allclose(q["covariance_eigenvalues"].sum(), lam.sum(), rtol=1e-12)
    np.testing.assert_allclose(q["precision_eigenvalues"], 1.0 / q["covariance_eigenvalues"],
                               rtol=1e-12)
    lis = oracle.inverse_shrinkage(lam, c, "lis")
    gis = oracle.inverse_shrinkage(lam, c, "gis")
    x = 1.0 / lam
    a2 = q["theta"] ** 2 + q["htheta"] ** 2
    raw_qis = 1.0 / ((1 - c) ** 2 * x + 2 * c * (1 - c) * x * q["theta"] + c * c * x * a2)
    np.testing.assert_allclose(gis["covariance_eigenvalues"],
                               np.sqrt(raw_qis * lis["covariance_eigenvalues"]), rtol=1e-12)


def test_evaluate_many_matches_single_eta(oracle):
    """chebcode.rs:1370-1400: the two-eta traversal equals per-eta single
    calls within 5e-8 (1 + |re|) (a node accepted for both etas can differ
    from one eta's own traversal at acceptance boundaries), also for
    unsorted input."""
    p = 512
    ev = np.log(np.arange(1, p + 1, dtype=np.float64))
    shuffled = ev[np.random.default_rng(7).permutation(p)]
    etas = [0.02, 0.05, 0.11]
    for inp in (ev, shuffled):
        re, im = oracle.evaluate_many(inp, etas, 0.5, 11, 32)
        for k, eta in enumerate(etas):
            sr, si = oracle.compute_all(inp, eta, "chebcode")
            sr, si = sr * p, si * p
            assert np.all(np.abs(re[k] - sr) <= 5e-8 * (1.0 + np.abs(sr)))
            assert np.all(np.abs(im[k] - si) <= 5e-8)


# ---------------------------------------------------------- matrix front --
def _spiked_matrix(p):
    """pipeline/mod.rs:771-784 symmetric_spiked_matrix."""
    i = np.arange(p)
    a = 0.2 / (1.0 + np.abs(i[:, None] - i[None, :]).astype(float))
    np.fill_diagonal(a, 1.0)
    return a


def test_symmetric_eigh_cases(oracle):
    """pipeline/mod.rs:602-684: identity, diagonal, and a random symmetric
    matrix plus a strong rank-1 spike (trace kept to 1e-8, top eigenvalue
    > 15); the Jacobi eigensystem also matches LAPACK's."""
    ev, vec = oracle.symmetric_eigh(np.eye(4))
    np.testing.assert_allclose(ev, 1.0, atol=1e-10)
    np.testing.assert_allclose(vec.T @ vec, np.eye(4), atol=1e-10)
    ev, _ = oracle.symmetric_eigh(np.diag([5.0, 4.0, 3.0, 2.0, 1.0]))
    np.testing.assert_allclose(ev, [1, 2, 3, 4, 5], atol=1e-10)
    rng = np.random.default_rng(11)
    p = 20
    a = rng.uniform(-1, 1, (p, p))
    a = (a + a.T) / 2
    v = rng.uniform(-1, 1, p)
    v /= np.linalg.norm(v)
    a += 20.0 * np.outer(v, v)
    ev, vec = oracle.symmetric_eigh(a)
    assert ev[-1] > 15.0
    assert abs(ev.sum() - np.trace(a)) < 1e-8
    np.testing.assert_allclose(ev, np.linalg.eigvalsh(a), atol=1e-12)
    np.testing.assert_allclose(vec @ np.diag(ev) @ vec.T, a, atol=1e-12)


def test_angular_overlaps_known_answers(oracle):
    """eigenvector_overlaps/mod.rs:27-44."""
    a2 = oracle.angular_overlaps([5.0, 4.0, 3.0, 2.0], 1e-6, 0.5)
    np.testing.assert_allclose(a2, 1.0, atol=1e-3)
    a2 = oracle.angular_overlaps([5.0, 4.0, 3.0, 2.0, 0.5, 0.3], 0.5, 1.0)
    assert a2[0] > 0 and a2[1] > 0 and a2[4] == 0.0 and a2[5] == 0.0


def test_clean_eigensystem_trivial(oracle):
    """pipeline/mod.rs:625-641: identity eigenvectors give a diagonal result."""
    r = oracle.clean_eigensystem(np.eye(3), [3.0, 2.0, 1.0], 0.3)
    s = r["covariance"]
    assert np.all(np.diag(s) > 0)
    np.testing.assert_allclose(s - np.diag(np.diag(s)), 0.0, atol=1e-12)


def test_precision_identity_basis_and_positive(oracle):
    """pipeline/mod.rs:686-769."""
    ev = [2.0, 1.5, 1.0, 0.7, 0.5]
    r = oracle.precision_from_eigensystem(np.eye(5), ev, 0.2)
    np.testing.assert_allclose(np.diag(r["precision"]), r["precision_eigenvalues"], rtol=1e-12)
    off = r["precision"] - np.diag(np.diag(r["precision"]))
    np.testing.assert_allclose(off, 0.0, atol=1e-12)
    p = 8
    cov = np.diag(1.0 + 0.2 * np.arange(p))
    cov += np.diag(np.full(p - 1, 0.05), 1) + np.diag(np.full(p - 1, 0.05), -1)
    r = oracle.estimate_precision_matrix(cov, 0.3)
    om = r["precision"]
    np.testing.assert_allclose(om, om.T, atol=1e-12)
    assert np.all(r["precision_eigenvalues"] > 0)
    np.testing.assert_allclose(np.trace(om), r["precision_eigenvalues"].sum(), rtol=1e-10)
    v = r["eigenvectors"]
    np.testing.assert_allclose(om, v @ np.diag(r["precision_eigenvalues"]) @ v.T, atol=1e-10)


def test_clean_matrix_paths_and_renormalize(oracle):
    """pipeline/mod.rs:786-847: covariance and correlation paths agree (one
    estimator); renormalisation gives a unit diagonal, equals the explicit
    congruence and stays symmetric; a non-positive diagonal is left alone."""
    a = _spiked_matrix(9)
    x = oracle.clean_matrix(a, 0.35)
    y = oracle.clean_matrix(a, 0.35)
    np.testing.assert_array_equal(x["covariance"], y["covariance"])
    s = oracle.clean_matrix(_spiked_matrix(11), 0.4)["covariance"]
    rn = oracle.renormalize_to_unit_diagonal(s)
    np.testing.assert_allclose(np.diag(rn), 1.0, atol=1e-12)
    d = np.sqrt(np.diag(s))
    np.testing.assert_allclose(rn, s / np.outer(d, d), atol=1e-12)
    np.testing.assert_allclose(rn, rn.T, atol=1e-14)
    m = np.array([[0.0, 0.5], [0.5, 4.0]])
    np.testing.assert_array_equal(oracle.renormalize_to_unit_diagonal(m), m)
    r2 = oracle.clean_matrix(_spiked_matrix(11), 0.4, renormalize=True)
    np.testing.assert_array_equal(r2["covariance"], rn)


def test_clean_matrix_properties(oracle):
    """test_python_api.py:168-300 on the restatement: symmetric output,
    positive diagonal, trace preserved in covariance units."""
    rng = np.random.default_rng(42)
    corr = np.corrcoef(rng.standard_normal((400, 60)), rowvar=False)
    r = oracle.clean_matrix(corr, 60 / 400)
    np.testing.assert_allclose(r["covariance"], r["covariance"].T, atol=1e-12)
    assert np.all(np.diag(r["covariance"]) > 0) and r["sigma2"] >= 0
    rng = np.random.default_rng(3)
    cov = np.cov(rng.standard_normal((500, 40)), rowvar=False) * 3.0
    r = oracle.clean_matrix(cov, 40 / 499)
    assert np.isclose(r["eigenvalues"].sum(), np.trace(cov), rtol=1e-9)
