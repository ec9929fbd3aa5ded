"""The matrix front-end on the GPU (shrk_clean_covariance_matrix and
friends) against the oracle's restatement of src/pipeline/mod.rs, and the
reference's Python tests of clean_correlation_matrix / clean_covariance_matrix
/ estimate_precision_matrix (test_python_api.py:165-470) restated.

The GPU eigensolver (the library's own: Householder tridiagonalisation,
multisection, inverse iteration) and the reference's Jacobi iteration agree
to rounding on the spectrum and, up to sign, on the eigenvectors; the
cleaned matrices are sign-invariant.  Bars: 1e-10 relative to the largest
entry for matrices built from different eigensolvers, 1e-12 when both sides
start from the same eigensystem.
"""
import numpy as np
import pytest

from shrinkers_b200 import spectra

pytestmark = pytest.mark.gpu


def close(a, b, tol):
    return np.max(np.abs(a - b)) <= tol * max(1.0, np.max(np.abs(b)))


def same_up_to_sign(u, v, tol=1e-8):
    """Columns of u and v span the same lines (non-degenerate spectrum)."""
    dots = np.abs(np.sum(u * v, axis=0))
    return np.all(np.abs(dots - 1.0) < tol)


def sample_corr(seed=42, n=400, p=60):
    x = np.random.default_rng(seed).standard_normal((n, p))
    return np.ascontiguousarray(np.corrcoef(x, rowvar=False))


def sample_cov(p, n, seed):
    """A random population a a^T/p + I/2, a demeaned sample of n rows, its
    covariance with 1/(n-1), c = p/(n-1), and the population eigenvalues."""
    rng = np.random.default_rng(seed)
    a = rng.standard_normal((p, p))
    pop = a @ a.T / p + 0.5 * np.eye(p)
    w, v = np.linalg.eigh(pop)
    y = rng.standard_normal((n, p)) @ (v * np.sqrt(w)).T
    y -= y.mean(axis=0)
    return np.ascontiguousarray(y.T @ y / (n - 1)), p / (n - 1), w


def test_clean_correlation_matches_oracle(rk, oracle):
    corr = sample_corr()
    c = 60 / 400
    got = rk.clean_correlation_matrix(corr, c=c)
    ref = oracle.clean_matrix(corr, c)
    assert close(got["covariance"], ref["covariance"], 1e-10)
    np.testing.assert_allclose(got["eigenvalues"], ref["eigenvalues"], rtol=1e-10)
    np.testing.assert_allclose(got["overlaps"], ref["overlaps"], atol=1e-10)
    assert abs(got["sigma2"] - ref["sigma2"]) <= 1e-12 * ref["sigma2"]
    assert same_up_to_sign(got["eigenvectors"], ref["eigenvectors"])


def test_same_eigensystem_matches_oracle_tightly(rk, oracle):
    """clean_eigensystem / precision_from_eigensystem fed the same (shuffled)
    eigensystem on both sides."""
    cov, c, _ = sample_cov(80, 400, 21)
    w, v = np.linalg.eigh(cov)
    perm = np.random.default_rng(0).permutation(w.size)
    w, v = np.ascontiguousarray(w[perm]), np.ascontiguousarray(v[:, perm])
    got = rk.clean_eigensystem(v, w, c)
    ref = oracle.clean_eigensystem(v, w, c)
    assert close(got["covariance"], ref["covariance"], 1e-12)
    np.testing.assert_array_equal(got["eigenvectors"], ref["eigenvectors"])
    np.testing.assert_allclose(got["eigenvalues"], ref["eigenvalues"], rtol=1e-12)
    np.testing.assert_array_equal(got["overlaps"] > 0, ref["overlaps"] > 0)
    for method in ("qis", "lis", "gis"):
        g = rk.precision_from_eigensystem(v, w, c, method=method)
        r = oracle.precision_from_eigensystem(v, w, c, method=method)
        assert close(g["precision"], r["precision"], 1e-12)
        np.testing.assert_allclose(g["precision_eigenvalues"], r["precision_eigenvalues"],
                                   rtol=1e-10)
        assert g["smoothing"] == r["smoothing"]


@pytest.mark.parametrize("p", [100, 300])
def test_few_spikes_reference_order_kernel(rk, oracle, p):
    """A bulk in [0.5, 1.5] plus spikes 10, 20, 30 in a random basis: 3-4
    active directions, summed by the kernel in the reference's order."""
    ev = np.concatenate([np.sort(0.5 + np.random.default_rng(1).uniform(0, 1, p - 3)),
                         [10.0, 20.0, 30.0]])
    q, _ = np.linalg.qr(np.random.default_rng(2).standard_normal((p, p)))
    q = np.ascontiguousarray(q)
    got = rk.clean_eigensystem(q, ev, 0.1)
    ref = oracle.clean_eigensystem(q, ev, 0.1)
    assert 0 < np.sum(ref["overlaps"] > 0) <= 16
    assert close(got["covariance"], ref["covariance"], 1e-12)
    np.testing.assert_allclose(got["overlaps"], ref["overlaps"], rtol=1e-10)


def test_large_spiked_matrix(rk, oracle):
    """p = 1500 with three factors: GPU end to end vs the oracle's cleaning of
    LAPACK's eigensystem of the same matrix."""
    rng = np.random.default_rng(7)
    p, n = 1500, 6000
    b = rng.standard_normal((p, 3)) * np.array([6.0, 4.0, 3.0])
    x = rng.standard_normal((n, 3)) @ b.T + rng.standard_normal((n, p))
    cov = np.ascontiguousarray(np.cov(x, rowvar=False))
    c = p / n
    got = rk.clean_covariance_matrix(cov, c=c)
    w, v = np.linalg.eigh(cov)
    ref = oracle.clean_eigensystem(v, w, c)
    assert close(got["covariance"], ref["covariance"], 1e-9)
    np.testing.assert_allclose(got["eigenvalues"], ref["eigenvalues"], rtol=1e-9)
    # the trace rescale lifts the whole cleaned bulk above sigma^2 (1 + sqrt(c)):
    # every direction is active and the rank-k update is the DGEMM path
    assert np.sum(got["overlaps"] > 0) == np.sum(ref["overlaps"] > 0) > 16
    ev, _ = rk.symmetric_eigh(cov)
    np.testing.assert_allclose(ev, w, rtol=1e-10, atol=1e-12 * w[-1])


# --- test_python_api.py:165-300, restated ---------------------------------
def test_shapes_symmetry_positive_diagonal(rk):
    corr = sample_corr()
    res = rk.clean_correlation_matrix(corr, c=60 / 400)
    cov = res["covariance"]
    assert cov.shape == (60, 60)
    assert np.allclose(cov, cov.T, atol=1e-12)
    assert res["eigenvalues"].shape == (60,) and res["overlaps"].shape == (60,)
    assert res["sigma2"] >= 0.0
    assert np.all(np.diag(cov) > 0)


def test_validation_messages(rk):
    with pytest.raises(ValueError, match="square"):
        rk.clean_correlation_matrix(np.ones((3, 4)), c=0.5)
    bad = sample_corr()
    bad[0, 1] = np.inf
    with pytest.raises(ValueError, match="finite"):
        rk.clean_correlation_matrix(bad, c=0.15)
    with pytest.raises(ValueError, match="square"):
        rk.clean_covariance_matrix(np.ones((3, 4)), c=0.5)
    bad = np.eye(3)
    bad[0, 1] = np.nan
    with pytest.raises(ValueError, match="finite"):
        rk.clean_covariance_matrix(bad, c=0.5)
    with pytest.raises(ValueError, match="symmetric"):
        rk.clean_correlation_matrix(np.array([[1.0, 0.5], [0.1, 1.0]]), c=0.25)
    sym = np.array([[1.0, 0.5], [0.5, 1.0]])
    assert rk.clean_correlation_matrix(sym, c=0.25)["covariance"].shape == (2, 2)
    cov = np.eye(5)
    cov[0, 1] = 0.3
    with pytest.raises(ValueError, match="symmetric"):
        rk.estimate_precision_matrix(cov, c=0.3)


def test_renormalize(rk):
    """A factor model: the raw reconstruction's diagonal drifts from one, the
    renormalised one is exactly the D^-1/2 S D^-1/2 congruence, only the
    matrix changes, and it moves closer to the population correlation."""
    rng = np.random.default_rng(0)
    p, n, k = 40, 300, 3
    b = rng.standard_normal((p, k)) * np.sqrt([3.0, 2.0, 1.5])
    s = b @ b.T + np.diag(0.5 + rng.uniform(0.0, 0.5, size=p))
    d0 = np.sqrt(np.diag(s))
    pop = s / np.outer(d0, d0)
    x = rng.standard_normal((n, p)) @ np.linalg.cholesky(pop).T
    corr = np.ascontiguousarray(np.corrcoef(x, rowvar=False))
    c = p / n
    raw = rk.clean_correlation_matrix(corr, c=c)
    ren = rk.clean_correlation_matrix(corr, c=c, renormalize=True)
    assert np.abs(np.diag(raw["covariance"]) - 1.0).max() > 1e-3
    np.testing.assert_allclose(np.diag(ren["covariance"]), 1.0, atol=1e-12)
    d = np.sqrt(np.diag(raw["covariance"]))
    np.testing.assert_allclose(ren["covariance"], raw["covariance"] / np.outer(d, d), atol=1e-12)
    np.testing.assert_array_equal(ren["eigenvalues"], raw["eigenvalues"])
    np.testing.assert_array_equal(ren["overlaps"], raw["overlaps"])
    assert ren["sigma2"] == raw["sigma2"]
    assert np.linalg.norm(ren["covariance"] - pop) < np.linalg.norm(raw["covariance"] - pop)
    implicit = rk.clean_correlation_matrix(corr, c=c)["covariance"]
    np.testing.assert_array_equal(implicit, raw["covariance"])
    m = np.array([[0.0, 0.5], [0.5, 4.0]])
    np.testing.assert_array_equal(rk.renormalize_to_unit_diagonal(m), m)


def test_covariance_path_and_units(rk):
    rng = np.random.default_rng(11)
    m = np.ascontiguousarray(np.cov(rng.standard_normal((400, 30)), rowvar=False))
    a = rk.clean_covariance_matrix(m, c=30 / 399)
    b = rk.clean_correlation_matrix(m, c=30 / 399)
    np.testing.assert_allclose(a["covariance"], b["covariance"], atol=1e-12)
    np.testing.assert_allclose(a["eigenvalues"], b["eigenvalues"], atol=1e-12)
    np.testing.assert_allclose(a["overlaps"], b["overlaps"], atol=1e-12)
    assert set(a) == {"covariance", "eigenvectors", "eigenvalues", "overlaps", "sigma2"}
    rng = np.random.default_rng(3)
    cov = np.ascontiguousarray(np.cov(rng.standard_normal((500, 40)), rowvar=False) * 3.0)
    res = rk.clean_covariance_matrix(cov, c=40 / 499)
    assert np.isclose(res["eigenvalues"].sum(), np.trace(cov), rtol=1e-9)
    assert not np.allclose(np.diag(res["covariance"]), 1.0, atol=1e-6)


# --- test_python_api.py:412-464, restated ---------------------------------
def test_precision_matrix(rk, oracle):
    sample, c, _ = sample_cov(12, 60, 11)
    res = rk.estimate_precision_matrix(sample, c=c)
    assert set(res) == {"precision", "eigenvectors", "precision_eigenvalues",
                        "covariance_eigenvalues", "smoothing"}
    om = res["precision"]
    np.testing.assert_allclose(om, om.T, atol=1e-10)
    np.testing.assert_allclose(np.trace(om), res["precision_eigenvalues"].sum(), rtol=1e-10)
    sample, c, _ = sample_cov(10, 50, 12)
    res = rk.estimate_precision_matrix(sample, c=c)
    np.testing.assert_allclose(np.sort(np.linalg.eigvalsh(res["precision"])),
                               np.sort(res["precision_eigenvalues"]), rtol=1e-8)
    sample, c, _ = sample_cov(14, 70, 13)
    mat = rk.estimate_precision_matrix(sample, c=c)
    spec = rk.inverse_nonlinear_shrinkage(np.ascontiguousarray(np.linalg.eigvalsh(sample)), c=c)
    for key in ("precision_eigenvalues", "covariance_eigenvalues"):
        np.testing.assert_allclose(np.sort(mat[key]), np.sort(spec[key]), rtol=1e-9)
    ref = oracle.estimate_precision_matrix(sample, c)
    assert close(mat["precision"], ref["precision"], 1e-10)
    for method in ("lis", "gis"):
        g = rk.estimate_precision_matrix(sample, c=c, method=method)
        r = oracle.estimate_precision_matrix(sample, c, method=method)
        assert close(g["precision"], r["precision"], 1e-10)


def test_small_and_trivial(rk, oracle):
    """pipeline/mod.rs:602-641, 686-716 on the GPU path: identity and
    diagonal matrices, identity eigenbases."""
    ev, vec = rk.symmetric_eigh(np.eye(4))
    np.testing.assert_allclose(ev, 1.0, atol=1e-12)
    np.testing.assert_allclose(vec.T @ vec, np.eye(4), atol=1e-12)
    ev, _ = rk.symmetric_eigh(np.diag([5.0, 4.0, 3.0, 2.0, 1.0]))
    np.testing.assert_allclose(ev, [1, 2, 3, 4, 5], atol=1e-12)
    r = rk.clean_eigensystem(np.eye(3), np.array([3.0, 2.0, 1.0]), 0.3)
    s = r["covariance"]
    assert np.all(np.diag(s) > 0)
    np.testing.assert_allclose(s - np.diag(np.diag(s)), 0.0, atol=1e-12)
    r = rk.precision_from_eigensystem(np.eye(5), np.array([2.0, 1.5, 1.0, 0.7, 0.5]), 0.2)
    np.testing.assert_allclose(np.diag(r["precision"]), r["precision_eigenvalues"], rtol=1e-12)
    one = rk.clean_covariance_matrix(np.array([[2.0]]), c=0.5)
    ref = oracle.clean_matrix(np.array([[2.0]]), 0.5)
    np.testing.assert_allclose(one["covariance"], ref["covariance"], rtol=1e-12)


def test_device_forms_match_host_forms(rk):
    """shrk_*_dev: the matrix produced on the caller's stream just before
    the call (the call must wait for it), outputs on the device; the same
    values as the host forms, bit for bit."""
    import ctypes as C

    import torch
    from shrinkers_b200 import _native

    L = _native.load()
    cov, c, _ = sample_cov(300, 1200, 21)
    p = cov.shape[0]
    host = rk.clean_covariance_matrix(cov, c=c)
    prec_host = rk.estimate_precision_matrix(cov, c=c)
    ev_host, vec_host = rk.symmetric_eigh(cov)
    d = torch.device("cuda", 0)
    st = torch.cuda.Stream(device=d)
    with torch.cuda.stream(st):
        src = torch.from_numpy(cov).to(d)
        m = (src * 2.0) * 0.5  # queued on st right before the call
        out = torch.empty(p, p, dtype=torch.float64, device=d)
        vec = torch.empty_like(out)
        rie = torch.empty(p, dtype=torch.float64, device=d)
        ov = torch.empty_like(rie)
        s2 = C.c_double()
        _native.check(L.shrk_clean_covariance_matrix_dev(
            m.data_ptr(), p, c, 0, out.data_ptr(), vec.data_ptr(), rie.data_ptr(), ov.data_ptr(),
            C.byref(s2), st.cuda_stream), "clean_covariance_matrix_dev")
        res = {k: v.cpu().numpy() for k, v in
               (("covariance", out), ("eigenvectors", vec), ("eigenvalues", rie),
                ("overlaps", ov))}
        pe = torch.empty(p, dtype=torch.float64, device=d)
        ce = torch.empty_like(pe)
        om = torch.empty(p, p, dtype=torch.float64, device=d)
        h = C.c_double()
        _native.check(L.shrk_estimate_precision_matrix_dev(
            m.data_ptr(), p, c, 0, om.data_ptr(), vec.data_ptr(), pe.data_ptr(), ce.data_ptr(),
            C.byref(h), st.cuda_stream), "estimate_precision_matrix_dev")
        prec = {"precision": om.cpu().numpy(), "eigenvectors": vec.cpu().numpy(),
                "precision_eigenvalues": pe.cpu().numpy(),
                "covariance_eigenvalues": ce.cpu().numpy()}
        w = torch.empty(p, dtype=torch.float64, device=d)
        _native.check(L.shrk_symmetric_eigh_dev(m.data_ptr(), p, w.data_ptr(), vec.data_ptr(),
                                                st.cuda_stream), "symmetric_eigh_dev")
        ev_dev, vec_dev = w.cpu().numpy(), vec.cpu().numpy()
    for k in ("covariance", "eigenvectors", "eigenvalues", "overlaps"):
        np.testing.assert_array_equal(res[k], host[k])
    assert s2.value == host["sigma2"]
    for k in ("precision", "eigenvectors", "precision_eigenvalues", "covariance_eigenvalues"):
        np.testing.assert_array_equal(prec[k], prec_host[k])
    assert h.value == prec_host["smoothing"]
    np.testing.assert_array_equal(ev_dev, ev_host)
    np.testing.assert_array_equal(vec_dev, vec_host)
    # argument checks before any device work
    assert L.shrk_clean_covariance_matrix_dev(None, p, c, 0, out.data_ptr(), None, None, None,
                                              None, None) == _native.SHRK_EINVAL
    assert L.shrk_symmetric_eigh_dev(m.data_ptr(), p, None, None, None) == _native.SHRK_EINVAL


@pytest.mark.parametrize("ta,tb", [(0, 0), (0, 1), (1, 0), (1, 1)])
@pytest.mark.parametrize("m,n,k", [(1, 1, 1), (64, 2048, 1000), (1000, 700, 64), (300, 257, 2049),
                                   (129, 130, 131)])
def test_dgemm_matches_torch(ta, tb, m, n, k):
    """The library's FP64 GEMM (the eigensolver's back-transform and the
    reconstructions) against torch's FP64 matmul: every tile shape, split-K
    and edge case; beta = 0 and 1."""
    import torch
    from shrinkers_b200 import _native

    L = _native.load()
    d = torch.device("cuda", 0)
    g = torch.Generator(device="cpu").manual_seed(m * 7 + n * 3 + k + 11 * ta + 5 * tb)
    a = torch.randn((k, m) if ta else (m, k), generator=g, dtype=torch.float64)
    b = torch.randn((n, k) if tb else (k, n), generator=g, dtype=torch.float64)
    c0 = torch.randn((m, n), generator=g, dtype=torch.float64)
    # column-major storage: pass the transposes' contiguous buffers
    A = a.t().contiguous().to(d)  # column-major a, ld = rows of a
    B = b.t().contiguous().to(d)
    for beta in (0.0, 1.0):
        C = c0.t().contiguous().to(d)
        _native.check(L.shrk_diag_dgemm(ta, tb, m, n, k, 0.75, A.data_ptr(), a.shape[0],
                                        B.data_ptr(), b.shape[0], beta, C.data_ptr(), m,
                                        torch.cuda.current_stream().cuda_stream), "dgemm")
        ref = 0.75 * ((a.t() if ta else a) @ (b.t() if tb else b)) + beta * c0
        got = C.cpu().t()
        err = (got - ref).abs().max().item()
        assert err <= 1e-12 * max(1.0, k ** 0.5) * max(1.0, ref.abs().max().item()), (beta, err)


def _hard_matrices():
    """Spectra that stress the eigensolver: sample covariances (one above
    the size where the multisection narrows to 8 probes), the identity,
    repeated and clustered eigenvalues, a rank-one update of the identity,
    a wide dynamic range, and the Wilkinson tridiagonal (pairs of eigenvalues
    equal to many digits)."""
    rng = np.random.default_rng(2024)
    out = []
    for p, n in ((700, 2800), (3100, 12400)):
        x = rng.standard_normal((n, p))
        out.append((f"sample_cov_{p}", np.ascontiguousarray(x.T @ x / n)))
    out.append(("identity_300", np.eye(300)))

    def with_spectrum(name, w, seed):
        q, _ = np.linalg.qr(np.random.default_rng(seed).standard_normal((w.size, w.size)))
        a = (q * w) @ q.T
        return (name, np.ascontiguousarray((a + a.T) / 2))

    out.append(with_spectrum("repeated_400", np.repeat([1.0, 2.0, 5.0, 9.0], 100), 1))
    w = np.concatenate([1.0 + 1e-13 * np.arange(40), np.linspace(2.0, 3.0, 216)])
    out.append(with_spectrum("cluster_1e-13_256", w, 2))
    v = rng.standard_normal(512)
    out.append(("rank_one_512", np.ascontiguousarray(np.eye(512) + 50.0 * np.outer(v, v) / 512)))
    out.append(with_spectrum("range_1e-8_1e4_300", np.geomspace(1e-8, 1e4, 300), 3))
    m = 150
    wil = np.diag(np.abs(np.arange(-m, m + 1)).astype(float)) + np.diag(np.ones(2 * m), 1) \
        + np.diag(np.ones(2 * m), -1)
    out.append(("wilkinson_301", np.ascontiguousarray(wil)))
    return out


@pytest.mark.parametrize("name,a", _hard_matrices(), ids=lambda v: v if isinstance(v, str) else "")
def test_symmetric_eigh_hard_spectra(rk, name, a):
    """The library's eigensolver against LAPACK (numpy): eigenvalues to
    1e-13 of the largest, residual ||A V - V diag(w)|| and orthogonality
    ||V^T V - I|| to 1e-12 (relative to the largest entry of A)."""
    w, v = rk.symmetric_eigh(a)
    w_ref = np.linalg.eigvalsh(a)
    scale = max(np.max(np.abs(w_ref)), 1e-300)
    assert np.max(np.abs(w - w_ref)) <= 1e-13 * scale, name
    amax = np.max(np.abs(a))
    assert np.max(np.abs(a @ v - v * w)) <= 1e-12 * amax, name
    assert np.max(np.abs(v.T @ v - np.eye(a.shape[0]))) <= 1e-12, name


@pytest.mark.parametrize("form", ["shared", "global", "two_barrier"])
def test_symmetric_eigh_tridiagonalisation_forms(rk, monkeypatch, form):
    """The three forms of the tridiagonalisation (per-CTA vectors in shared
    memory, the same in global memory as used above ~8 500 rows, and the
    two-barrier form) give the same decomposition to rounding."""
    if form == "global":
        monkeypatch.setenv("SHRK_EIGH_TRI1_GLOBAL", "1")
    elif form == "two_barrier":
        monkeypatch.setenv("SHRK_EIGH_TRIDIAG", "2")
    rng = np.random.default_rng(31)
    x = rng.standard_normal((2000, 500))
    a = np.ascontiguousarray(x.T @ x / 2000)
    w, v = rk.symmetric_eigh(a)
    w_ref = np.linalg.eigvalsh(a)
    assert np.max(np.abs(w - w_ref)) <= 1e-13 * np.max(np.abs(w_ref))
    assert np.max(np.abs(a @ v - v * w)) <= 1e-12 * np.max(np.abs(a))
    assert np.max(np.abs(v.T @ v - np.eye(500))) <= 1e-12
