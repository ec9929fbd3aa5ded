"""torch.autograd over the transform and the hand-written adjoint.

Loss L = sum_j (w_j Re m_j + v_j Im m_j), m_j = (1/p) sum_i 1/(ev_i - z_j),
z_j = ev_j + i eta, w, v ~ N(0, 1): the gradient from backward() is checked
against FP64 central differences (h = 1e-6) of the GPU forward on 64 random
eigenvalues and against the oracle's FP64 direct-sum gradient.
"""
import math

import numpy as np
import pytest
import torch

from shrinkers_b200 import spectra
from shrinkers_b200.autograd import stieltjes_m

gpu = pytest.mark.gpu


def _loss(ev, eta, w, v, precision="f64"):
    m = stieltjes_m(ev, eta, precision)
    return (w * m.real + v * m.imag).sum()


def _setup(p):
    dev = torch.device("cuda", 0)
    ev = torch.from_numpy(spectra.config5(p)).to(dev)
    rng = np.random.default_rng(5)
    w = torch.from_numpy(rng.standard_normal(p)).to(dev)
    v = torch.from_numpy(rng.standard_normal(p)).to(dev)
    return ev, 1.0 / math.sqrt(p), w, v


@gpu
def test_gradient_matches_central_differences():
    p = 20000
    ev, eta, w, v = _setup(p)
    x = ev.clone().requires_grad_(True)
    _loss(x, eta, w, v).backward()
    g = x.grad.cpu().numpy()
    idx = np.random.default_rng(6).choice(p, 64, replace=False)
    h = 1e-6
    fd = np.empty(idx.size)
    with torch.no_grad():
        for n, k in enumerate(idx):
            xp = ev.clone()
            xp[k] += h
            xm = ev.clone()
            xm[k] -= h
            fd[n] = (_loss(xp, eta, w, v).item() - _loss(xm, eta, w, v).item()) / (2 * h)
    err = np.abs(g[idx] - fd) / (np.abs(fd) + 1e-6 * np.max(np.abs(fd)))
    assert np.max(err) < 1e-5, np.max(err)


@gpu
@pytest.mark.parametrize("precision,med_tol,max_tol", [("f64", 1e-13, 1e-11),
                                                       ("mixed", 1e-8, 1e-5)])
def test_gradient_matches_direct_sum(oracle, precision, med_tol, max_tol):
    p = 20000
    ev, eta, w, v = _setup(p)
    x = ev.clone().requires_grad_(True)
    _loss(x, eta, w, v, precision).backward()
    g = x.grad.cpu().numpy()
    ref = oracle.adjoint_direct(ev.cpu().numpy(), eta, w.cpu().numpy(), v.cpu().numpy())
    err = np.abs(g - ref) / (np.abs(ref) + 1e-3 * np.max(np.abs(ref)))
    assert np.median(err) < med_tol and np.max(err) < max_tol, (np.median(err), np.max(err))


@gpu
def test_forward_is_the_m_convention(oracle):
    p = 3000
    ev, eta, _, _ = _setup(p)
    m = stieltjes_m(ev, eta).cpu().numpy()
    o_re, o_im = oracle.compute_all(ev.cpu().numpy(), eta, "blocked")
    np.testing.assert_allclose(m.real, -o_re, rtol=1e-12, atol=1e-12)
    np.testing.assert_allclose(m.imag, o_im, rtol=1e-12, atol=1e-12)


@gpu
def test_gradient_flows_through_a_graph():
    """Composes with other torch ops (chain rule through the cotangent)."""
    p = 2048
    ev, eta, w, _ = _setup(p)
    x = ev.clone().requires_grad_(True)
    m = stieltjes_m(x, eta)
    (m.abs() ** 2 * w).sum().backward()
    assert torch.isfinite(x.grad).all()
    # same cotangent by hand: d|m|^2 = 2 Re(conj(m) dm) -> g = 2 w m
    g = (2 * w * m.detach())
    x2 = ev.clone().requires_grad_(True)
    m2 = stieltjes_m(x2, eta)
    (g.real * m2.real + g.imag * m2.imag).sum().backward()
    torch.testing.assert_close(x.grad, x2.grad, rtol=1e-12, atol=1e-12)


def test_cpu_tensor_is_rejected():
    with pytest.raises(ValueError, match="CUDA"):
        stieltjes_m(torch.ones(4, dtype=torch.float64))
    with pytest.raises(TypeError):
        stieltjes_m(np.ones(4))
