"""Treecode adjoint (shrk_stieltjes_adjoint_treecode) against the oracle's
FP64 direct-sum gradient.

The gradient has no counterpart in the reference, so there is nothing to be
bit-exact with: each ChebCode preset has an accuracy class (normwise
relative L2 error of the gradient, measured on this workload and set here
with a margin of about 4x).  The gradient is a sum of terms of both signs,
so its relative error is larger than the forward transform's for the same
tree.
"""
import ctypes as C
import math

import numpy as np
import pytest

import shrinkers_b200 as rk
from shrinkers_b200 import _native, spectra

pytestmark = pytest.mark.gpu
_D = C.POINTER(C.c_double)
IDS = {"chebcode": 13, "chebcode_fast": 14, "chebcode_xtreme": 15, "chebcode_balanced": 16}

# (p, preset) -> relative L2 bar; measured: p=2e4: 3.4e-8, 3.8e-4, 1.2e-10,
# 2.0e-7; p=2e5: 1.1e-6, 6.3e-3, 7.7e-10, 1.1e-6.
BARS = {
    20000: {"chebcode": 2e-7, "chebcode_fast": 2e-3, "chebcode_xtreme": 1e-9,
            "chebcode_balanced": 1e-6},
    200000: {"chebcode": 5e-6, "chebcode_fast": 3e-2, "chebcode_xtreme": 5e-9,
             "chebcode_balanced": 5e-6},
}


def _grad(ev, w, v, eta, method):
    L = _native.load()
    g = np.empty(ev.size)
    _native.check(L.shrk_stieltjes_adjoint_treecode(ev.ctypes.data_as(_D), ev.size, eta,
                                                    w.ctypes.data_as(_D), v.ctypes.data_as(_D),
                                                    IDS[method], g.ctypes.data_as(_D)))
    return g


def _case(p):
    ev = spectra.config5(p)
    rng = np.random.default_rng(5)
    return ev, rng.standard_normal(p), rng.standard_normal(p), 1.0 / math.sqrt(p)


@pytest.mark.parametrize("p", [20000, 200000])
@pytest.mark.parametrize("method", list(IDS))
def test_treecode_adjoint_accuracy_class(oracle, p, method):
    ev, w, v, eta = _case(p)
    idx = None if p <= 20000 else np.sort(np.random.default_rng(1).choice(p, 2000, replace=False))
    ref = oracle.adjoint_direct(ev, eta, w, v, idx)
    g = _grad(ev, w, v, eta, method)
    if idx is not None:
        g = g[idx]
    assert np.all(np.isfinite(g))
    rel = np.linalg.norm(g - ref) / np.linalg.norm(ref)
    assert rel <= BARS[p][method], rel


@pytest.mark.parametrize("p", [1, 2, 33, 257])
def test_small_sizes(oracle, p):
    """One leaf (p <= 32), two leaves (33) and a few levels (257): the sums
    are exact or nearly so."""
    ev = np.sort(np.random.default_rng(p).uniform(0.5, 2.5, p))
    rng = np.random.default_rng(7)
    w, v = rng.standard_normal(p), rng.standard_normal(p)
    eta = 1.0 / math.sqrt(p)
    ref = oracle.adjoint_direct(ev, eta, w, v)
    g = _grad(ev, w, v, eta, "chebcode_xtreme" if p > 33 else "chebcode")
    assert np.max(np.abs(g - ref)) <= 1e-9 * (np.max(np.abs(ref)) + 1e-300)


def test_unsorted_input_gives_the_permuted_gradient():
    ev, w, v, eta = _case(50000)
    perm = np.random.default_rng(2).permutation(ev.size)
    g = _grad(ev, w, v, eta, "chebcode")
    gp = _grad(np.ascontiguousarray(ev[perm]), np.ascontiguousarray(w[perm]),
               np.ascontiguousarray(v[perm]), eta, "chebcode")
    np.testing.assert_array_equal(gp, g[perm])


def test_python_api_and_autograd_with_a_preset(oracle):
    import torch
    from shrinkers_b200.autograd import stieltjes_m

    ev, w, v, eta = _case(20000)
    ref = oracle.adjoint_direct(ev, eta, w, v)
    g = rk.stieltjes_adjoint(ev, w, v, eta=eta, method="chebcode_xtreme")
    assert np.linalg.norm(g - ref) / np.linalg.norm(ref) <= 1e-9
    dev = torch.device("cuda", 0)
    x = torch.from_numpy(ev).to(dev).requires_grad_(True)
    m = stieltjes_m(x, eta, method="chebcode_xtreme")
    wt, vt = torch.from_numpy(w).to(dev), torch.from_numpy(v).to(dev)
    (wt * m.real + vt * m.imag).sum().backward()
    np.testing.assert_array_equal(x.grad.cpu().numpy(), g)
    # the forward is the preset's transform
    f = rk.stieltjes_transform(ev, eta=eta, method="chebcode_xtreme")
    np.testing.assert_array_equal(m.detach().real.cpu().numpy(), -f["real"])
    np.testing.assert_array_equal(m.detach().imag.cpu().numpy(), f["imag"])
