"""Multi-eta treecode evaluation (ChebCodeBatch::evaluate_many) on the GPU:
bit-exact with the oracle's restatement of the reference's two-lane
traversal, for every preset, odd and even eta counts and unsorted input."""
import ctypes as C
import math

import numpy as np
import pytest

import shrinkers_b200 as rk
from shrinkers_b200 import _native, spectra

pytestmark = pytest.mark.gpu
PRESETS = {"chebcode": (0.5, 11, 32), "chebcode_fast": (1.0, 8, 32),
           "chebcode_xtreme": (0.25, 11, 16), "chebcode_balanced": (0.55, 11, 32)}


@pytest.mark.parametrize("method", list(PRESETS))
@pytest.mark.parametrize("p", [1, 33, 5000, 100000])
def test_bit_exact_vs_oracle(oracle, method, p):
    ev = spectra.config3(p) if p > 33 else np.sort(np.random.default_rng(p).uniform(0.2, 3.0, p))
    etas = [0.5 / math.sqrt(p), 1.0 / math.sqrt(p), 3e-3, 0.07, 0.2]
    g = rk.chebcode_evaluate_many(ev, etas, method=method)
    o_re, o_im = oracle.evaluate_many(ev, etas, *PRESETS[method])
    np.testing.assert_array_equal(g["real"], o_re)
    np.testing.assert_array_equal(g["imag"], o_im)


def test_unsorted_input_and_even_count(oracle):
    p = 20000
    ev = spectra.config2(p)[np.random.default_rng(3).permutation(p)]
    etas = [1e-3, 1e-2]
    g = rk.chebcode_evaluate_many(ev, etas)
    o_re, o_im = oracle.evaluate_many(ev, etas, *PRESETS["chebcode"])
    np.testing.assert_array_equal(g["real"], o_re)
    np.testing.assert_array_equal(g["imag"], o_im)


def test_close_to_single_eta_transforms():
    """The reference's batch-vs-single criterion, on the GPU paths."""
    p = 512
    ev = spectra.log_spectrum(p)
    etas = [0.02, 0.05, 0.11]
    g = rk.chebcode_evaluate_many(ev, etas)
    for k, eta in enumerate(etas):
        s = rk.stieltjes_transform(ev, eta=eta, method="chebcode")
        sr, si = s["real"] * p, s["imag"] * p
        assert np.all(np.abs(g["real"][k] - sr) <= 5e-8 * (1.0 + np.abs(sr)))
        assert np.all(np.abs(g["imag"][k] - si) <= 5e-8)


def test_device_entry_matches_host_entry():
    import torch

    p = 4096
    ev = spectra.config3(p)
    etas = np.array([1e-3, 5e-3, 2e-2])
    host = rk.chebcode_evaluate_many(ev, etas)
    dev = torch.device("cuda", 0)
    e = torch.from_numpy(ev).to(dev)
    t = torch.from_numpy(etas).to(dev)
    re = torch.empty(3, p, dtype=torch.float64, device=dev)
    im = torch.empty_like(re)
    L = _native.load()
    _native.check(L.shrk_chebcode_evaluate_many_dev(e.data_ptr(), p, t.data_ptr(), 3, 13,
                                                    re.data_ptr(), im.data_ptr(),
                                                    torch.cuda.current_stream().cuda_stream))
    torch.cuda.synchronize()
    np.testing.assert_array_equal(re.cpu().numpy(), host["real"])
    np.testing.assert_array_equal(im.cpu().numpy(), host["imag"])
