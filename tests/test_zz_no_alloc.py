"""shrk_stieltjes_at_points_noalloc: the allocation-free exact entry point.

Checked against shrk_stieltjes_at_points_dev (exact method, same precision)
on two calls in a row whose sizes differ, in both orders, so that a call
reading the previous call's leftovers in the shared static scratch would
show.  One of the two sizes forces fewer source splits than the allocating
path uses (the static scratch caps the split count), so the two paths sum
the splits in a different order: the bar is the FP64 bar of the exact tests
(1e-12 relative per point, floor scale max(|re|, |im|, 1e-12)).

This file is collected last on purpose: it must pass both in a fresh
process and after every other GPU test has used the library.
"""
import ctypes as C

import numpy as np
import pytest
import torch

from shrinkers_b200 import _native, spectra

pytestmark = pytest.mark.gpu

F64, MIXED = 0, 1
EINVAL = 1
MAX_POINTS = 262144
MAX_EIGS = 16777216
BAR = 1e-12


def _dev():
    return torch.device("cuda", 0)


def _case(p, nq, seed):
    """MP(c=0.5) spectrum of size p, nq query points: a third at eigenvalues,
    the rest spread over and beyond the support (shuffled)."""
    rng = np.random.default_rng(seed)
    ev = spectra.mp_spectrum(p, 0.5, seed=seed)
    k = nq // 3
    q = np.concatenate([rng.choice(ev, size=k, replace=False),
                        rng.uniform(ev.min() - 0.5, ev.max() + 0.5, size=nq - k)])
    rng.shuffle(q)
    d = _dev()
    return (torch.from_numpy(ev).to(d), torch.from_numpy(q).to(d), 1.0 / np.sqrt(p))


def _out(nq):
    d = _dev()
    return (torch.empty(nq, dtype=torch.float64, device=d),
            torch.empty(nq, dtype=torch.float64, device=d))


def _noalloc(L, q, ev, eta, precision, re, im, stream):
    st = L.shrk_stieltjes_at_points_noalloc(q.data_ptr(), q.numel(), ev.data_ptr(), ev.numel(),
                                            eta, precision, re.data_ptr(), im.data_ptr(), stream)
    _native.check(st, "stieltjes_at_points_noalloc")


def _allocating(L, q, ev, eta, precision, stream):
    m = C.c_int()
    assert L.shrk_parse_method(b"blocked", C.byref(m)) == 0
    re, im = _out(q.numel())
    st = L.shrk_stieltjes_at_points_dev(q.data_ptr(), q.numel(), ev.data_ptr(), ev.numel(), eta,
                                        m.value, precision, float("nan"), 0, re.data_ptr(),
                                        im.data_ptr(), stream)
    _native.check(st, "stieltjes_at_points_dev")
    return re, im


def _rel(re, im, ref_re, ref_im):
    re, im, ref_re, ref_im = (t.cpu().numpy() for t in (re, im, ref_re, ref_im))
    assert np.all(np.isfinite(re)) and np.all(np.isfinite(im))
    scale = np.maximum(np.maximum(np.abs(ref_re), np.abs(ref_im)), 1e-12)
    return float(np.max((np.abs(re - ref_re) + np.abs(im - ref_im)) / scale))


# (p, nq): the first forces a split count capped by the static scratch
# (200000 points leave room for 2 splits), the second is uncapped.
BIG, SMALL = (300_000, 200_000), (50_000, 3_000)


@pytest.mark.parametrize("precision", [F64, MIXED], ids=["f64", "mixed"])
@pytest.mark.parametrize("order", [(BIG, SMALL), (SMALL, BIG)], ids=["big_then_small",
                                                                   "small_then_big"])
def test_two_calls_in_a_row_match_allocating_path(precision, order):
    L = _native.load()
    stream = torch.cuda.current_stream().cuda_stream
    cases = [_case(p, nq, seed=11 + i) for i, (p, nq) in enumerate(order)]
    outs = [_out(q.numel()) for (_, q, _) in cases]
    # Two back-to-back calls on one stream, no synchronisation in between.
    for (ev, q, eta), (re, im) in zip(cases, outs):
        _noalloc(L, q, ev, eta, precision, re, im, stream)
    torch.cuda.synchronize()
    for (ev, q, eta), (re, im) in zip(cases, outs):
        ref_re, ref_im = _allocating(L, q, ev, eta, precision, stream)
        torch.cuda.synchronize()
        assert _rel(re, im, ref_re, ref_im) <= BAR


def test_repeated_calls_reserve_no_device_memory():
    L = _native.load()
    stream = torch.cuda.current_stream().cuda_stream
    ev, q, eta = _case(*BIG, seed=5)
    re, im = _out(q.numel())
    _noalloc(L, q, ev, eta, MIXED, re, im, stream)  # first call: one-time setup
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for prec in (F64, MIXED, F64):
        _noalloc(L, q, ev, eta, prec, re, im, stream)
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    # The allocating path would reserve >= 2 splits x 200000 points x 16 B
    # (6.4 MB) of partials here, plus bounds; allow only page-level noise.
    assert free0 - free1 < (2 << 20)


def test_sizes_beyond_the_static_scratch_are_rejected():
    L = _native.load()
    ev, q, eta = _case(1024, 16, seed=3)
    re, im = _out(16)
    st = L.shrk_stieltjes_at_points_noalloc(q.data_ptr(), MAX_POINTS + 1, ev.data_ptr(),
                                            ev.numel(), eta, F64, re.data_ptr(), im.data_ptr(),
                                            None)
    assert st == EINVAL
    assert str(MAX_POINTS) in _native.last_error()
    st = L.shrk_stieltjes_at_points_noalloc(q.data_ptr(), q.numel(), ev.data_ptr(), MAX_EIGS + 1,
                                            eta, MIXED, re.data_ptr(), im.data_ptr(), None)
    assert st == EINVAL
    assert str(MAX_EIGS) in _native.last_error()
