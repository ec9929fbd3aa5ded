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


def _memory_probe_cases():
    """(p, nq) cases whose allocating-path temporaries would be large: the
    BIG case and the largest spectrum the static array admits."""
    return [BIG, (MAX_EIGS, 4096)]


def test_repeated_calls_reserve_no_device_memory():
    """The one-time setup runs on a tiny case; then calls far larger than it
    (and than anything the allocating path's slots may hold from earlier
    tests) must not change the device's free memory.  A path that drew its
    temporaries from a growable slot would grow it here."""
    L = _native.load()
    stream = torch.cuda.current_stream().cuda_stream
    ev0, q0, eta0 = _case(1024, 16, seed=4)
    re0, im0 = _out(16)
    _noalloc(L, q0, ev0, eta0, F64, re0, im0, stream)  # one-time setup, tiny
    cases = []
    for i, (p, nq) in enumerate(_memory_probe_cases()):
        ev, q, eta = _case(p, nq, seed=6 + i)
        cases.append((ev, q, eta) + _out(nq))
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for ev, q, eta, re, im in cases:
        for prec in (F64, MIXED):
            _noalloc(L, q, ev, eta, prec, re, im, stream)
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    # The allocating path would reserve >= 2 splits x 200000 points x 16 B
    # (6.4 MB) of partials for BIG and 1 MB of bounds for the largest
    # spectrum; allow only page-level noise.
    assert free0 - free1 < (2 << 20)
    for _, _, _, re, im in cases:
        assert torch.isfinite(re).all() and torch.isfinite(im).all()


_FRESH = r"""
import sys, torch
sys.path.insert(0, sys.argv[1])
from shrinkers_b200 import _native
L = _native.load()
d = torch.device("cuda", 0)
s = torch.cuda.current_stream().cuda_stream
def call(p, nq, prec):
    ev = torch.linspace(0.1, 3.0, p, dtype=torch.float64, device=d)
    q = torch.linspace(0.0, 3.1, nq, dtype=torch.float64, device=d)
    re, im = torch.empty_like(q), torch.empty_like(q)
    _native.check(L.shrk_stieltjes_at_points_noalloc(q.data_ptr(), nq, ev.data_ptr(), p,
                  1e-3, prec, re.data_ptr(), im.data_ptr(), s))
    return ev, q, re, im
call(1024, 16, 0)
keep = [call(300000, 200000, 1)]
torch.cuda.synchronize()
del keep
torch.cuda.empty_cache()
ins = [torch.linspace(0.1, 3.0, 300000, dtype=torch.float64, device=d),
       torch.linspace(0.0, 3.1, 200000, dtype=torch.float64, device=d)]
outs = [torch.empty(200000, dtype=torch.float64, device=d) for _ in range(2)]
torch.cuda.synchronize()
f0, _ = torch.cuda.mem_get_info()
for prec in (0, 1, 0):
    _native.check(L.shrk_stieltjes_at_points_noalloc(ins[1].data_ptr(), 200000, ins[0].data_ptr(),
                  300000, 1e-3, prec, outs[0].data_ptr(), outs[1].data_ptr(), s))
torch.cuda.synchronize()
f1, _ = torch.cuda.mem_get_info()
print(f0 - f1)
"""


def test_no_device_memory_in_a_fresh_process():
    """The same check in a process where no other entry point has run (so
    no library slot exists at all)."""
    import os
    import subprocess
    import sys

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    out = subprocess.run([sys.executable, "-c", _FRESH, root], capture_output=True, text=True,
                         timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    assert int(out.stdout.strip().splitlines()[-1]) < (2 << 20)


def test_mixed_and_f64_against_the_oracle(oracle):
    """The allocation-free call against the oracle, not only against the
    allocating GPU path: FP64 within the exact bar of the oracle's at-points
    sums; MIXED against the double-double truth at p = 10^6 (sorted query
    points, every 4th eigenvalue, so warps hold compact target ranges and the
    FP32 far field is used), median relative error of the complex sum below
    1e-9 and max below 3e-8."""
    L = _native.load()
    stream = torch.cuda.current_stream().cuda_stream
    d = _dev()
    p = 1_000_000
    ev_h = spectra.config2(p, seed=2)
    eta = 1.0 / np.sqrt(p)
    ev = torch.from_numpy(ev_h).to(d)
    q_h = np.ascontiguousarray(ev_h[::4])
    q = torch.from_numpy(q_h).to(d)
    idx = np.random.default_rng(8).choice(q_h.size, 48, replace=False)
    t_re, t_im = oracle.truth_points(q_h[idx], ev_h, eta)
    re, im = _out(q_h.size)
    _noalloc(L, q, ev, eta, MIXED, re, im, stream)
    torch.cuda.synchronize()
    m_re, m_im = re.cpu().numpy()[idx], im.cpu().numpy()[idx]
    err = np.hypot(m_re - t_re, m_im - t_im) / np.hypot(t_re, t_im)
    assert np.median(err) < 1e-9 and np.max(err) < 3e-8, (np.median(err), np.max(err))
    _noalloc(L, q, ev, eta, F64, re, im, stream)
    torch.cuda.synchronize()
    f_re, f_im = re.cpu().numpy()[idx], im.cpu().numpy()[idx]
    o_re, o_im = oracle.compute_at_points(q_h[idx], ev_h, eta, "blocked")
    scale = np.maximum(np.maximum(np.abs(o_re), np.abs(o_im)), 1e-12)
    assert np.max((np.abs(f_re - o_re) + np.abs(f_im - o_im)) / scale) <= BAR


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
