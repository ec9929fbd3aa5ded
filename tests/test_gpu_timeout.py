"""The timeout path of the bounded device-side waits, exercised without a
fault: with a wait budget of zero cycles (shrk_diag_set_wait_limit) every
bulk-copy wait of the exact pair kernels gives up at once, the kernels record
the timeout in the device error word, wait for their own copies in flight
and return.  Then:

* the host-pointer entry point returns SHRK_ETIMEOUT with a message;
* the allocation-free entry point (stream-ordered, no read-back) writes NaN
  to every output;
* with the budget restored, the next calls are correct (bit-identical to the
  calls before, and equal to the oracle), so the context and the library's
  state survived.

Nothing here traps, faults or hangs: the waits return, and the drain of the
copies in flight keeps its own (long) budget.
"""
import ctypes as C
import math

import numpy as np
import pytest
import torch

from shrinkers_b200 import _native, spectra

pytestmark = pytest.mark.gpu

F64, MIXED = 0, 1
BLOCKED = 2
ETIMEOUT = 3
NAN = float("nan")
_D = C.POINTER(C.c_double)


def dp(a):
    return a.ctypes.data_as(_D)


def host_all(L, ev, eta, precision):
    re, im = np.empty(ev.size), np.empty(ev.size)
    st = L.shrk_stieltjes_all(dp(ev), ev.size, eta, BLOCKED, precision, NAN, 0, dp(re), dp(im))
    return st, re, im


def noalloc(L, q, ev, eta, precision):
    re, im = torch.empty_like(q), torch.empty_like(q)
    st = L.shrk_stieltjes_at_points_noalloc(q.data_ptr(), q.numel(), ev.data_ptr(), ev.numel(),
                                            eta, precision, re.data_ptr(), im.data_ptr(),
                                            torch.cuda.current_stream().cuda_stream)
    _native.check(st, "noalloc")
    torch.cuda.synchronize()
    return re.cpu().numpy(), im.cpu().numpy()


def test_zero_wait_budget_times_out_and_the_library_recovers(oracle):
    L = _native.load()
    # 65 536 targets and sources: full 256 x 4 target tiles and splits of
    # whole 1 024-source chunks, so every item stages its sources by TMA.
    p = 65536
    ev = spectra.config2(p, seed=21)
    eta = 1.0 / math.sqrt(p)
    d = torch.device("cuda", 0)
    tev = torch.from_numpy(ev).to(d)
    tq = tev[::16].contiguous()
    before = {prec: host_all(L, ev, eta, prec) for prec in (F64, MIXED)}
    for prec in (F64, MIXED):
        assert before[prec][0] == 0
    old = L.shrk_diag_set_wait_limit(0)
    try:
        assert old > 0
        for prec in (F64, MIXED):
            st, _, _ = host_all(L, ev, eta, prec)
            assert st == ETIMEOUT, (prec, st)
            assert "timeout" in _native.last_error()
            re, im = noalloc(L, tq, tev, eta, prec)
            assert np.all(np.isnan(re)) and np.all(np.isnan(im)), prec
    finally:
        assert L.shrk_diag_set_wait_limit(-1) == 0
    assert L.shrk_diag_set_wait_limit(-1) == old
    for prec in (F64, MIXED):
        st, re, im = host_all(L, ev, eta, prec)
        assert st == 0, _native.last_error()
        np.testing.assert_array_equal(re, before[prec][1])
        np.testing.assert_array_equal(im, before[prec][2])
    o_re, o_im = oracle.compute_all(ev, eta, "blocked", parallel=True)
    scale = np.maximum(np.maximum(np.abs(o_re), np.abs(o_im)), 1e-12)
    err = (np.abs(before[F64][1] - o_re) + np.abs(before[F64][2] - o_im)) / scale
    assert np.max(err) < 1e-12
    q = tq.cpu().numpy()
    re, im = noalloc(L, tq, tev, eta, F64)
    q_re, q_im = oracle.compute_at_points(q, ev, eta, "blocked")
    scale = np.maximum(np.maximum(np.abs(q_re), np.abs(q_im)), 1e-12)
    assert np.max((np.abs(re - q_re) + np.abs(im - q_im)) / scale) < 1e-12
