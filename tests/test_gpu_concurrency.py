"""Calls from several host threads and on several streams at once.

The library keeps its device scratch per (device, stream), and per (device,
host thread) for host-pointer calls, so concurrent calls neither serialise
on one process-wide lock nor share temporaries.  The reference releases the
GIL for the whole computation (python.rs:806-810) and its Python tests pin
that other threads keep running during a call (tests/test_python_api.py:
635-665); here ctypes releases the GIL around every foreign call, and:

* two host threads, each on its own spectrum and query grid, get the
  oracle's sums (bit for bit for the treecode) while the other runs;
* the pair of threads takes less wall time than the two runs one after the
  other (the calls are latency-bound query-grid calls, so they overlap);
* `_dev` calls on two CUDA streams from two threads, of different sizes,
  each match the oracle (no scratch shared between the streams), and
  shrk_stream_check / shrk_stream_release work on those streams.
"""
import ctypes as C
import math
import threading
import time

import numpy as np
import pytest
import torch

from shrinkers_b200 import _native, spectra

pytestmark = pytest.mark.gpu
NAN = float("nan")
_D = C.POINTER(C.c_double)
CHEB_FAST, BLOCKED = 14, 2


def dp(a):
    return a.ctypes.data_as(_D)


def grid_call(L, q, ev, eta):
    re, im = np.empty(q.size), np.empty(q.size)
    _native.check(L.shrk_stieltjes_at_points(dp(q), q.size, dp(ev), ev.size, eta, CHEB_FAST, 0,
                                             NAN, 0, dp(re), dp(im)))
    return re, im


def _cases():
    out = []
    for i, p in enumerate((20_000, 30_011)):
        ev = spectra.config2(p, seed=40 + i)
        q = np.linspace(ev[0] - 0.05, ev[-1] + 0.05, 200)
        out.append((q, ev, 1.0 / math.sqrt(p)))
    return out


def _run_threads(fns):
    errors = []

    def wrap(fn):
        try:
            fn()
        except BaseException as e:  # noqa: BLE001 - reported below
            errors.append(e)

    ts = [threading.Thread(target=wrap, args=(f,)) for f in fns]
    t0 = time.perf_counter()
    for t in ts:
        t.start()
    for t in ts:
        t.join()
    dt = time.perf_counter() - t0
    if errors:
        raise errors[0]
    return dt


def test_two_host_threads_match_oracle_and_overlap(oracle):
    L = _native.load()
    cases = _cases()
    refs = [oracle.compute_at_points(q, ev, eta, "chebcode_fast") for q, ev, eta in cases]
    reps = 60
    results = [None, None]

    def worker(k):
        def fn():
            q, ev, eta = cases[k]
            for _ in range(reps):
                results[k] = grid_call(L, q, ev, eta)
        return fn

    for k in range(2):  # warm both threads' paths (tree scratch, first launches)
        worker(k)()
    best_pair, best_serial = float("inf"), float("inf")
    for _ in range(3):
        t0 = time.perf_counter()
        worker(0)()
        worker(1)()
        best_serial = min(best_serial, time.perf_counter() - t0)
        best_pair = min(best_pair, _run_threads([worker(0), worker(1)]))
    for k in range(2):
        np.testing.assert_array_equal(results[k][0], refs[k][0])
        np.testing.assert_array_equal(results[k][1], refs[k][1])
    assert best_pair < 0.9 * best_serial, (best_pair, best_serial)


def test_dev_calls_on_two_streams_match_oracle(oracle):
    L = _native.load()
    d = torch.device("cuda", 0)
    sizes = (40_000, 65_537)
    evs = [spectra.config2(p, seed=50 + i) for i, p in enumerate(sizes)]
    refs = [oracle.compute_all(ev, 1.0 / math.sqrt(ev.size), "blocked", parallel=True)
            for ev in evs]
    streams = [torch.cuda.Stream(device=d) for _ in sizes]
    outs = [None, None]

    def worker(k):
        def fn():
            ev = evs[k]
            p = ev.size
            with torch.cuda.stream(streams[k]):
                t = torch.from_numpy(ev).to(d, non_blocking=False)
                re = torch.empty(p, dtype=torch.float64, device=d)
                im = torch.empty_like(re)
                for prec in (0, 1, 0):
                    _native.check(L.shrk_stieltjes_all_dev(
                        t.data_ptr(), p, 1.0 / math.sqrt(p), BLOCKED, prec, NAN, 0,
                        re.data_ptr(), im.data_ptr(), streams[k].cuda_stream))
                _native.check(L.shrk_stream_check(C.c_void_p(streams[k].cuda_stream)))
                outs[k] = (re.cpu().numpy(), im.cpu().numpy())
        return fn

    _run_threads([worker(0), worker(1)])
    for k in range(2):
        o_re, o_im = refs[k]
        scale = np.maximum(np.maximum(np.abs(o_re), np.abs(o_im)), 1e-12)
        err = (np.abs(outs[k][0] - o_re) + np.abs(outs[k][1] - o_im)) / scale
        assert np.max(err) < 1e-12, (k, np.max(err))
    for s in streams:
        _native.check(L.shrk_stream_release(C.c_void_p(s.cuda_stream)))
    # a released stream allocates afresh on its next call
    worker(0)()
    o_re, o_im = refs[0]
    assert np.max(np.abs(outs[0][0] - o_re) / np.maximum(np.abs(o_re), 1e-12)) < 1e-9
    _native.check(L.shrk_stream_release(C.c_void_p(streams[0].cuda_stream)))
