"""Batched uneven spectra in one persistent launch (GPU; through the C ABI).

Every spectrum of a batch must match its own single transform: the FP64
batched path within the exact kernels' FP64 bar (1e-12 relative, normwise
and per point with the floor scale max(|re|, |im|, 1e-12)) against the
oracle's compute_all_stieltjes; the mixed path within the mixed bar against
the double-double truth (median over all points of all spectra).
"""
import ctypes as C
import math

import numpy as np
import pytest

import shrinkers_b200 as rk
from shrinkers_b200 import _native, spectra

pytestmark = pytest.mark.gpu

F64, MIXED = 0, 1
_D = C.POINTER(C.c_double)
_I64 = C.POINTER(C.c_int64)


def _ragged(sizes, seed):
    rng = np.random.default_rng(seed)
    arrs = []
    for p in sizes:
        c = rng.uniform(0.05, 0.9)
        arrs.append(spectra.mp_spectrum(int(p), c, seed=int(rng.integers(1 << 30))))
    return arrs


def _batched_host(arrs, etas, precision):
    L = _native.load()
    offs = np.zeros(len(arrs) + 1, np.int64)
    offs[1:] = np.cumsum([a.size for a in arrs])
    vals = np.ascontiguousarray(np.concatenate(arrs))
    etas = np.ascontiguousarray(np.asarray(etas, dtype=np.float64))
    re, im = np.empty(vals.size), np.empty(vals.size)
    st = L.shrk_stieltjes_batched(vals.ctypes.data_as(_D), offs.ctypes.data_as(_I64), len(arrs),
                                  etas.ctypes.data_as(_D), precision, re.ctypes.data_as(_D),
                                  im.ctypes.data_as(_D))
    _native.check(st, "stieltjes_batched")
    return [(re[offs[s]:offs[s + 1]], im[offs[s]:offs[s + 1]]) for s in range(len(arrs))]


def _rel_pointwise(re, im, rr, ri):
    scale = np.maximum(np.maximum(np.abs(rr), np.abs(ri)), 1e-12)
    return (np.abs(re - rr) + np.abs(im - ri)) / scale


# Sizes straddle every tile / split / chunk boundary of both R = 2 and R = 4
# plans and include odd lengths (offsets that break 16-byte alignment, so
# some spectra take the plain-load path instead of bulk copies).
SIZES = [1, 2, 3, 255, 256, 257, 511, 513, 1023, 1024, 1025, 2047, 2049, 4095, 4097, 8193,
         16384, 700, 3001, 5]


def test_f64_matches_oracle_per_spectrum(oracle):
    arrs = _ragged(SIZES, seed=1)
    etas = [1.0 / math.sqrt(a.size) for a in arrs]
    out = _batched_host(arrs, etas, F64)
    for a, eta, (re, im) in zip(arrs, etas, out):
        rr, ri = oracle.compute_all(a, eta, "blocked")
        assert np.max(_rel_pointwise(re, im, rr, ri)) <= 1e-12, a.size


def test_mixed_median_error_vs_truth(oracle):
    arrs = _ragged([300, 1500, 4000, 9000, 16000, 777], seed=2)
    etas = [1.0 / math.sqrt(a.size) for a in arrs]
    out = _batched_host(arrs, etas, MIXED)
    errs = []
    for a, eta, (re, im) in zip(arrs, etas, out):
        tr, ti = oracle.truth_points(a, a, eta)
        tr, ti = tr / a.size, ti / a.size
        e = np.abs((re + 1j * im) - (tr + 1j * ti)) / np.abs(tr + 1j * ti)
        errs.append(e)
        assert np.max(e) <= 1e-6, a.size
    assert np.median(np.concatenate(errs)) <= 2e-9


def test_uneven_batch_like_config4_matches_single_transforms():
    vals, offs, etas = spectra.config4(n_spectra=96, seed=4)
    arrs = [vals[offs[s]:offs[s + 1]] for s in range(offs.size - 1)]
    out64 = _batched_host(arrs, etas, F64)
    outm = _batched_host(arrs, etas, MIXED)
    errs = []
    for a, eta, (re, im), (mre, mim) in zip(arrs, etas, out64, outm):
        res = rk.stieltjes_transform(a, eta=float(eta), method="blocked")
        assert np.max(_rel_pointwise(re, im, res["real"], res["imag"])) <= 1e-12
        errs.append(np.abs((mre + 1j * mim) - (re + 1j * im)) / np.abs(re + 1j * im))
    e = np.concatenate(errs)
    assert np.median(e) <= 2e-9 and np.max(e) <= 1e-6


def test_graph_replay_is_bit_identical():
    arrs = _ragged([2000, 3000, 517, 4096], seed=3)
    etas = [1.0 / math.sqrt(a.size) for a in arrs]
    for prec in (F64, MIXED):
        first = _batched_host(arrs, etas, prec)
        L = _native.load()
        n0 = L.shrk_launch_count()
        again = _batched_host(arrs, etas, prec)
        assert L.shrk_launch_count() > n0
        for (a, b), (c, d) in zip(first, again):
            assert np.array_equal(a, c) and np.array_equal(b, d)


def test_device_entry_matches_host_entry():
    import torch

    arrs = _ragged([1000, 2500, 33, 4097], seed=5)
    etas = np.array([1.0 / math.sqrt(a.size) for a in arrs])
    host = _batched_host(arrs, etas, MIXED)
    dev = torch.device("cuda", 0)
    offs = np.zeros(len(arrs) + 1, np.int64)
    offs[1:] = np.cumsum([a.size for a in arrs])
    v = torch.from_numpy(np.concatenate(arrs)).to(dev)
    o = torch.from_numpy(offs).to(dev)
    e = torch.from_numpy(etas).to(dev)
    re, im = torch.empty_like(v), torch.empty_like(v)
    L = _native.load()
    st = L.shrk_stieltjes_batched_dev(v.data_ptr(), o.data_ptr(), len(arrs), e.data_ptr(), MIXED,
                                      re.data_ptr(), im.data_ptr(),
                                      torch.cuda.current_stream().cuda_stream)
    _native.check(st, "stieltjes_batched_dev")
    torch.cuda.synchronize()
    re, im = re.cpu().numpy(), im.cpu().numpy()
    for s, (hr, hi) in enumerate(host):
        assert np.array_equal(re[offs[s]:offs[s + 1]], hr)
        assert np.array_equal(im[offs[s]:offs[s + 1]], hi)


def test_autotuner_table_and_retune():
    L = _native.load()
    arrs = _ragged([600, 3000, 12000], seed=6)
    etas = [1.0 / math.sqrt(a.size) for a in arrs]
    before = _batched_host(arrs, etas, F64)
    table = (C.c_int32 * 16)()
    _native.check(L.shrk_batched_autotune(F64, 1, table), "batched_autotune")
    t = list(table)
    assert all(r in (2, 4) for r in t[0::2])
    assert all(sl in (1024, 2048, 4096, 8192) for sl in t[1::2])
    after = _batched_host(arrs, etas, F64)
    for (a, b), (c, d) in zip(before, after):
        assert np.max(_rel_pointwise(c, d, a, b)) <= 1e-12


def test_set_tune_installs_a_saved_table():
    """A table saved from one run (or written by hand) installs without
    tuning; plans then follow it (here every bucket forced to R = 2 and
    SL = 1024, then to R = 4, SL = 8192), and results stay within the FP64
    bar; out-of-range entries are rejected."""
    L = _native.load()
    arrs = _ragged([300, 2500, 9000, 17000], seed=8)
    etas = [1.0 / math.sqrt(a.size) for a in arrs]
    saved = (C.c_int32 * 16)()
    _native.check(L.shrk_batched_autotune(F64, 0, saved), "batched_autotune")
    ref = _batched_host(arrs, etas, F64)
    try:
        for r, sl in ((2, 1024), (4, 8192)):
            t = (C.c_int32 * 16)(*([r, sl] * 8))
            _native.check(L.shrk_batched_set_tune(F64, t), "batched_set_tune")
            got = (C.c_int32 * 16)()
            _native.check(L.shrk_batched_autotune(F64, 0, got), "batched_autotune")
            assert list(got) == [r, sl] * 8
            for (a, b), (c, d) in zip(ref, _batched_host(arrs, etas, F64)):
                assert np.max(_rel_pointwise(c, d, a, b)) <= 1e-12
        bad = (C.c_int32 * 16)(*([3, 1024] * 8))
        assert L.shrk_batched_set_tune(F64, bad) == 1
        assert "R must be 2 or 4" in _native.last_error()
    finally:
        _native.check(L.shrk_batched_set_tune(F64, saved), "batched_set_tune")


def test_python_api_batched_matches_single():
    arrs = _ragged([100, 2000, 5000], seed=7)
    out = rk.stieltjes_transform_batched(arrs, precision="f64")
    for a, o in zip(arrs, out):
        res = rk.stieltjes_transform(a, eta=1.0 / math.sqrt(a.size), method="blocked")
        assert np.max(_rel_pointwise(o["real"], o["imag"], res["real"], res["imag"])) <= 1e-12


def test_validation():
    with pytest.raises(ValueError, match="non-empty"):
        rk.stieltjes_transform_batched([np.ones(3), np.empty(0)])
    with pytest.raises(ValueError, match="eta"):
        rk.stieltjes_transform_batched([np.ones(3)], eta=-1.0)
