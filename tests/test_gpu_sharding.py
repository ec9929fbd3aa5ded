"""The per-rank GPU work of the multi-GPU forms, on one GPU.

Every shard of a multi-GPU call is an independent launch on its rank's GPU
(the NUFFT's density all-reduce being the one exchange), so one GPU can run
all shards of a call one after the other and check that they assemble into
the single call's values:

* shrk_stieltjes_shard_dev, all points: the treecode presets, the NUFFT, the
  fft5 grid and the FMM ("treecode") give the single call's values bit for
  bit at every slice; the exact sums to 1e-13 (their split reduction follows
  the launch shape);
* shrk_stieltjes_shard_dev at points: the treecode's shards with the whole
  query count bit for bit; with only their own count the leaf capacity (and
  so the tree) changes, which is why the entry point takes nq_total;
* the NUFFT stages: splatting a whole spectrum and evaluating is the fused
  call bit for bit; densities of source shards summed give the oracle's
  NUFFT to 1e-10 of its largest value (the NUFFT bar);
* the batched launch over a p^2-weighted range of spectra matches the whole
  batch's slice;
* the Python helpers without a process group run the whole call on this GPU.
"""
import ctypes as C
import math

import numpy as np
import pytest
import torch

from shrinkers_b200 import _native, spectra
from shrinkers_b200.sharding import (GpuBackend, nufft_sharded, shard_range,
                                     stieltjes_at_points_sharded, stieltjes_batched_sharded,
                                     stieltjes_transform_sharded, weighted_shard_ranges)

pytestmark = pytest.mark.gpu
NAN = float("nan")
IDS = {"blocked": 2, "nufft": 11, "fft5": 8, "treecode": 12, "chebcode": 13,
       "chebcode_fast": 14, "chebcode_xtreme": 15}


def dev():
    return torch.device("cuda", 0)


def all_dev(ev_t, eta, method, precision=0):
    L = _native.load()
    p = ev_t.numel()
    re = torch.empty(p, dtype=torch.float64, device=dev())
    im = torch.empty_like(re)
    _native.check(L.shrk_stieltjes_all_dev(ev_t.data_ptr(), p, eta, IDS[method], precision, NAN,
                                           0, re.data_ptr(), im.data_ptr(),
                                           torch.cuda.current_stream().cuda_stream))
    return re.cpu().numpy(), im.cpu().numpy()


def points_dev(q_t, ev_t, eta, method):
    L = _native.load()
    re = torch.empty(q_t.numel(), dtype=torch.float64, device=dev())
    im = torch.empty_like(re)
    _native.check(L.shrk_stieltjes_at_points_dev(q_t.data_ptr(), q_t.numel(), ev_t.data_ptr(),
                                                 ev_t.numel(), eta, IDS[method], 0, NAN, 0,
                                                 re.data_ptr(), im.data_ptr(),
                                                 torch.cuda.current_stream().cuda_stream))
    return re.cpu().numpy(), im.cpu().numpy()


def shard(q_t, nq_total, all_points, ev_t, eta, method, precision=0):
    L = _native.load()
    re = torch.empty(q_t.numel(), dtype=torch.float64, device=dev())
    im = torch.empty_like(re)
    _native.check(L.shrk_stieltjes_shard_dev(q_t.data_ptr(), q_t.numel(), nq_total, all_points,
                                             ev_t.data_ptr(), ev_t.numel(), eta, IDS[method],
                                             precision, NAN, 0, re.data_ptr(), im.data_ptr(),
                                             torch.cuda.current_stream().cuda_stream))
    return re.cpu().numpy(), im.cpu().numpy()


@pytest.mark.parametrize("method", ["chebcode", "chebcode_fast", "chebcode_xtreme", "nufft",
                                    "fft5", "treecode", "blocked"])
@pytest.mark.parametrize("world", [2, 3])
def test_all_points_shards_assemble_into_the_single_call(method, world):
    p = 30011
    ev = spectra.config3(p, seed=5)
    eta = 1.0 / math.sqrt(p)
    t = torch.from_numpy(ev).to(dev())
    full_re, full_im = all_dev(t, eta, method)
    re, im = np.empty(p), np.empty(p)
    for r in range(world):
        a, b = shard_range(p, world, r)
        re[a:b], im[a:b] = shard(t.narrow(0, a, b - a), p, 1, t, eta, method)
    if method == "blocked":
        scale = np.maximum(np.maximum(np.abs(full_re), np.abs(full_im)), 1e-300)
        assert np.max((np.abs(re - full_re) + np.abs(im - full_im)) / scale) < 1e-13
    else:
        np.testing.assert_array_equal(re, full_re)
        np.testing.assert_array_equal(im, full_im)


def test_all_points_shard_rejects_targets_outside_the_spectrum():
    L = _native.load()
    ev = torch.from_numpy(spectra.config2(1000, seed=1)).to(dev())
    q = ev.clone()
    re = torch.empty_like(ev)
    st = L.shrk_stieltjes_shard_dev(q.data_ptr(), 1000, 1000, 1, ev.data_ptr(), 1000, 0.03, 13, 0,
                                    NAN, 0, re.data_ptr(), re.data_ptr(),
                                    torch.cuda.current_stream().cuda_stream)
    assert st == _native.SHRK_EINVAL
    st = L.shrk_stieltjes_shard_dev(q.data_ptr(), 10, 5, 0, ev.data_ptr(), 1000, 0.03, 13, 0,
                                    NAN, 0, re.data_ptr(), re.data_ptr(),
                                    torch.cuda.current_stream().cuda_stream)
    assert st == _native.SHRK_EINVAL


@pytest.mark.parametrize("method", ["chebcode", "chebcode_fast", "nufft"])
def test_query_shards_use_the_whole_query_count(method):
    p, nq, world = 50000, 4000, 4
    ev = spectra.config3(p, seed=6)
    eta = 1.0 / math.sqrt(p)
    q = np.linspace(ev[0] - 0.2, ev[-1] + 0.2, nq)
    t, tq = torch.from_numpy(ev).to(dev()), torch.from_numpy(q).to(dev())
    full_re, full_im = points_dev(tq, t, eta, method)
    re, im = np.empty(nq), np.empty(nq)
    for r in range(world):
        a, b = shard_range(nq, world, r)
        re[a:b], im[a:b] = shard(tq.narrow(0, a, b - a), nq, 0, t, eta, method)
    np.testing.assert_array_equal(re, full_re)
    np.testing.assert_array_equal(im, full_im)


def test_nufft_stages(oracle):
    p = 200_003
    ev = spectra.config3(p, seed=8)
    eta = 1.0 / math.sqrt(p)
    be = GpuBackend()
    m, lo, dx = be.nufft_grid(ev[0], ev[-1], eta)
    assert (m, lo, dx) == oracle.nufft_geometry(ev[0], ev[-1], eta)
    t = torch.from_numpy(ev).to(dev())
    # one stage pair over every source = the fused call, bit for bit
    dens = be.nufft_density(ev, m, lo, dx)
    re, im = be.nufft_eval(dens, m, lo, dx, eta, ev)
    f_re, f_im = all_dev(t, eta, "nufft")
    np.testing.assert_array_equal((re * (1.0 / p)).cpu().numpy(), f_re)
    np.testing.assert_array_equal((im * (1.0 / p)).cpu().numpy(), f_im)
    # the density equals the oracle's sequential splat to rounding
    o_dens = oracle.grid_density(ev, m, lo, dx)
    assert np.max(np.abs(dens.cpu().numpy() - o_dens)) <= 1e-12 * np.max(np.abs(o_dens))
    # three source shards, densities summed (the all-reduce), queries shared
    parts = [be.nufft_density(ev[a:b], m, lo, dx)
             for a, b in (shard_range(p, 3, r) for r in range(3))]
    total = parts[0] + parts[1] + parts[2]
    q = np.linspace(ev[0] - 1.0, ev[-1] + 1.0, 5000)
    re, im = be.nufft_eval(total, m, lo, dx, eta, q)
    o_re, o_im = oracle.nufft_points(q, ev, eta)
    scale = max(np.abs(o_re).max(), np.abs(o_im).max())
    assert np.max(np.abs(re.cpu().numpy() - o_re)) <= 1e-10 * scale
    assert np.max(np.abs(im.cpu().numpy() - o_im)) <= 1e-10 * scale
    # an empty shard splats nothing
    z = be.nufft_density(np.empty(0), m, lo, dx)
    assert torch.count_nonzero(z).item() == 0


def test_nufft_stage_arguments_are_checked():
    L = _native.load()
    d = torch.zeros(16, dtype=torch.float64, device=dev())
    s = torch.cuda.current_stream().cuda_stream
    assert L.shrk_nufft_density_dev(d.data_ptr(), 4, 1, 0.0, 0.1, d.data_ptr(), s) == \
        _native.SHRK_EINVAL
    assert L.shrk_nufft_density_dev(d.data_ptr(), 4, 16, 0.0, 0.0, d.data_ptr(), s) == \
        _native.SHRK_EINVAL
    assert L.shrk_nufft_eval_dev(d.data_ptr(), 16, 0.0, 0.1, -1.0, d.data_ptr(), 4, d.data_ptr(),
                                 d.data_ptr(), s) == _native.SHRK_EINVAL


def test_batched_spectrum_shards_match_the_whole_batch():
    vals, offs, etas = spectra.config4(n_spectra=300, seed=12)
    be = GpuBackend()
    full_re, full_im = be.batched(vals, offs, etas, "f64")
    full_re, full_im = full_re.cpu().numpy(), full_im.cpu().numpy()
    sizes = np.diff(offs)
    for world in (2, 3):
        for s_lo, s_hi in weighted_shard_ranges(sizes.astype(np.float64) ** 2, world):
            a, b = int(offs[s_lo]), int(offs[s_hi])
            re, im = be.batched(vals[a:b], offs[s_lo:s_hi + 1] - a, etas[s_lo:s_hi], "f64")
            scale = np.maximum(np.maximum(np.abs(full_re[a:b]), np.abs(full_im[a:b])), 1e-300)
            err = (np.abs(re.cpu().numpy() - full_re[a:b]) +
                   np.abs(im.cpu().numpy() - full_im[a:b])) / scale
            assert np.max(err) < 1e-13


def test_helpers_without_a_process_group(oracle):
    p = 20011
    ev = spectra.config2(p, seed=13)
    eta = 1.0 / math.sqrt(p)
    q = np.linspace(ev[0] - 0.1, ev[-1] + 0.1, 3001)
    re, im = stieltjes_transform_sharded(ev, eta, method="chebcode")
    o_re, o_im = oracle.compute_all(ev, eta, "chebcode")
    np.testing.assert_array_equal(re.cpu().numpy(), o_re)
    np.testing.assert_array_equal(im.cpu().numpy(), o_im)
    re, im = stieltjes_at_points_sharded(q, ev, eta)
    o_re, o_im = oracle.compute_at_points(q, ev, eta, "blocked")
    scale = np.maximum(np.maximum(np.abs(o_re), np.abs(o_im)), 1e-300)
    assert np.max((np.abs(re.cpu().numpy() - o_re) + np.abs(im.cpu().numpy() - o_im)) / scale) \
        < 1e-12
    re, im = nufft_sharded(ev, eta, queries=q)
    o_re, o_im = oracle.nufft_points(q, ev, eta)
    scale = max(np.abs(o_re).max(), np.abs(o_im).max())
    assert np.max(np.abs(re.cpu().numpy() - o_re)) <= 1e-10 * scale
    vals, offs, etas = spectra.config4(n_spectra=40, seed=14)
    b_re, b_im, rng = stieltjes_batched_sharded(vals, offs, etas)
    assert rng == (0, 40)
    for s_ in range(0, 40, 7):
        a, b = offs[s_], offs[s_ + 1]
        o_re, o_im = oracle.compute_all(vals[a:b], float(etas[s_]), "blocked")
        scale = np.maximum(np.maximum(np.abs(o_re), np.abs(o_im)), 1e-300)
        err = (np.abs(b_re.cpu().numpy()[a:b] - o_re) + np.abs(b_im.cpu().numpy()[a:b] - o_im))
        assert np.max(err / scale) < 1e-12
