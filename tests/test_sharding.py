"""The multi-GPU forms (CPU, gloo, world 2 and 3).

The ranks' logic (shard ranges, the p^2-weighted spectrum partition, the
density all-reduce of the point-sharded NUFFT, padded all-gathers,
rank-order assembly) runs on the host with the oracle standing in for the
GPU: its exact at-points sums, its per-spectrum transforms and its NUFFT
stages (splat of a source shard onto a given grid; convolution + interpolation
of a density).  Bars: the gathered exact transform equals the oracle's
unsharded compute_all_stieltjes within the FP64 bar (1e-12 relative per
point); the batched shards are bit-identical to the per-spectrum transforms;
the sharded NUFFT equals the single-call NUFFT to 1e-13 of its largest value
(only the densities' summation order differs).
"""
import datetime
import os
import socket
import tempfile

import numpy as np
import pytest
import torch.multiprocessing as mp

from shrinkers_b200.sharding import shard_range, weighted_shard_ranges


@pytest.mark.parametrize("n", [0, 1, 5, 100, 1001])
@pytest.mark.parametrize("world", [1, 2, 3, 8])
def test_shard_ranges_partition_the_targets(n, world):
    ranges = [shard_range(n, world, r) for r in range(world)]
    assert ranges[0][0] == 0 and ranges[-1][1] == n
    for (a, b), (c, d) in zip(ranges, ranges[1:]):
        assert b == c and a <= b and c <= d
    sizes = [b - a for a, b in ranges]
    assert max(sizes) - min(sizes) <= 1


def test_shard_range_rejects_bad_rank():
    with pytest.raises(ValueError):
        shard_range(10, 2, 2)


@pytest.mark.parametrize("world", [1, 2, 3, 8])
@pytest.mark.parametrize("seed", [0, 1, 2])
def test_weighted_ranges_partition_and_balance(world, seed):
    rng = np.random.default_rng(seed)
    sizes = np.exp(rng.uniform(np.log(256), np.log(16384), 500)).astype(np.int64)
    w = sizes.astype(np.float64) ** 2
    ranges = weighted_shard_ranges(w, world)
    assert len(ranges) == world and ranges[0][0] == 0 and ranges[-1][1] == w.size
    for (a, b), (c, d) in zip(ranges, ranges[1:]):
        assert b == c and a <= b
    loads = np.array([w[a:b].sum() for a, b in ranges])
    # every rank's load is within one item of the ideal share
    assert np.all(np.abs(loads - w.sum() / world) <= w.max())


def test_weighted_ranges_edge_cases():
    assert weighted_shard_ranges([], 3) == [(0, 0)] * 3
    assert weighted_shard_ranges([0.0, 0.0, 0.0, 0.0], 2) == [(0, 2), (2, 4)]
    assert weighted_shard_ranges([1.0], 3) == [(0, 1), (1, 1), (1, 1)]
    with pytest.raises(ValueError):
        weighted_shard_ranges([1.0, -1.0], 2)
    with pytest.raises(ValueError):
        weighted_shard_ranges([1.0], 0)


class OracleBackend:
    """The per-rank work on the host through the oracle (exact sums and the
    NUFFT stages), returning CPU tensors like the GPU backend's."""

    def __init__(self):
        from oracle import oracle as O
        self.O = O

    @staticmethod
    def _t(a):
        import torch
        return torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64))

    def transform(self, ev, lo, hi, eta, method, precision):
        re, im = self.O.compute_at_points(ev[lo:hi], ev, eta, "blocked")
        return self._t(re * (1.0 / ev.size)), self._t(im * (1.0 / ev.size))

    def points(self, q, nq_total, ev, eta, method, precision):
        re, im = self.O.compute_at_points(q, ev, eta, "blocked")
        return self._t(re), self._t(im)

    def batched(self, values, offsets, etas, precision):
        re, im = np.empty(values.size), np.empty(values.size)
        for s_ in range(offsets.size - 1):
            a, b = offsets[s_], offsets[s_ + 1]
            re[a:b], im[a:b] = self.O.compute_all(values[a:b], float(etas[s_]), "blocked")
        return self._t(re), self._t(im)

    def nufft_grid(self, first, last, eta):
        return self.O.nufft_geometry(first, last, eta)

    def nufft_density(self, src, m, lo, dx):
        return self._t(self.O.grid_density(src, m, lo, dx))

    def nufft_eval(self, density, m, lo, dx, eta, q):
        re, im = self.O.grid_eval(density.numpy(), m, lo, dx, eta, q)
        return self._t(re), self._t(im)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, p, eta, gather, out_dir):
    import torch
    import torch.distributed as dist
    from oracle import oracle as O
    from shrinkers_b200 import spectra
    from shrinkers_b200.sharding import stieltjes_transform_sharded

    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank,
                            world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        ev = spectra.config2(p, seed=7) if p > 3 else np.array([0.5, 1.0, 2.0])[:p]

        def compute(targets, sources, e):
            re, im = O.compute_at_points(targets, sources, e, "blocked")
            return torch.from_numpy(re), torch.from_numpy(im)

        re, im = stieltjes_transform_sharded(ev, eta, group=None, gather=gather, compute=compute)
        np.save(os.path.join(out_dir, f"re{rank}.npy"), re.numpy())
        np.save(os.path.join(out_dir, f"im{rank}.npy"), im.numpy())
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("p,gather", [(3001, True), (3001, False), (1, True)])
def test_sharded_transform_matches_unsharded(oracle, p, gather):
    from shrinkers_b200 import spectra

    world = 2
    eta = 1.0 / np.sqrt(p)
    with tempfile.TemporaryDirectory() as d:
        mp.start_processes(_worker, args=(world, _free_port(), p, eta, gather, d), nprocs=world,
                           join=True, start_method="spawn")
        outs = [(np.load(os.path.join(d, f"re{r}.npy")), np.load(os.path.join(d, f"im{r}.npy")))
                for r in range(world)]
    ev = spectra.config2(p, seed=7) if p > 3 else np.array([0.5, 1.0, 2.0])[:p]
    o_re, o_im = oracle.compute_all(ev, eta, "blocked")
    scale = np.maximum(np.maximum(np.abs(o_re), np.abs(o_im)), 1e-12)
    if gather:
        for re, im in outs:  # every rank holds the whole transform
            assert np.max((np.abs(re - o_re) + np.abs(im - o_im)) / scale) <= 1e-12
    else:
        for r, (re, im) in enumerate(outs):
            a, b = shard_range(p, world, r)
            assert re.size == b - a
            assert np.max((np.abs(re - o_re[a:b]) + np.abs(im - o_im[a:b])) / scale[a:b]) <= 1e-12


@pytest.mark.gpu
@pytest.mark.parametrize("precision,bar", [("f64", 1e-12), ("mixed", 1e-8)])
def test_single_rank_gpu_path_matches_oracle(oracle, precision, bar):
    """Without a process group the helper runs the whole transform on the
    current GPU through shrk_stieltjes_at_points_dev."""
    from shrinkers_b200 import spectra
    from shrinkers_b200.sharding import stieltjes_transform_sharded

    p = 4099
    ev = spectra.config2(p, seed=3)
    eta = 1.0 / np.sqrt(p)
    re, im = stieltjes_transform_sharded(ev, eta, precision=precision)
    o_re, o_im = oracle.compute_all(ev, eta, "blocked")
    scale = np.maximum(np.maximum(np.abs(o_re), np.abs(o_im)), 1e-12)
    err = (np.abs(re.cpu().numpy() - o_re) + np.abs(im.cpu().numpy() - o_im)) / scale
    assert np.median(err) <= bar and np.max(err) <= max(bar, 1e-6)


def _batch_case():
    """20 spectra, p log-uniform in [50, 3000], eta = 1/sqrt(p)."""
    rng = np.random.default_rng(11)
    sizes = np.exp(rng.uniform(np.log(50), np.log(3000), 20)).astype(np.int64)
    offs = np.concatenate(([0], np.cumsum(sizes))).astype(np.int64)
    vals = np.concatenate([np.sort(rng.gamma(2.0, 0.5, n_)) for n_ in sizes])
    return vals, offs, 1.0 / np.sqrt(sizes.astype(np.float64))


def _forms_worker(rank, world, port, out_dir):
    import torch
    import torch.distributed as dist
    from shrinkers_b200 import spectra
    from shrinkers_b200.sharding import (nufft_sharded, stieltjes_at_points_sharded,
                                         stieltjes_batched_sharded)

    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank,
                            world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        be = OracleBackend()
        ev = spectra.config2(5003, seed=9)
        eta = 1.0 / np.sqrt(ev.size)
        q = np.linspace(ev[0] - 0.1, ev[-1] + 0.1, 777)
        res = {}
        res["nufft_all"] = nufft_sharded(ev, eta, backend=be)
        res["nufft_pts"] = nufft_sharded(ev, eta, queries=q, backend=be)
        res["nufft_part"] = nufft_sharded(ev, eta, queries=q, gather=False, backend=be)
        res["pts"] = stieltjes_at_points_sharded(q, ev, eta, backend=be)
        vals, offs, etas = _batch_case()
        b_re, b_im, rng_all = stieltjes_batched_sharded(vals, offs, etas, backend=be)
        p_re, p_im, rng_mine = stieltjes_batched_sharded(vals, offs, etas, gather=False,
                                                         backend=be)
        res["batched"] = (b_re, b_im)
        res["batched_part"] = (p_re, p_im)
        res["ranges"] = (torch.tensor(rng_all), torch.tensor(rng_mine))
        for k, (a, b) in res.items():
            np.save(os.path.join(out_dir, f"{k}_re{rank}.npy"), a.numpy())
            np.save(os.path.join(out_dir, f"{k}_im{rank}.npy"), b.numpy())
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_sharded_forms_match_single_calls(oracle, world):
    from shrinkers_b200 import spectra

    with tempfile.TemporaryDirectory() as d:
        mp.start_processes(_forms_worker, args=(world, _free_port(), d), nprocs=world, join=True,
                           start_method="spawn")

        def load(k, r):
            return (np.load(os.path.join(d, f"{k}_re{r}.npy")),
                    np.load(os.path.join(d, f"{k}_im{r}.npy")))

        ev = spectra.config2(5003, seed=9)
        eta = 1.0 / np.sqrt(ev.size)
        q = np.linspace(ev[0] - 0.1, ev[-1] + 0.1, 777)
        n_re, n_im = oracle.nufft_points(ev, ev, eta)
        q_re, q_im = oracle.nufft_points(q, ev, eta)
        e_re, e_im = oracle.compute_at_points(q, ev, eta, "blocked")
        vals, offs, etas = _batch_case()
        sizes = np.diff(offs)
        spec = weighted_shard_ranges(sizes.astype(np.float64) ** 2, world)
        for r in range(world):
            re, im = load("nufft_all", r)
            scale = max(np.abs(n_re).max(), np.abs(n_im).max()) / ev.size
            assert np.max(np.abs(re - n_re / ev.size)) <= 1e-13 * scale
            assert np.max(np.abs(im - n_im / ev.size)) <= 1e-13 * scale
            scale = max(np.abs(q_re).max(), np.abs(q_im).max())
            re, im = load("nufft_pts", r)
            assert np.max(np.abs(re - q_re)) <= 1e-13 * scale
            assert np.max(np.abs(im - q_im)) <= 1e-13 * scale
            a, b = shard_range(q.size, world, r)
            re, im = load("nufft_part", r)
            assert re.size == b - a
            assert np.max(np.abs(re - q_re[a:b])) <= 1e-13 * scale
            re, im = load("pts", r)
            np.testing.assert_array_equal(re, e_re)
            np.testing.assert_array_equal(im, e_im)
            # batched: every spectrum's own transform, bit for bit
            re, im = load("batched", r)
            pr, pi = load("batched_part", r)
            rng_all, rng_mine = load("ranges", r)
            assert tuple(rng_all) == (0, sizes.size)
            assert tuple(rng_mine) == spec[r]
            s_lo, s_hi = spec[r]
            for s_ in range(sizes.size):
                a, b = offs[s_], offs[s_ + 1]
                o_re, o_im = oracle.compute_all(vals[a:b], float(etas[s_]), "blocked")
                np.testing.assert_array_equal(re[a:b], o_re)
                np.testing.assert_array_equal(im[a:b], o_im)
                if s_lo <= s_ < s_hi:
                    base = offs[s_lo]
                    np.testing.assert_array_equal(pr[a - base:b - base], o_re)
            assert pr.size == offs[s_hi] - offs[s_lo]
