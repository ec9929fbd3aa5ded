"""Target sharding of the exact transform across ranks (CPU, gloo, world 2).

The ranks' logic (shard ranges, padded all-gather, rank-order assembly)
runs on the host with the oracle's exact at-points sums standing in for the
GPU kernel; the gathered transform must equal the oracle's unsharded
compute_all_stieltjes within the FP64 bar (1e-12 relative per point).
"""
import datetime
import os
import socket
import tempfile

import numpy as np
import pytest
import torch.multiprocessing as mp

from shrinkers_b200.sharding import shard_range


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
