"""Target-sharded exact transform over several GPUs (one process per GPU).

The exact all-points transform is independent per target: rank r of a
world of N computes the targets ``shard_range(p, N, r)`` against the whole
(replicated) spectrum on its own GPU and no data crosses between GPUs while
computing.  ``gather=True`` then assembles the full result on every rank
with one all-gather (the only collective, and only when the caller wants
the whole array).

The per-rank work is a raw at-points sum (``shrk_stieltjes_at_points_dev``
with the exact method) scaled by 1/p, i.e. the all-points convention of
``compute_all_stieltjes`` (src/stieltjes/mod.rs:601-790) restricted to the
shard's targets.  ``compute`` can be replaced (the CPU tests pass a host
implementation so the rank logic runs under ``gloo`` without a GPU).
"""
from __future__ import annotations

from typing import Callable, Optional, Tuple

import numpy as np

_PREC = {"f64": 0, "mixed": 1}


def shard_range(n: int, world: int, rank: int) -> Tuple[int, int]:
    """Contiguous, balanced [lo, hi) of n items for `rank` of `world`
    (the first n % world ranks get one extra item)."""
    if world <= 0 or not (0 <= rank < world):
        raise ValueError("rank must lie in [0, world)")
    if n < 0:
        raise ValueError("n must be non-negative")
    base, extra = divmod(n, world)
    lo = rank * base + min(rank, extra)
    return lo, lo + base + (1 if rank < extra else 0)


def _gpu_compute(precision: str):
    """Raw exact sums at `targets` against `sources` on the current CUDA device."""
    import torch
    from . import _native

    def compute(targets, sources, eta):
        L = _native.load()
        dev = torch.device("cuda", torch.cuda.current_device())
        t = torch.as_tensor(targets, dtype=torch.float64, device=dev).contiguous()
        s = torch.as_tensor(sources, dtype=torch.float64, device=dev).contiguous()
        re = torch.empty_like(t)
        im = torch.empty_like(t)
        st = L.shrk_stieltjes_at_points_dev(t.data_ptr(), t.numel(), s.data_ptr(), s.numel(), eta,
                                            2, _PREC[precision], float("nan"), 0, re.data_ptr(),
                                            im.data_ptr(), torch.cuda.current_stream().cuda_stream)
        _native.check(st, "stieltjes_at_points_dev")
        return re, im

    return compute


def stieltjes_transform_sharded(eigenvalues, eta: Optional[float] = None, precision: str = "f64",
                                group=None, gather: bool = True,
                                compute: Optional[Callable] = None):
    """Exact all-points transform S(ev_i)/p sharded by targets over the ranks
    of ``group`` (default: the world).

    Returns ``(re, im)`` for this rank's targets, or for all p targets when
    ``gather`` (assembled in rank order).  Arrays are torch tensors on the
    compute device (host tensors with a host ``compute``)."""
    import torch
    import torch.distributed as dist

    ev = np.ascontiguousarray(np.asarray(eigenvalues, dtype=np.float64))
    p = ev.size
    if p == 0:
        raise ValueError("eigenvalues must be non-empty")
    if precision not in _PREC:
        raise ValueError(f"unknown precision '{precision}' (expected 'f64' or 'mixed')")
    eta_v = 1.0 / np.sqrt(p) if eta is None else float(eta)
    if not (np.isfinite(eta_v) and eta_v > 0.0):
        raise ValueError("eta must be a positive finite number")
    world = dist.get_world_size(group) if dist.is_initialized() else 1
    rank = dist.get_rank(group) if dist.is_initialized() else 0
    lo, hi = shard_range(p, world, rank)
    fn = compute or _gpu_compute(precision)
    if hi > lo:
        re, im = fn(ev[lo:hi], ev, eta_v)
        re = torch.as_tensor(re) / p
        im = torch.as_tensor(im) / p
    else:
        re = im = torch.empty(0, dtype=torch.float64)
    if not gather or world == 1:
        return re, im
    # Equal-size all-gather: pad every shard to the largest one.
    width = shard_range(p, world, 0)[1]
    buf = torch.zeros(2, width, dtype=torch.float64, device=re.device)
    buf[0, :hi - lo] = re
    buf[1, :hi - lo] = im
    parts = [torch.empty_like(buf) for _ in range(world)]
    dist.all_gather(parts, buf, group=group)
    out_re = torch.empty(p, dtype=torch.float64, device=re.device)
    out_im = torch.empty_like(out_re)
    for r, part in enumerate(parts):
        a, b = shard_range(p, world, r)
        out_re[a:b] = part[0, :b - a]
        out_im[a:b] = part[1, :b - a]
    return out_re, out_im
