"""Multi-GPU forms of the transform, one process per GPU.

Every form splits independent work across the ranks of a process group and
keeps the data path free of collectives except where the algorithm has a
real exchange step:

* ``stieltjes_transform_sharded`` -- all-points transform (any method) split
  by targets, spectrum replicated.  No collective while computing; one
  all-gather when the caller wants the whole array.  The treecode presets
  build their tree on every rank (the tree is small) and evaluate only the
  rank's targets.
* ``stieltjes_at_points_sharded`` -- the same for query points
  (compute_stieltjes_at_points, src/stieltjes/mod.rs:394-494): queries split,
  each rank using the policies of the whole query set (the treecode's grid
  leaf capacity, mod.rs:475-489), so the shards assemble into the single
  call's values.
* ``stieltjes_batched_sharded`` -- many uneven spectra split by spectrum,
  contiguous ranges balanced by the pair count sum p_s^2 (the work of the
  exact batched launch); no collective while computing.
* ``nufft_sharded`` -- the coarse-grid NUFFT (src/stieltjes/nufft.rs:164-220)
  split by points: each rank splats its shard of the sources onto the common
  grid, the densities are summed by one all-reduce of m <= 65 536 doubles
  (the only exchange the algorithm has), and each rank runs the (replicated)
  transforms and interpolates its shard of the queries.

The per-rank work runs through a backend; the default is the current CUDA
device through the C ABI.  The CPU tests pass a host backend (the oracle) so
the rank logic runs under ``gloo`` without a GPU.  A backend provides:

  transform(ev, lo, hi, eta, method, precision) -> (re, im)   S/p at ev[lo:hi]
  points(q, nq_total, ev, eta, method, precision) -> (re, im) raw sums at q
  batched(values, offsets, etas, precision) -> (re, im)       S/p_s per spectrum
  nufft_grid(first, last, eta) -> (m, lo, dx)
  nufft_density(src, m, lo, dx) -> float64 tensor [m]
  nufft_eval(density, m, lo, dx, eta, q) -> (re, im)          raw sums at q

Arrays come back as torch tensors (on the device for the GPU backend).
"""
from __future__ import annotations

import math
from typing import Callable, List, Optional, Sequence, Tuple

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


def weighted_shard_ranges(weights: Sequence[float], world: int) -> List[Tuple[int, int]]:
    """Contiguous [lo, hi) ranges of len(weights) items, one per rank, whose
    weight sums are balanced: rank r starts at the first item whose prefix
    weight (exclusive) reaches r / world of the total.  Deterministic, so
    every rank computes the same partition without communicating."""
    if world <= 0:
        raise ValueError("world must be positive")
    w = np.asarray(weights, dtype=np.float64).ravel()
    if np.any(w < 0) or not np.all(np.isfinite(w)):
        raise ValueError("weights must be finite and non-negative")
    n = w.size
    excl = np.concatenate(([0.0], np.cumsum(w)[:-1])) if n else np.zeros(0)
    total = float(np.sum(w))
    starts = [0]
    for r in range(1, world):
        starts.append(int(np.searchsorted(excl, total * r / world, side="left")) if total > 0
                      else shard_range(n, world, r)[0])
    starts.append(n)
    for r in range(1, world + 1):  # non-decreasing
        starts[r] = max(starts[r], starts[r - 1])
    return [(starts[r], starts[r + 1]) for r in range(world)]


def _world(group):
    import torch.distributed as dist
    if dist.is_available() and dist.is_initialized():
        return dist.get_world_size(group), dist.get_rank(group)
    return 1, 0


def _method_id(method) -> int:
    if isinstance(method, int):
        return method
    from . import parse_method
    return parse_method(method)


class GpuBackend:
    """The per-rank work on the current CUDA device, through the C ABI
    (shrk_stieltjes_shard_dev, shrk_stieltjes_batched_dev and the NUFFT
    stage entry points)."""

    def __init__(self):
        import torch
        from . import _native
        self._torch = torch
        self._L = _native.load()
        self._check = _native.check
        self.device = torch.device("cuda", torch.cuda.current_device())

    def _t(self, a):
        return self._torch.as_tensor(np.ascontiguousarray(a, dtype=np.float64),
                                     device=self.device)

    def _stream(self):
        return self._torch.cuda.current_stream(self.device).cuda_stream

    def transform(self, ev, lo, hi, eta, method, precision):
        t = self._t(ev)
        re = self._torch.empty(hi - lo, dtype=self._torch.float64, device=self.device)
        im = self._torch.empty_like(re)
        if hi > lo:
            self._check(self._L.shrk_stieltjes_shard_dev(
                t.data_ptr() + 8 * lo, hi - lo, t.numel(), 1, t.data_ptr(), t.numel(), eta,
                _method_id(method), _PREC[precision], float("nan"), 0, re.data_ptr(),
                im.data_ptr(), self._stream()), "stieltjes_shard_dev")
        return re, im

    def points(self, q, nq_total, ev, eta, method, precision):
        tq, t = self._t(q), self._t(ev)
        re = self._torch.empty(tq.numel(), dtype=self._torch.float64, device=self.device)
        im = self._torch.empty_like(re)
        if tq.numel():
            self._check(self._L.shrk_stieltjes_shard_dev(
                tq.data_ptr(), tq.numel(), nq_total, 0, t.data_ptr(), t.numel(), eta,
                _method_id(method), _PREC[precision], float("nan"), 0, re.data_ptr(),
                im.data_ptr(), self._stream()), "stieltjes_shard_dev")
        return re, im

    def batched(self, values, offsets, etas, precision):
        torch = self._torch
        v = self._t(values)
        o = torch.as_tensor(np.ascontiguousarray(offsets, dtype=np.int64), device=self.device)
        e = self._t(etas)
        re = torch.empty_like(v)
        im = torch.empty_like(v)
        n = o.numel() - 1
        if n > 0:
            self._check(self._L.shrk_stieltjes_batched_dev(
                v.data_ptr(), o.data_ptr(), n, e.data_ptr(), _PREC[precision], re.data_ptr(),
                im.data_ptr(), self._stream()), "stieltjes_batched_dev")
        return re, im

    def nufft_grid(self, first, last, eta):
        import ctypes as C
        m, lo, dx = C.c_int64(), C.c_double(), C.c_double()
        self._check(self._L.shrk_nufft_grid(float(first), float(last), float(eta), C.byref(m),
                                            C.byref(lo), C.byref(dx)), "nufft_grid")
        return int(m.value), lo.value, dx.value

    def nufft_density(self, src, m, lo, dx):
        t = self._t(src)
        dens = self._torch.empty(m, dtype=self._torch.float64, device=self.device)
        self._check(self._L.shrk_nufft_density_dev(t.data_ptr(), t.numel(), m, lo, dx,
                                                   dens.data_ptr(), self._stream()),
                    "nufft_density_dev")
        return dens

    def nufft_eval(self, density, m, lo, dx, eta, q):
        tq = self._t(q)
        d = density.to(self.device, self._torch.float64).contiguous()
        re = self._torch.empty(tq.numel(), dtype=self._torch.float64, device=self.device)
        im = self._torch.empty_like(re)
        if tq.numel():
            self._check(self._L.shrk_nufft_eval_dev(d.data_ptr(), m, lo, dx, eta, tq.data_ptr(),
                                                    tq.numel(), re.data_ptr(), im.data_ptr(),
                                                    self._stream()), "nufft_eval_dev")
        return re, im


def _gather_ranges(parts_re, parts_im, ranges, total, group, device):
    """All-gather of per-rank 1-D pieces whose [lo, hi) ranges every rank
    knows: pad to the widest range, gather, place in rank order."""
    import torch
    import torch.distributed as dist
    world, rank = _world(group)
    width = max(b - a for a, b in ranges)
    buf = torch.zeros(2, max(width, 1), dtype=torch.float64, device=device)
    a, b = ranges[rank]
    buf[0, :b - a] = parts_re
    buf[1, :b - a] = parts_im
    parts = [torch.empty_like(buf) for _ in range(world)]
    dist.all_gather(parts, buf, group=group)
    out_re = torch.empty(total, dtype=torch.float64, device=device)
    out_im = torch.empty_like(out_re)
    for r, part in enumerate(parts):
        a, b = ranges[r]
        out_re[a:b] = part[0, :b - a]
        out_im[a:b] = part[1, :b - a]
    return out_re, out_im


def _f64_vec(a, what):
    v = np.ascontiguousarray(np.asarray(a, dtype=np.float64).ravel())
    if v.size == 0:
        raise ValueError(f"{what} must be non-empty")
    if not np.all(np.isfinite(v)):
        raise ValueError(f"{what} must be finite")
    return v


def _eta(eta, p):
    e = 1.0 / math.sqrt(p) if eta is None else float(eta)
    if not (math.isfinite(e) and e > 0.0):
        raise ValueError("eta must be a positive finite number")
    return e


def stieltjes_transform_sharded(eigenvalues, eta: Optional[float] = None, precision: str = "f64",
                                group=None, gather: bool = True,
                                compute: Optional[Callable] = None, method="blocked",
                                backend=None):
    """All-points transform S(ev_i)/p (compute_all_stieltjes, mod.rs:601-790)
    sharded by targets over the ranks of ``group`` (default: the world).

    ``method``: any method name of ``parse_method`` (default the exact
    "blocked" sums).  Returns ``(re, im)`` for this rank's targets, or for all p
    targets when ``gather`` (assembled in rank order).  ``compute(targets,
    sources, eta) -> raw sums`` replaces the per-rank exact sums (host
    tests); ``backend`` replaces the GPU backend as a whole."""
    import torch

    ev = _f64_vec(eigenvalues, "eigenvalues")
    p = ev.size
    if precision not in _PREC:
        raise ValueError(f"unknown precision '{precision}' (expected 'f64' or 'mixed')")
    eta_v = _eta(eta, p)
    world, rank = _world(group)
    ranges = [shard_range(p, world, r) for r in range(world)]
    lo, hi = ranges[rank]
    if compute is not None:
        if hi > lo:
            re, im = compute(ev[lo:hi], ev, eta_v)
            re = torch.as_tensor(re) / p
            im = torch.as_tensor(im) / p
        else:
            re = im = torch.empty(0, dtype=torch.float64)
    else:
        be = backend or GpuBackend()
        re, im = be.transform(ev, lo, hi, eta_v, method, precision)
    if not gather or world == 1:
        return re, im
    return _gather_ranges(re, im, ranges, p, group, re.device)


def stieltjes_at_points_sharded(queries, eigenvalues, eta: Optional[float] = None,
                                method="blocked", precision: str = "f64", group=None,
                                gather: bool = True, backend=None):
    """RAW sums at query points (compute_stieltjes_at_points, mod.rs:394-494)
    sharded by queries, spectrum and tree replicated: every rank evaluates
    its contiguous shard of the queries with the policies of the whole query
    set.  Returns ``(re, im)`` for this rank's queries, or for all when
    ``gather``."""
    ev = _f64_vec(eigenvalues, "eigenvalues")
    q = np.ascontiguousarray(np.asarray(queries, dtype=np.float64).ravel())
    if not np.all(np.isfinite(q)):
        raise ValueError("queries must be finite")
    if precision not in _PREC:
        raise ValueError(f"unknown precision '{precision}' (expected 'f64' or 'mixed')")
    eta_v = _eta(eta, ev.size)
    world, rank = _world(group)
    ranges = [shard_range(q.size, world, r) for r in range(world)]
    lo, hi = ranges[rank]
    be = backend or GpuBackend()
    re, im = be.points(q[lo:hi], q.size, ev, eta_v, method, precision)
    if not gather or world == 1:
        return re, im
    return _gather_ranges(re, im, ranges, q.size, group, re.device)


def stieltjes_batched_sharded(values, offsets, etas=None, precision: str = "f64", group=None,
                              gather: bool = True, backend=None):
    """Many uneven spectra (spectrum s = values[offsets[s]:offsets[s+1]], at
    etas[s], default 1/sqrt(p_s)) split by spectrum: rank r runs the batched
    launch on the contiguous spectra ``weighted_shard_ranges(p_s^2, world)[r]``.

    Returns ``(re, im, (s_lo, s_hi))``: S/p_s laid out like ``values`` for
    this rank's spectra (their values from offsets[s_lo] on), or for all
    spectra when ``gather`` (then (0, n))."""
    vals = np.ascontiguousarray(np.asarray(values, dtype=np.float64).ravel())
    offs = np.ascontiguousarray(np.asarray(offsets, dtype=np.int64).ravel())
    n = offs.size - 1
    if n < 1 or offs[0] != 0 or offs[-1] != vals.size:
        raise ValueError("offsets must start at 0 and end at len(values)")
    sizes = np.diff(offs)
    if np.any(sizes <= 0):
        raise ValueError("every spectrum must be non-empty")
    if not np.all(np.isfinite(vals)):
        raise ValueError("eigenvalues must be finite")
    if etas is None:
        et = 1.0 / np.sqrt(sizes.astype(np.float64))
    else:
        et = np.broadcast_to(np.asarray(etas, dtype=np.float64), (n,)).copy()
    if not np.all(np.isfinite(et) & (et > 0)):
        raise ValueError("eta must be a positive finite number")
    if precision not in _PREC:
        raise ValueError(f"unknown precision '{precision}' (expected 'f64' or 'mixed')")
    world, rank = _world(group)
    spec = weighted_shard_ranges(sizes.astype(np.float64) ** 2, world)
    s_lo, s_hi = spec[rank]
    be = backend or GpuBackend()
    a, b = int(offs[s_lo]), int(offs[s_hi])
    re, im = be.batched(vals[a:b], offs[s_lo:s_hi + 1] - a, et[s_lo:s_hi], precision)
    if not gather or world == 1:
        return re, im, (s_lo, s_hi)
    ranges = [(int(offs[x]), int(offs[y])) for x, y in spec]
    out_re, out_im = _gather_ranges(re, im, ranges, vals.size, group, re.device)
    return out_re, out_im, (0, n)


def nufft_sharded(eigenvalues, eta: Optional[float] = None, queries=None, group=None,
                  gather: bool = True, backend=None):
    """The coarse-grid NUFFT (nufft.rs:164-220) split by points.

    The grid comes from the first and last entries (caller's order) as in
    the single call.  Rank r splats sources ``shard_range(p, world, r)``; one
    all-reduce sums the m-cell densities; rank r evaluates its shard of the
    queries.  ``queries=None``: the all-points transform S/p at every
    eigenvalue; else RAW sums at the queries.  Returns ``(re, im)`` for this
    rank's points, or for all when ``gather``.  Only the densities' summation
    order differs from the single call (1e-15 of the grid's largest value)."""
    import torch
    import torch.distributed as dist

    ev = _f64_vec(eigenvalues, "eigenvalues")
    p = ev.size
    eta_v = _eta(eta, p)
    all_points = queries is None
    q = ev if all_points else np.ascontiguousarray(np.asarray(queries, dtype=np.float64).ravel())
    if not np.all(np.isfinite(q)):
        raise ValueError("queries must be finite")
    world, rank = _world(group)
    be = backend or GpuBackend()
    m, lo, dx = be.nufft_grid(ev[0], ev[-1], eta_v)
    a, b = shard_range(p, world, rank)
    dens = be.nufft_density(ev[a:b], m, lo, dx)
    if world > 1:
        dist.all_reduce(dens, op=dist.ReduceOp.SUM, group=group)
    ranges = [shard_range(q.size, world, r) for r in range(world)]
    qa, qb = ranges[rank]
    re, im = be.nufft_eval(dens, m, lo, dx, eta_v, q[qa:qb])
    if all_points:
        re = re * (1.0 / p)
        im = im * (1.0 / p)
    if not gather or world == 1:
        return re, im
    return _gather_ranges(re, im, ranges, q.size, group, re.device)
