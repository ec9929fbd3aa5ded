#!/usr/bin/env python
"""Benchmark of the B200 Stieltjes-transform hot path.

Workload (default): the exact-kernel scale-up case -- p = 1,000,000
eigenvalues drawn i.i.d. from the Marchenko-Pastur law (c = 0.5,
sigma^2 = 1) by inverse CDF on a 2^20-point grid, sorted, f64 storage,
eta = 1/sqrt(p), all p targets -- with the mixed-precision exact kernel
(FP32 compensated far field, FP64 near field).  One "step" is one full
transform of that spectrum.  Metric: pair evaluations per second
(p_targets * p_sources / t) and ms per transform.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

For N > 1 the driver launches one process per GPU with torch.distributed;
every rank transforms its own spectrum (weak scaling, no data-path
collective), timing is the max over ranks.  ``--impl reference`` times the
reference algorithm's CPU implementation (the C++ restatement of the
crate's parallel route, run with every host thread) on a bounded sample of
the same workload.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "Stieltjes pairs/s & ms @p=50k/1M, mixed vs FP64 at stated err; fwd+adj ms"
UNIT = "pairs/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--spectra", type=int, default=4096,
                    help="batched workload: number of spectra")
    ap.add_argument("--p", type=int, default=None,
                    help="spectrum size (default: the workload's own size)")
    ap.add_argument("--workload", default="exact",
                    choices=["exact", "adjoint", "batched", "chebcode_fast", "chebcode",
                             "chebcode_xtreme", "nufft", "fft5", "clean", "fmm", "deconv"],
                    help="exact (default, the headline): all-points exact transform at p=1M; "
                         "adjoint: the adjoint kernel at p=20000; batched: 4096 uneven "
                         "spectra; chebcode*/nufft/fft5: the method at p=1M on the spiked "
                         "spectrum; clean: clean_covariance_matrix of a p=2048 3-factor "
                         "sample covariance")
    ap.add_argument("--precision", default="mixed", choices=["mixed", "f64"])
    ap.add_argument("--fmm-order", type=int, default=16, help="fmm workload: expansion order")
    ap.add_argument("--fmm-m2l", type=int, default=0, choices=[0, 1],
                    help="fmm workload: 0 = FP64 M2L, 1 = tensor-core M2L (TF32 x3)")
    ap.add_argument("--no-extras", action="store_true", help="skip the secondary measurements")
    ap.add_argument("--cpu-seconds", type=float, default=12.0,
                    help="target duration of one CPU baseline sample")
    return ap.parse_args()


def dist_setup(n_gpus):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


# --------------------------------------------------------------- clocks --
class ClockSampler:
    """Samples nvidia-smi clocks and throttle reasons during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.rows = []
        self.proc = None
        self.thread = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
            return

        def reader():
            for line in self.proc.stdout:
                self.rows.append([x.strip() for x in line.split(",")])

        self.thread = threading.Thread(target=reader, daemon=True)
        self.thread.start()

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        if self.thread:
            self.thread.join(timeout=5)
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in self.rows:
            try:
                sm.append(float(r[1]))
                mx = float(r[2])
            except (ValueError, IndexError):
                continue
            for name, val in zip(names, r[5:9]):
                if val.strip().lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


# ------------------------------------------------------------ reference --
def cpu_isa():
    """x86-64-v3 build of the restatement when the host runs it (hardware
    FMA, as the reference's published native builds have), else the v2 one."""
    from oracle import oracle as O

    return "v3" if O.host_has_v3() else "v2"


def cpu_baseline_sample(ev, eta, seconds, shape="block", isa=None):
    """Time the reference's parallel all-points route (C++ restatement of
    cacheblock.rs:1286-1513 in its loop shape: 32-target blocks x source
    quads, every host thread) on a target sample sized to about `seconds`
    of work; returns pairs/s, the sample size, its time and the threads."""
    from oracle import oracle as O

    O.build()
    isa = isa or cpu_isa()
    p = ev.size
    probe = min(p, 256)
    t0 = time.perf_counter()
    O.tiled_targets(ev[:probe], ev, eta, shape, isa)
    rate = probe * p / max(time.perf_counter() - t0, 1e-6)
    n = int(min(p, max(probe, rate * seconds / p)))
    idx = np.linspace(0, p - 1, n).astype(np.int64)
    t0 = time.perf_counter()
    O.tiled_targets(ev[idx], ev, eta, shape, isa)
    dt = time.perf_counter() - t0
    return n * p / dt, n, dt, O.num_threads()


def cpu_variants(ev, eta, seconds=2.0):
    """Short timings of the restatement's other forms (pairs/s): the
    reference's x86 build target (x86-64-v2, fma() out of line) and one
    accumulation chain per target.  All forms give the same sums."""
    out = {}
    for shape, isa in [("block", "v2"), ("target", "v2"), ("target", cpu_isa())]:
        key = f"{shape}_{isa}"
        if key not in out:
            out[key] = cpu_baseline_sample(ev, eta, seconds, shape, isa)[0]
    return out


def run_reference(args, world, rank):
    from shrinkers_b200 import spectra

    if rank != 0:
        return
    p = args.p
    ev = spectra.config2(p)
    eta = 1.0 / math.sqrt(p)
    vals, samples = [], []
    for i in range(args.warmup + args.steps):
        rate, n, dt, cores = cpu_baseline_sample(ev, eta, args.cpu_seconds / max(1, args.steps))
        if i >= args.warmup:
            vals.append(rate)
            samples.append((n, dt))
    value = float(np.median(vals))
    n, dt = samples[-1]
    ms = p * p / value * 1e3
    isa = cpu_isa()
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": f"exact all-points transform, MP(c=0.5) p={p}, eta=1/sqrt(p)",
                   "p": p, "route": "reference parallel all-points route (tiled full square, "
                                    "32-target blocks x source quads)", "isa": f"x86-64-{isa}"},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port",
                         "sample": f"{n} targets x {p} sources per step ({dt:.1f} s), "
                                   f"x86-64-{isa} build; ms_per_step extrapolated to all p "
                                   "targets",
                         "per_core": value / cores,
                         "variants": cpu_variants(ev, eta)},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ------------------------------------------------------------------ ours --
def run_ours(args, world, rank, local):
    import torch
    import shrinkers_b200 as rk
    from shrinkers_b200 import _native, spectra

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    pg = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=dev)
        pg = dist
    L = _native.load()
    p = args.p
    prec = {"mixed": 1, "f64": 0}[args.precision]
    ev_h = spectra.config2(p, seed=2 + rank)
    eta = 1.0 / math.sqrt(p)
    ev = torch.from_numpy(ev_h).to(dev)
    re = torch.empty(p, dtype=torch.float64, device=dev)
    im = torch.empty_like(re)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)  # > L2
    stream = torch.cuda.current_stream(dev)

    def step(precision=prec, out=(re, im)):
        st = L.shrk_stieltjes_all_dev(ev.data_ptr(), p, eta, 2, precision, float("nan"), 0,
                                      out[0].data_ptr(), out[1].data_ptr(), stream.cuda_stream)
        _native.check(st, "stieltjes_all_dev")

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()

    # ---- device-resident timed region
    L.shrk_timing_reset()
    L.shrk_timing_enable(1)
    clocks = ClockSampler(local)
    if pg:
        pg.barrier()
    torch.cuda.synchronize()
    clocks.start()
    times = []
    for _ in range(args.steps):
        flush.fill_(1.0)  # L2 flush between timed iterations (outside the events)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        step()
        e1.record(stream)
        e1.synchronize()
        times.append(e0.elapsed_time(e1))
    torch.cuda.synchronize()
    if pg:
        pg.barrier()
    clk = clocks.stop()
    launches = int(L.shrk_launch_count())
    L.shrk_timing_enable(0)
    import ctypes as C
    kname = b"pair_sum_mixed" if prec == 1 else b"pair_sum_f64"
    kn, kms = C.c_int64(), C.c_double()
    L.shrk_timing_read(kname, C.byref(kn), C.byref(kms))
    total_ms = float(np.sum(times))
    if pg:
        t = torch.tensor([total_ms], dtype=torch.float64, device=dev)
        pg.all_reduce(t, op=pg.ReduceOp.MAX)
        total_ms = float(t.item())
    ms = total_ms / args.steps
    value = world * p * p / (ms * 1e-3)

    # ---- end-to-end through the public C ABI with host buffers
    ev_pin = torch.from_numpy(ev_h).pin_memory()
    ore = torch.empty(p, dtype=torch.float64).pin_memory()
    oim = torch.empty(p, dtype=torch.float64).pin_memory()
    _D = C.POINTER(C.c_double)

    def e2e_call():
        st = L.shrk_stieltjes_all(C.cast(ev_pin.data_ptr(), _D), p, eta, 2, prec, float("nan"), 0,
                                  C.cast(ore.data_ptr(), _D), C.cast(oim.data_ptr(), _D))
        _native.check(st, "stieltjes_all")

    e2e_call()
    e2e_times = []
    for _ in range(max(2, min(args.steps, 5))):
        t0 = time.perf_counter()
        e2e_call()
        e2e_times.append(time.perf_counter() - t0)
    e2e_s = float(np.mean(e2e_times))
    if pg:
        t = torch.tensor([e2e_s], dtype=torch.float64, device=dev)
        pg.all_reduce(t, op=pg.ReduceOp.MAX)
        e2e_s = float(t.item())
    e2e_value = world * p * p / e2e_s

    extras = {}
    roof = None
    cpu = None
    if rank == 0:
        # ---- roofline of the dominant kernel (library CUDA-event timing)
        f32r, f64r = C.c_double(), C.c_double()
        _native.check(L.shrk_measure_pipe_rates(C.byref(f32r), C.byref(f64r)))
        k_avg_s = kms.value / max(kn.value, 1) * 1e-3
        ops_per_pair = 6.0 if prec == 1 else 7.0
        peak = f32r.value if prec == 1 else f64r.value
        achieved = p * p * ops_per_pair / k_avg_s
        traffic = None
        tpath = os.path.join(ROOT, "profiles", "traffic.json")
        if os.path.exists(tpath):
            traffic = json.load(open(tpath)).get(kname.decode())
        mufu = None
        if prec == 1:  # one MUFU reciprocal per two far-field pairs
            mhz = clk.get("sm_mhz")
            sms = torch.cuda.get_device_properties(dev).multi_processor_count
            rr = 16.0 * sms * mhz * 1e6 if mhz else None
            mufu = {"achieved": 0.5 * p * p / k_avg_s / 1e12,
                    "peak": rr / 1e12 if rr else None, "unit": "T rcp/s",
                    "frac": 0.5 * p * p / k_avg_s / rr if rr else None,
                    "basis": "0.5 MUFU reciprocal per pair (the FP64 near field, ~1 % of the "
                             "pairs here, counted as far) / nominal 16 reciprocals per clock "
                             "per SM x SMs x the SM clock nvidia-smi reports"}
        roof = {"bound": "fp32" if prec == 1 else "fp64", "achieved": achieved / 1e12,
                "peak": peak / 1e12, "unit": "Tops/s", "frac": achieved / peak,
                "xu_pipe": mufu,
                "traffic": traffic, "kernel": kname.decode(),
                "kernel_ms": k_avg_s * 1e3, "kernel_launches": kn.value,
                "basis": (f"{ops_per_pair:g} pipe lane-ops per pair evaluation x p^2 pairs per "
                          "launch / CUDA-event kernel time; peak = measured FMA lane-op rate "
                          "of this GPU (shrk_measure_pipe_rates)")}
        if not args.no_extras:
            extras = secondary(args, L, dev, ev, ev_h, eta, p, stream)
        cpu_rate, n, dt, cores = cpu_baseline_sample(ev_h, eta, args.cpu_seconds)
        cpu = {"value": cpu_rate, "unit": UNIT, "cores": cores, "kind": "port",
               "sample": f"{n} of {p} targets x {p} sources, {dt:.1f} s, reference parallel "
                         "route restated in C++ in its loop shape (32-target blocks x source "
                         f"quads, OpenMP), x86-64-{cpu_isa()} build",
               "per_core": cpu_rate / cores,
               "variants": cpu_variants(ev_h, eta)}
        if "fp64_pairs_per_s" in extras:  # like for like: FP64 GPU kernel vs FP64 CPU route
            extras["fp64_gpu_over_cpu"] = extras["fp64_pairs_per_s"] / cpu_rate

    if pg:
        pg.barrier()
        pg.destroy_process_group()
    if rank != 0:
        return
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32+f64" if prec == 1 else "f64", "data": "synthetic",
        "config": {"workload": f"exact all-points transform, MP(c=0.5) p={p}, eta=1/sqrt(p), "
                               f"{args.precision} kernel",
                   "p": p, "eta": eta, "precision": args.precision,
                   "l2": "flushed between timed iterations (256 MiB write)",
                   "parallelism": f"{world} GPU(s), one transform per GPU"},
        "roofline": roof,
        "cpu_baseline": cpu,
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": 8 * p,
                "d2h_bytes_per_step": 16 * p, "ms_per_step": e2e_s * 1e3},
        "gpu_launches": launches,
        "clocks": clk,
        "extras": extras,
    }
    print(json.dumps(line), flush=True)


METHOD_IDS = {"chebcode": 13, "chebcode_fast": 14, "chebcode_xtreme": 15, "nufft": 11,
              "fft5": 8}
FFT5_FAMILIES = (b"fft5_splat", b"fft5_fft", b"fft5_spectral", b"fft5_interp")
CHEB_PRESETS = {"chebcode": (0.5, 11, 32, False), "chebcode_fast": (1.0, 8, 32, True),
                "chebcode_xtreme": (0.25, 11, 16, False)}


def run_path(args, world, rank, local):
    """One JSON line for a secondary workload: the adjoint, the batched launch,
    a treecode preset or the NUFFT.  Same timing rules as the headline
    (device-resident input, CUDA events on the launching stream, L2 flushed
    between steps, max over ranks); e2e goes through the host-pointer entry
    point; the CPU baseline is the oracle's restatement of the reference's
    parallel route on a bounded sample."""
    import ctypes as C
    import torch
    from shrinkers_b200 import _native, spectra
    from oracle import oracle as O

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    pg = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=dev)
        pg = dist
    L = _native.load()
    stream = torch.cuda.current_stream(dev)
    sp = stream.cuda_stream
    prec = {"mixed": 1, "f64": 0}[args.precision]
    wl = args.workload
    p = args.p
    _D = C.POINTER(C.c_double)
    _I64 = C.POINTER(C.c_int64)

    def dptr(t):
        return C.cast(t.data_ptr(), _D)

    roof = None
    if wl == "adjoint":
        ev_h = spectra.config5(p, seed=5 + rank)
        eta = 1.0 / math.sqrt(p)
        ev = torch.from_numpy(ev_h).to(dev)
        g = torch.randn(2, p, dtype=torch.float64, device=dev,
                        generator=torch.Generator(device=dev).manual_seed(5 + rank))
        out = torch.empty(p, dtype=torch.float64, device=dev)
        units = float(p) * p
        family = b"adjoint_mixed" if prec == 1 else b"adjoint_f64"
        desc = f"adjoint of the all-points transform, MP(c=0.3)+5 spikes p={p}, eta=1/sqrt(p)"

        def step():
            _native.check(L.shrk_stieltjes_adjoint_dev(ev.data_ptr(), p, eta, g[0].data_ptr(),
                                                       g[1].data_ptr(), prec, out.data_ptr(), sp))
        gh = g.cpu().pin_memory()
        evp = torch.from_numpy(ev_h).pin_memory()
        oh = torch.empty(p, dtype=torch.float64).pin_memory()

        def e2e():
            _native.check(L.shrk_stieltjes_adjoint(dptr(evp), p, eta, dptr(gh[0]), dptr(gh[1]),
                                                   prec, dptr(oh)))
        io = (24 * p, 8 * p)

        def cpu():
            w, v = gh[0].numpy(), gh[1].numpy()
            t0 = time.perf_counter()
            O.adjoint_direct(ev_h, eta, w, v)
            dt = time.perf_counter() - t0
            return float(p) * p / dt, f"direct-sum gradient at all {p} points, {dt:.2f} s"
    elif wl == "batched":
        vals, offs, etas = spectra.config4(n_spectra=args.spectra, seed=4 + rank)
        n = offs.size - 1
        bv = torch.from_numpy(vals).to(dev)
        bo = torch.from_numpy(offs).to(dev)
        be = torch.from_numpy(etas).to(dev)
        br = torch.empty_like(bv)
        bi = torch.empty_like(bv)
        units = float(np.sum(np.diff(offs).astype(np.float64) ** 2))
        family = b"batched"
        desc = (f"batched exact transform, {n} spectra, p log-uniform in [256, 16384], "
                f"eta=1/sqrt(p) per spectrum, {args.precision} kernel")

        def step():
            _native.check(L.shrk_stieltjes_batched_dev(bv.data_ptr(), bo.data_ptr(), n,
                                                       be.data_ptr(), prec, br.data_ptr(),
                                                       bi.data_ptr(), sp))
        vp = torch.from_numpy(vals).pin_memory()
        op = torch.from_numpy(offs).pin_memory()
        ep = torch.from_numpy(etas).pin_memory()
        rp = torch.empty(vals.size, dtype=torch.float64).pin_memory()
        ip = torch.empty(vals.size, dtype=torch.float64).pin_memory()

        def e2e():
            _native.check(L.shrk_stieltjes_batched(dptr(vp), C.cast(op.data_ptr(), _I64), n,
                                                   dptr(ep), prec, dptr(rp), dptr(ip)))
        io = (8 * vals.size + 8 * (n + 1) + 8 * n, 16 * vals.size)

        def cpu():
            pairs, t0 = 0.0, time.perf_counter()
            for s_ in range(0, n, max(1, n // 64)):
                a = vals[offs[s_]:offs[s_ + 1]]
                O.compute_all(a, float(etas[s_]), "blocked", parallel=True)
                pairs += float(a.size) ** 2
            dt = time.perf_counter() - t0
            return pairs / dt, f"every {max(1, n // 64)}th spectrum, {dt:.2f} s"
    else:
        ev_h = spectra.config3(p, seed=3 + rank)
        eta = 1.0 / math.sqrt(p)
        ev = torch.from_numpy(ev_h).to(dev)
        xr = torch.empty(p, dtype=torch.float64, device=dev)
        xi = torch.empty_like(xr)
        mid = METHOD_IDS.get(wl, -1)
        units = float(p) * p
        family = {"nufft": b"nufft_splat", "fft5": b"fft5_fft",
                  "chebcode_fast": b"cheb_eval_f32"}.get(wl, b"cheb_eval_f64")
        desc = (f"{wl} all-points transform (tree build / grid included), MP(c=0.1)+20 spikes "
                f"in [3,50] p={p}, eta=1/sqrt(p)")

        if wl == "fmm":
            family = b"fmm_l2p_near"
            desc = (f"fmm (order {args.fmm_order}, M2L {'tensor cores TF32x3' if args.fmm_m2l else 'FP64'}) "
                    f"all-points transform (tree build included), "
                    f"MP(c=0.1)+20 spikes in [3,50] p={p}, eta=1/sqrt(p)")

        def step():
            if wl == "fmm":
                _native.check(L.shrk_stieltjes_fmm_dev(ev.data_ptr(), p, eta, args.fmm_order,
                                                       args.fmm_m2l, xr.data_ptr(), xi.data_ptr(),
                                                       sp))
                return
            _native.check(L.shrk_stieltjes_all_dev(ev.data_ptr(), p, eta, mid, 0, float("nan"),
                                                   0, xr.data_ptr(), xi.data_ptr(), sp))
        evp = torch.from_numpy(ev_h).pin_memory()
        rp = torch.empty(p, dtype=torch.float64).pin_memory()
        ip = torch.empty(p, dtype=torch.float64).pin_memory()

        def e2e():
            if wl == "fmm":
                _native.check(L.shrk_stieltjes_fmm(dptr(evp), p, eta, args.fmm_order,
                                                   args.fmm_m2l, dptr(rp), dptr(ip)))
                return
            _native.check(L.shrk_stieltjes_all(dptr(evp), p, eta, mid, 0, float("nan"), 0,
                                               dptr(rp), dptr(ip)))
        io = (8 * p, 16 * p)

        def cpu():
            t0 = time.perf_counter()
            if wl == "nufft":
                O.nufft_points(ev_h, ev_h, eta, parallel=True)
            elif wl == "fft5":  # the reference's fft5 runs sequentially (fft5.rs:589)
                O.fft5_points(ev_h, ev_h, eta)
            elif wl == "fmm":  # no CPU FMM: the reference's accurate treecode preset
                O.chebcode_points(ev_h, ev_h, eta, 0.25, 11, 16, False, parallel=True)
            else:
                th, nn_, leaf, f32 = CHEB_PRESETS[wl]
                O.chebcode_points(ev_h, ev_h, eta, th, nn_, leaf, f32, parallel=True)
            dt = time.perf_counter() - t0
            return units / dt, f"full transform (tree build / grid included), {dt:.2f} s"

    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()

    def timed_steps():
        times = []
        for _ in range(args.steps):
            flush.fill_(1.0)
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            step()
            e1.record(stream)
            e1.synchronize()
            times.append(e0.elapsed_time(e1))
        torch.cuda.synchronize()
        return times

    # The timed steps run without the library's per-launch event timing (two
    # events per launch cost host time that a launch-bound step would show);
    # a second, instrumented pass gives the per-family kernel times.
    clocks = ClockSampler(local)
    if pg:
        pg.barrier()
    torch.cuda.synchronize()
    n0 = int(L.shrk_launch_count())
    clocks.start()
    times = timed_steps()
    clk = clocks.stop()
    launches = int(L.shrk_launch_count()) - n0
    L.shrk_timing_reset()
    L.shrk_timing_enable(1)
    timed_steps()
    L.shrk_timing_enable(0)
    kn, kms = C.c_int64(), C.c_double()
    L.shrk_timing_read(family, C.byref(kn), C.byref(kms))
    fams = {}
    if wl == "fmm":
        for f in (b"fmm_build", b"fmm_p2m", b"fmm_m2m", b"fmm_top", b"fmm_down", b"fmm_m2l_tc",
                  b"fmm_l2l", b"fmm_l2p_near"):
            n_, ms_ = C.c_int64(), C.c_double()
            L.shrk_timing_read(f, C.byref(n_), C.byref(ms_))
            fams[f.decode()] = (n_.value, ms_.value)
    if wl == "fft5":  # the dominant launch family of the pipeline
        for f in FFT5_FAMILIES:
            n_, ms_ = C.c_int64(), C.c_double()
            L.shrk_timing_read(f, C.byref(n_), C.byref(ms_))
            fams[f.decode()] = (n_.value, ms_.value)
        family = max(FFT5_FAMILIES, key=lambda f: fams[f.decode()][1])
        kn, kms = C.c_int64(fams[family.decode()][0]), C.c_double(fams[family.decode()][1])
    total_ms = float(np.sum(times))
    if pg:
        t = torch.tensor([total_ms], dtype=torch.float64, device=dev)
        pg.all_reduce(t, op=pg.ReduceOp.MAX)
        total_ms = float(t.item())
    ms = total_ms / args.steps
    value = world * units / (ms * 1e-3)
    e2e()
    te = []
    for _ in range(max(2, min(args.steps, 5))):
        t0 = time.perf_counter()
        e2e()
        te.append(time.perf_counter() - t0)
    e2e_s = float(np.mean(te))
    if pg:
        t = torch.tensor([e2e_s], dtype=torch.float64, device=dev)
        pg.all_reduce(t, op=pg.ReduceOp.MAX)
        e2e_s = float(t.item())
    cpu_line = None
    if rank == 0:
        k_s = kms.value / max(kn.value, 1) * 1e-3
        if wl in ("adjoint", "batched") and kn.value:
            f32r, f64r = C.c_double(), C.c_double()
            _native.check(L.shrk_measure_pipe_rates(C.byref(f32r), C.byref(f64r)))
            # adjoint: 15 ops per unordered pair = 7.5 per ordered pair
            ops = (7.5 if wl == "adjoint" else (6.0 if prec == 1 else 7.0))
            peak = f32r.value if prec == 1 else f64r.value
            ach = units * ops / k_s
            roof = {"bound": "fp32" if prec == 1 else "fp64", "achieved": ach / 1e12,
                    "peak": peak / 1e12, "unit": "Tops/s", "frac": ach / peak, "traffic": None,
                    "kernel": family.decode(), "kernel_ms": k_s * 1e3,
                    "basis": f"{ops:g} pipe lane-ops per pair evaluation; peak = measured FMA "
                             "lane-op rate of this GPU"}
        elif wl == "nufft" and kn.value:
            m = O.nufft_grid_size(float(ev_h[-1] - ev_h[0]), eta)
            # every launch family of the call; the roofline is the splat's
            # (its HBM GB/s is the figure asked for), the call's total
            # algorithmic bytes and rate are given beside it
            alg_fam = {"nufft_splat": (8 * p + 16 * m, "8 B per source read + 16 B per "
                                       "grid cell written"),
                       "nufft_fft": (128 * m, "two transforms of two four-step passes: "
                                     "16 B per cell read + 16 B written per pass"),
                       "nufft_spectral": (40 * m, "16+8 B per cell read, 16 B written"),
                       "nufft_interp": (24 * p + 16 * m, "8 B per query read, 16 B written, "
                                        "the grid read once")}
            for f in alg_fam:
                n_, ms_ = C.c_int64(), C.c_double()
                L.shrk_timing_read(f.encode(), C.byref(n_), C.byref(ms_))
                fams[f] = (n_.value, ms_.value)
            alg, basis = alg_fam["nufft_splat"]
            k_s = fams["nufft_splat"][1] / max(1, args.steps) * 1e-3  # the family, per step
            ach = alg / k_s / 1e9
            tr = None
            tpath = os.path.join(ROOT, "profiles", "traffic.json")
            if os.path.exists(tpath):
                tr = json.load(open(tpath)).get("nufft_splat")
            total_alg = sum(v[0] for k_, v in alg_fam.items() if fams[k_][0])
            roof = {"bound": "hbm", "achieved": ach, "peak": _measured_hbm(), "unit": "GB/s",
                    "frac": ach / _measured_hbm(), "traffic": tr, "kernel": "nufft_splat",
                    "kernel_ms": k_s * 1e3, "grid_cells": m,
                    "basis": "splat family (keys + short-run sums, long-run sums, pack: three "
                             "launches) per step: " + basis + "; traffic = DRAM bytes of those "
                             "launches per step (ncu at p = 2^24, scaled by the source count)",
                    "families_ms": {k_: v[1] / max(1, args.steps) for k_, v in fams.items()},
                    "call_algorithmic_bytes": total_alg,
                    "call_gbs": total_alg / (ms * 1e-3) / 1e9}
        elif wl == "fft5" and kn.value:
            m = O.fft5_grid_size(ev_h, eta)
            fam = family.decode()
            alg_step, basis = {
                "fft5_splat": (8 * p + 16 * m, "splat (cell, key, run-sum and pack launches): 8 B per "
                               "source read + 16 B per grid cell written, per step"),
                "fft5_fft": (128 * m, "two transforms of two four-step passes: 16 B per cell "
                             "read + 16 B written per pass, per step"),
                "fft5_spectral": (40 * m, "spectral product: 16+8 B per cell read, 16 B "
                                  "written, per step"),
                "fft5_interp": (24 * p + 16 * m, "interpolation: 8 B per point read, 16 B "
                                "written, the grid read once, per step"),
            }[fam]
            per_step = kn.value / max(1, args.steps)  # launches of the family per step
            alg = alg_step / per_step
            ach = alg / k_s / 1e9
            roof = {"bound": "hbm", "achieved": ach, "peak": _measured_hbm(), "unit": "GB/s",
                    "frac": ach / _measured_hbm(), "traffic": None, "kernel": fam,
                    "kernel_ms": k_s * 1e3, "grid_cells": m, "basis": basis,
                    "families_ms": {k: v[1] / max(1, args.steps) for k, v in fams.items()}}
        if wl == "fmm" and fams:
            roof = {"bound": None, "kernel": "fmm (all families)",
                    "families_ms": {k: v[1] / max(1, args.steps) for k, v in fams.items()},
                    "basis": "no single dominant kernel bound reported; see families_ms"}
        rate, sample = cpu()
        cpu_line = {"value": rate, "unit": UNIT, "cores": O.num_threads(), "kind": "port",
                    "sample": sample}
    if pg:
        pg.barrier()
        pg.destroy_process_group()
    if rank != 0:
        return
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": ("f32+f64" if prec == 1 else "f64")
        if wl in ("adjoint", "batched") else ("f32+f64" if wl == "chebcode_fast" else "f64"),
        "data": "synthetic",
        "config": {"workload": desc, "p": p if wl != "batched" else None,
                   "l2": "flushed between timed iterations (256 MiB)",
                   "parallelism": f"{world} GPU(s), one workload per GPU",
                   "units": "pair evaluations (effective p^2 for the treecode and NUFFT)"},
        "roofline": roof, "cpu_baseline": cpu_line,
        "e2e": {"value": world * units / e2e_s, "unit": UNIT, "h2d_bytes_per_step": io[0],
                "d2h_bytes_per_step": io[1], "ms_per_step": e2e_s * 1e3},
        "gpu_launches": launches, "clocks": clk,
    }
    print(json.dumps(line), flush=True)


def _measured_hbm():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        for k in ("hbm_gbs", "hbm_GBs", "hbm"):
            if k in d:
                return float(d[k])
    except (OSError, ValueError):
        pass
    return 6650.0


def secondary(args, L, dev, ev, ev_h, eta, p, stream):
    """FP64 vs mixed at p (speed + error), p = 50k both kernels, the forward +
    adjoint cost at p = 20k and 200k, the batched launch on 4096 uneven
    spectra, and the treecode presets and NUFFT at p = 1M."""
    import torch
    from shrinkers_b200 import _native, spectra

    def timed(fn, reps):
        fn()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(reps):
            fn()
        e1.record(stream)
        e1.synchronize()
        return e0.elapsed_time(e1) / reps

    out = {}
    r64 = torch.empty(p, dtype=torch.float64, device=dev)
    i64 = torch.empty_like(r64)
    rmx = torch.empty_like(r64)
    imx = torch.empty_like(r64)

    def run(prec, a, b, evt=ev, pp=p, e=eta):
        _native.check(L.shrk_stieltjes_all_dev(evt.data_ptr(), pp, e, 2, prec, float("nan"), 0,
                                               a.data_ptr(), b.data_ptr(), stream.cuda_stream))

    out["fp64_ms"] = timed(lambda: run(0, r64, i64), 2)
    out["mixed_ms"] = timed(lambda: run(1, rmx, imx), 3)
    out["mixed_speedup_vs_fp64"] = out["fp64_ms"] / out["mixed_ms"]
    torch.cuda.synchronize()  # results read back only after every launch has finished
    a64 = torch.complex(r64, i64)
    amx = torch.complex(rmx, imx)
    rel = (torch.abs(amx - a64) / torch.abs(a64)).cpu().numpy()
    out["mixed_vs_fp64_rel_err_median"] = float(np.median(rel))
    out["mixed_vs_fp64_rel_err_max"] = float(np.max(rel))
    out["mixed_pairs_per_s"] = p * p / (out["mixed_ms"] * 1e-3)
    out["fp64_pairs_per_s"] = p * p / (out["fp64_ms"] * 1e-3)
    # p = 50k
    p2 = 50_000
    ev2 = torch.from_numpy(spectra.config2(p2)).to(dev)
    e2 = 1.0 / math.sqrt(p2)
    a = torch.empty(p2, dtype=torch.float64, device=dev)
    b = torch.empty_like(a)
    out["p50k_fp64_ms"] = timed(lambda: run(0, a, b, ev2, p2, e2), 10)
    out["p50k_mixed_ms"] = timed(lambda: run(1, a, b, ev2, p2, e2), 10)
    # forward + adjoint at p = 20k (exact)
    p3 = 20_000
    ev3 = torch.from_numpy(spectra.config5(p3)).to(dev)
    e3 = 1.0 / math.sqrt(p3)
    g = torch.randn(2, p3, dtype=torch.float64, device=dev, generator=torch.Generator(device=dev).manual_seed(5))
    fr = torch.empty(p3, dtype=torch.float64, device=dev)
    fi = torch.empty_like(fr)
    gr = torch.empty_like(fr)
    for prec, name in [(0, "f64"), (1, "mixed")]:
        f_ms = timed(lambda: run(prec, fr, fi, ev3, p3, e3), 10)

        def fa():
            run(prec, fr, fi, ev3, p3, e3)
            _native.check(L.shrk_stieltjes_adjoint_dev(ev3.data_ptr(), p3, e3, g[0].data_ptr(),
                                                       g[1].data_ptr(), prec, gr.data_ptr(),
                                                       stream.cuda_stream))
        fa_ms = timed(fa, 10)
        out[f"p20k_{name}_fwd_ms"] = f_ms
        out[f"p20k_{name}_fwd_adj_ms"] = fa_ms
        out[f"p20k_{name}_fwd_adj_over_fwd"] = fa_ms / f_ms
    # forward + adjoint at p = 200k (exact kernels)
    p4 = 200_000
    ev4 = torch.from_numpy(spectra.config5(p4)).to(dev)
    e4 = 1.0 / math.sqrt(p4)
    g4 = torch.randn(2, p4, dtype=torch.float64, device=dev,
                     generator=torch.Generator(device=dev).manual_seed(5))
    f4r = torch.empty(p4, dtype=torch.float64, device=dev)
    f4i = torch.empty_like(f4r)
    g4o = torch.empty_like(f4r)
    for prec, name in [(0, "f64"), (1, "mixed")]:
        f_ms = timed(lambda: run(prec, f4r, f4i, ev4, p4, e4), 3)
        a_ms = timed(lambda: _native.check(L.shrk_stieltjes_adjoint_dev(
            ev4.data_ptr(), p4, e4, g4[0].data_ptr(), g4[1].data_ptr(), prec, g4o.data_ptr(),
            stream.cuda_stream)), 3)
        out[f"p200k_{name}_fwd_ms"] = f_ms
        out[f"p200k_{name}_adj_ms"] = a_ms
        out[f"p200k_{name}_fwd_adj_over_fwd"] = (f_ms + a_ms) / f_ms
    # batched: 4096 spectra, p log-uniform in [256, 16384], eta = 1/sqrt(p)
    vals, offs, etas = spectra.config4()
    n = offs.size - 1
    bv = torch.from_numpy(vals).to(dev)
    bo = torch.from_numpy(offs).to(dev)
    be = torch.from_numpy(etas).to(dev)
    br = torch.empty_like(bv)
    bi = torch.empty_like(bv)
    out["batched_pairs"] = float(np.sum(np.diff(offs).astype(np.float64) ** 2))
    for prec, name in [(0, "f64"), (1, "mixed")]:
        b_ms = timed(lambda: _native.check(L.shrk_stieltjes_batched_dev(
            bv.data_ptr(), bo.data_ptr(), n, be.data_ptr(), prec, br.data_ptr(), bi.data_ptr(),
            stream.cuda_stream)), 3)
        out[f"batched_{name}_ms"] = b_ms
        out[f"batched_{name}_pairs_per_s"] = out["batched_pairs"] / (b_ms * 1e-3)
    # treecode presets and NUFFT at p = 1M (MP c = 0.1 + 20 spikes in [3, 50]),
    # eta = 1/sqrt(p): whole call on device-resident input (tree build
    # included), error vs the FP64 exact kernel
    # and again at eta = 1e-4 (the workload's second eta)
    p5 = 1_000_000
    ev5 = torch.from_numpy(spectra.config3(p5)).to(dev)
    x5r = torch.empty(p5, dtype=torch.float64, device=dev)
    x5i = torch.empty_like(x5r)
    for e5, tag in [(1.0 / math.sqrt(p5), ""), (1e-4, "_eta1e-4")]:
        run(0, x5r, x5i, ev5, p5, e5)
        torch.cuda.synchronize()
        ex5 = torch.complex(x5r, x5i)
        for name, mid in [("chebcode_fast", 14), ("chebcode", 13), ("chebcode_xtreme", 15),
                          ("nufft", 11)]:
            def call(mid=mid, e5=e5):
                _native.check(L.shrk_stieltjes_all_dev(ev5.data_ptr(), p5, e5, mid, 0,
                                                       float("nan"), 0, x5r.data_ptr(),
                                                       x5i.data_ptr(), stream.cuda_stream))
            ms = timed(call, 5)
            torch.cuda.synchronize()
            rel = torch.abs(torch.complex(x5r, x5i) - ex5) / torch.abs(ex5)
            out[f"p1m_{name}{tag}_ms"] = ms
            out[f"p1m_{name}{tag}_rel_err_median"] = float(rel.median())
            out[f"p1m_{name}{tag}_rel_err_max"] = float(rel.max())
    return out


def run_clean(args, world, rank, local):
    """clean_covariance_matrix (pipeline/mod.rs:273-306) of a p x p sample
    covariance of n = 4p rows with 3 factors.  A step = one call: `value`
    through the device-pointer form (matrix and outputs in HBM), `e2e`
    through the host-pointer C ABI (the p^2 copies included).  Its stages
    are timed by the library's CUDA events (the eigensolver's families,
    the GEMMs, the reconstruction).  The CPU baseline is the reference's
    recommended route for large p restated: a LAPACK eigendecomposition
    (numpy) plus the oracle's clean_eigensystem."""
    import ctypes as C
    import torch
    from shrinkers_b200 import _native
    from oracle import oracle as O

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    pg = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=dev)
        pg = dist
    L = _native.load()
    p = args.p
    n = 4 * p
    rng = np.random.default_rng(17 + rank)
    b = rng.standard_normal((p, 3)) * np.array([6.0, 4.0, 3.0])
    x = rng.standard_normal((n, 3)) @ b.T + rng.standard_normal((n, p))
    cov_h = np.ascontiguousarray(np.cov(x, rowvar=False))
    c = p / n
    pin = lambda shape: torch.empty(shape, dtype=torch.float64).pin_memory().numpy()
    m_in = pin((p, p))
    m_in[:] = cov_h
    o_cov, o_vec, o_ev, o_ov = pin((p, p)), pin((p, p)), pin(p), pin(p)
    s2 = C.c_double()
    _D = C.POINTER(C.c_double)
    dp = lambda a: a.ctypes.data_as(_D)

    d_in = torch.from_numpy(cov_h).to(dev)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)  # > L2
    d_cov = torch.empty(p, p, dtype=torch.float64, device=dev)
    d_vec = torch.empty_like(d_cov)
    d_ev = torch.empty(p, dtype=torch.float64, device=dev)
    d_ov = torch.empty_like(d_ev)
    stream = torch.cuda.current_stream(dev)

    def step():
        _native.check(L.shrk_clean_covariance_matrix_dev(
            d_in.data_ptr(), p, c, 0, d_cov.data_ptr(), d_vec.data_ptr(), d_ev.data_ptr(),
            d_ov.data_ptr(), C.byref(s2), stream.cuda_stream), "clean_covariance_matrix_dev")

    def e2e_step():
        _native.check(L.shrk_clean_covariance_matrix(dp(m_in), p, c, 0, dp(o_cov), dp(o_vec),
                                                     dp(o_ev), dp(o_ov), C.byref(s2)))
    for _ in range(args.warmup):
        step()
        e2e_step()
    torch.cuda.synchronize()
    # timed without the library's per-launch event timing, then one
    # instrumented step for the per-family kernel times
    clocks = ClockSampler(local)
    if pg:
        pg.barrier()
    torch.cuda.synchronize()
    n0 = int(L.shrk_launch_count())
    clocks.start()
    times = []
    for _ in range(args.steps):
        flush.fill_(1.0)  # L2 flush between timed iterations (outside the events)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        step()
        e1.record(stream)
        e1.synchronize()
        times.append(e0.elapsed_time(e1) * 1e-3)
    torch.cuda.synchronize()
    clk = clocks.stop()
    launches = int(L.shrk_launch_count()) - n0
    e2e_times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        e2e_step()
        e2e_times.append(time.perf_counter() - t0)
    L.shrk_timing_reset()
    L.shrk_timing_enable(1)
    for _ in range(args.steps):
        step()
    torch.cuda.synchronize()
    L.shrk_timing_enable(0)
    fams = {}
    for f in (b"eigh_tridiag", b"eigh_bisect", b"eigh_inverse_iteration", b"eigh_orthogonalise",
              b"eigh_back_transform", b"dgemm_wy_yty", b"dgemm_wy_ytz", b"dgemm_wy_tw",
              b"dgemm_wy_update", b"dgemm", b"matrix_reconstruct", b"pair_sum_f64",
              b"split_reduce"):
        kn, kms = C.c_int64(), C.c_double()
        L.shrk_timing_read(f, C.byref(kn), C.byref(kms))
        if kn.value:
            fams[f.decode()] = kms.value / args.steps
    tot = float(np.sum(times))
    tot_e2e = float(np.sum(e2e_times))
    if pg:
        t = torch.tensor([tot, tot_e2e], dtype=torch.float64, device=dev)
        pg.all_reduce(t, op=pg.ReduceOp.MAX)
        tot, tot_e2e = float(t[0].item()), float(t[1].item())
    ms = tot * 1e3 / args.steps
    ms_e2e = tot_e2e * 1e3 / args.steps
    cpu_line = None
    if rank == 0:
        t0 = time.perf_counter()
        w, v = np.linalg.eigh(cov_h)
        O.clean_eigensystem(v, w, c)
        dt = time.perf_counter() - t0
        cpu_line = {"value": 1.0 / dt, "unit": "matrices/s", "cores": os.cpu_count(),
                    "kind": "port", "sample": f"one full cleaning at p={p} (numpy LAPACK eigh on "
                    f"all cores + the oracle's clean_eigensystem), {dt:.2f} s"}
    if pg:
        pg.barrier()
        pg.destroy_process_group()
    if rank != 0:
        return
    rate = world * 1e3 / ms
    line = {
        "metric": "matrix cleanings/s (clean_covariance_matrix)", "value": rate,
        "unit": "matrices/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic",
        "config": {"workload": f"clean_covariance_matrix, p={p}, sample covariance of n={n} rows, "
                               "3 factors (scales 6, 4, 3) + unit noise, c=p/n",
                   "p": p, "parallelism": f"{world} GPU(s), one matrix per GPU",
                   "value_basis": "device-pointer C-ABI call (matrix and outputs in HBM), "
                                  "CUDA events on the caller's stream",
                   "l2": "flushed between timed iterations (256 MiB write)"},
        "roofline": None,
        "stages_ms": fams,
        "cpu_baseline": cpu_line,
        "e2e": {"value": world * 1e3 / ms_e2e, "unit": "matrices/s",
                "h2d_bytes_per_step": 8 * p * p,
                "d2h_bytes_per_step": 16 * p * p + 16 * p + 8, "ms_per_step": ms_e2e},
        "gpu_launches": launches, "clocks": clk,
    }
    print(json.dumps(line), flush=True)


def run_deconv(args, world, rank, local):
    """deconvolve_spiked (hybrid.rs:96-138: BEMA spike detection, inverse BBP,
    El Karoui deconvolution of the bulk on a 200-point grid with the default
    `auto` method, which the reference resolves to chebcode_fast up to
    p = 50 000) through the Python API with host arrays -- the path has no
    device form, so value and e2e both include the copies.  MP(c = 0.25) bulk
    + 3 spikes in [4, 12].  A step = one call at --p; the line also times
    p = 1 000 / 10 000 / 20 000 / 50 000, the sizes the reference publishes
    (docs/internals.md:236-238, 557-564).  The CPU
    baseline is the oracle's restatement of the same call on all host cores."""
    import ctypes as C
    import torch
    import shrinkers_b200 as rk
    from shrinkers_b200 import _native, spectra
    from oracle import oracle as O

    torch.cuda.set_device(local)
    L = _native.load()
    p = args.p
    c = 0.25
    spec = lambda n: spectra.mp_with_spikes(n, c, 3, 4.0, 12.0, seed=n + rank)
    ev = spec(p)
    step = lambda: rk.deconvolve_spiked(ev, c)
    for _ in range(max(args.warmup, 3)):
        step()
    torch.cuda.synchronize()
    n0 = int(L.shrk_launch_count())
    clocks = ClockSampler(local)
    clocks.start()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        step()
    torch.cuda.synchronize()
    ms = (time.perf_counter() - t0) * 1e3 / args.steps
    clk = clocks.stop()
    launches = int(L.shrk_launch_count()) - n0
    sizes = {}
    for n in (1_000, 10_000, 20_000, 50_000):
        e = spec(n)
        for _ in range(5):
            rk.deconvolve_spiked(e, c)
        reps = 200
        t1 = time.perf_counter()
        for _ in range(reps):
            rk.deconvolve_spiked(e, c)
        sizes[str(n)] = (time.perf_counter() - t1) * 1e3 / reps
    cpu_line = None
    if rank == 0 and not args.no_extras:
        O.deconvolve_spiked(ev, c, parallel=True)
        reps, t1 = 0, time.perf_counter()
        while time.perf_counter() - t1 < 2.0:
            O.deconvolve_spiked(ev, c, parallel=True)
            reps += 1
        dt = (time.perf_counter() - t1) / reps
        cpu_line = {"value": 1.0 / dt, "unit": "calls/s", "cores": os.cpu_count(), "kind": "port",
                    "sample": f"{reps} full calls at p={p} (auto -> chebcode_fast grid, "
                              f"parallel route), {dt * 1e3:.3f} ms each"}
    if rank != 0:
        return
    rate = world * 1e3 / ms
    line = {
        "metric": "deconvolve_spiked calls/s (host arrays)", "value": rate, "unit": "calls/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic",
        "config": {"workload": f"deconvolve_spiked(ev, c=0.25), p={p}, n_points=200, method auto, "
                               "MP(c=0.25) + 3 spikes in [4, 12]",
                   "p": p, "parallelism": f"{world} GPU(s), one call stream per GPU",
                   "value_basis": "Python API with host arrays (no device form)",
                   "l2": "inputs of 8p bytes copied in every step"},
        "roofline": None,
        "ms_by_p": sizes,
        "reference_published_ms_m1max": {"1000": 0.0632, "10000": 0.244, "20000": 0.368,
                                          "50000": 0.779},
        "cpu_baseline": cpu_line,
        "e2e": {"value": rate, "unit": "calls/s", "h2d_bytes_per_step": 8 * p + 8 * 200,
                "d2h_bytes_per_step": 48 * 200, "ms_per_step": ms},
        "gpu_launches": launches, "clocks": clk,
    }
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    world, rank, local = dist_setup(args.gpus)
    if args.p is None:
        args.p = {"adjoint": 20_000, "clean": 2048, "deconv": 50_000}.get(args.workload, 1_000_000)
    if args.impl == "reference":
        if args.workload != "exact":
            if rank == 0:
                print(json.dumps({"impl": "reference", "unavailable":
                                  "the reference arm times the headline workload only; "
                                  "secondary workload lines carry their own cpu_baseline"}))
            return
        run_reference(args, world, rank)
        return
    if args.workload == "clean":
        run_clean(args, world, rank, local)
        return
    if args.workload == "deconv":
        run_deconv(args, world, rank, local)
        return
    if args.workload != "exact":
        run_path(args, world, rank, local)
        return
    run_ours(args, world, rank, local)


if __name__ == "__main__":
    main()
