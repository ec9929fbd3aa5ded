"""TEST INFRASTRUCTURE ONLY: ctypes front-end of the CPU restatement.

The oracle restates the shrinkers crate's Stieltjes-transform algorithms in
C++ (``oracle_*.cpp``, each function citing the reference file:line it
follows) and is used as the parity checker for the CUDA path and as the
timed CPU baseline.  Only ``tests/``, ``__graft_entry__.smoke()`` and the
CPU-baseline leg of ``bench.py`` import this module; the product package
``shrinkers_b200`` never does.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_SO = os.path.join(_HERE, "_build", "liboracle.so")
# The same sources built for x86-64-v3 (hardware FMA, AVX2): identical
# results, used only to time the CPU baseline on an FMA-capable host.
_SO_V3 = os.path.join(_HERE, "_build", "liboracle_v3.so")

# Method identifiers: declaration order of StieltjesMethod (src/config.rs:19-89).
METHODS = [
    "naive", "autovec", "blocked", "blocked_autovec", "blocked_tiled",
    "blocked_windowed", "blocked_hybrid", "adaptive", "fft5", "fft3", "fft2",
    "nufft", "treecode", "chebcode", "chebcode_fast", "chebcode_xtreme",
    "chebcode_balanced", "ewald", "dst", "auto", "hodlr", "speed_auto",
    "accuracy_auto",
]
M = {name: i for i, name in enumerate(METHODS)}

_D = C.POINTER(C.c_double)
_F = C.POINTER(C.c_float)
_I64 = C.POINTER(C.c_int64)
_SZ = C.c_size_t


def build(force: bool = False) -> str:
    """Compile the oracle with its Makefile (idempotent)."""
    if force or not (os.path.exists(_SO) and os.path.exists(_SO_V3)):
        subprocess.run(["make", "-C", _HERE, "-s"], check=True)
    return _SO


_libs = {}


def host_has_v3() -> bool:
    """True when this host's CPU runs x86-64-v3 code (AVX2 + FMA + BMI2)."""
    try:
        with open("/proc/cpuinfo") as f:
            flags = next((ln for ln in f if ln.startswith("flags")), "").split()
    except OSError:
        return False
    return all(x in flags for x in ("avx2", "fma", "bmi2", "movbe"))


def lib_v3():
    """The x86-64-v3 build (same symbols, same results)."""
    return lib(_SO_V3)


def lib(path=None):
    path = path or _SO
    if path not in _libs:
        build()
        L = C.CDLL(path)
        sig = {
            "orc_resolve_auto_method": (C.c_int, [C.c_int, C.c_int, _SZ]),
            "orc_grid_appropriate": (C.c_int, [C.c_int, _SZ, _SZ]),
            "orc_term": (None, [C.c_double, C.c_double, C.c_double, _D, _D]),
            "orc_term_hoisted": (None, [C.c_double, C.c_double, C.c_double, _D, _D]),
            "orc_naive_sum": (None, [C.c_double, _D, _SZ, C.c_double, _D, _D]),
            "orc_autovec_sum": (None, [C.c_double, _D, _SZ, C.c_double, _D, _D]),
            "orc_symmetric_sweep": (None, [_D, _SZ, C.c_double, _D, _D]),
            "orc_tiled_full_square": (None, [_D, _SZ, C.c_double, _D, _D]),
            "orc_blocked_at_points": (None, [_D, _SZ, _D, _SZ, C.c_double, C.c_double, _D, _D]),
            "orc_compute_all": (C.c_int, [_D, _SZ, C.c_double, C.c_int, C.c_double, C.c_int, _D, _D]),
            "orc_compute_at_points": (C.c_int, [_D, _SZ, _D, _SZ, C.c_double, C.c_int, C.c_double, C.c_int, _D, _D]),
            "orc_tiled_targets": (None, [_D, _SZ, _D, _SZ, C.c_double, _D, _D]),
            "orc_tiled_targets_blocked": (None, [_D, _SZ, _D, _SZ, C.c_double, _D, _D]),
            "orc_all_f32": (None, [_F, _SZ, C.c_float, _F, _F]),
            "orc_with_deriv": (None, [_D, _SZ, C.c_double, _D, _D, _D, _D]),
            "orc_truth_points": (None, [_D, _SZ, _D, _SZ, C.c_double, _D, _D]),
            "orc_adjoint_direct": (None, [_D, _SZ, C.c_double, _D, _D, C.POINTER(C.c_long), _SZ, _D]),
            "orc_num_threads": (C.c_int, []),
            "orc_set_num_threads": (None, [C.c_int]),
            "orc_chebcode_points": (None, [_D, _SZ, _D, _SZ, C.c_double, C.c_double, C.c_int, C.c_int, C.c_int, C.c_int, _D, _D]),
            "orc_grid_leaf_cap": (_SZ, [_SZ, _SZ, _SZ, _SZ]),
            "orc_chebtree_export": (_SZ, [_D, _SZ, C.c_int, C.c_double, _SZ, _D, _D, _I64, _I64, C.POINTER(C.c_int32), _D, _D]),
            "orc_nufft_grid_size": (_SZ, [C.c_double, C.c_double]),
            "orc_nufft_points": (None, [_D, _SZ, _D, _SZ, C.c_double, C.c_int, _D, _D]),
            "orc_nufft_grid": (_SZ, [_D, _SZ, C.c_double, _D, _D, _D, _D]),
            "orc_fft": (None, [_D, _SZ, C.c_int]),
            "orc_nufft_geometry": (None, [C.c_double, C.c_double, C.c_double, C.POINTER(_SZ),
                                          _D, _D]),
            "orc_grid_density": (None, [_D, _SZ, _SZ, C.c_double, C.c_double, C.c_int, _D]),
            "orc_grid_eval": (None, [_D, _SZ, C.c_double, C.c_double, C.c_double, C.c_int, _D,
                                     _SZ, _D, _D]),
            "orc_lagrange4": (None, [C.c_double, _D]),
            "orc_lagrange": (None, [C.c_int, C.c_double, _D]),
            "orc_fft5_grid_size": (_SZ, [C.c_double, C.c_double, _SZ, C.c_double, C.c_double, C.c_double]),
            "orc_fft5_points": (C.c_int, [_D, _SZ, _D, _SZ, C.c_double, C.c_int, _SZ, C.c_double, C.c_double, _D, _D]),
            "orc_shrinkage_factor": (C.c_double, [C.c_double] * 4),
            "orc_inverse_bbp": (C.c_double, [C.c_double] * 3),
            "orc_bbp_threshold": (C.c_double, [C.c_double] * 2),
            "orc_mp_median_factor": (C.c_double, [C.c_double]),
            "orc_bema": (_SZ, [_D, _SZ, C.c_double, C.c_double, _I64, _D, _D]),
            "orc_ledoit_wolf": (C.c_int, [_D, _SZ, C.c_double, C.c_int, C.c_int, C.c_double, _D]),
            "orc_rie": (C.c_int, [_D, _SZ, C.c_double, C.c_int, C.c_int, _D]),
            "orc_spectral_deconvolution": (C.c_int, [_D, _SZ, C.c_double, _SZ, C.c_double, C.c_double, C.c_double, C.c_int, C.c_int, C.c_double, _D]),
            "orc_estimate_population": (C.c_int, [_D, _SZ, C.c_double, C.c_double, C.POINTER(_SZ), _D, _D, _D, _D, _D, _D]),
            "orc_deconvolve_spiked": (C.c_int, [_D, _SZ, C.c_double, _SZ, C.c_double, C.c_double, C.c_int, C.c_int, C.c_double, C.POINTER(_SZ), _D, _D, _D, _D, _D]),
            "orc_scaled_ray": (None, [_D, _SZ, C.c_double, _D, _D]),
            "orc_evaluate_many": (None, [_D, _SZ, _D, _SZ, C.c_double, C.c_int, C.c_int, _D, _D]),
            "orc_inverse_shrinkage": (None, [_D, _SZ, C.c_double, C.c_int, _D, _D, _D, _D, _D]),
            "orc_symmetric_eigh": (None, [_D, _SZ, _D, _D]),
            "orc_angular_overlaps": (None, [_D, _SZ, C.c_double, C.c_double, _D]),
            "orc_clean_eigensystem": (C.c_int, [_D, _D, _SZ, C.c_double, _D, _D, _D, _D, _D]),
            "orc_clean_matrix": (C.c_int, [_D, _SZ, C.c_double, C.c_int, _D, _D, _D, _D, _D]),
            "orc_renormalize": (None, [_D, _SZ, _D]),
            "orc_precision_from_eigensystem": (None, [_D, _D, _SZ, C.c_double, C.c_int, _D, _D, _D, _D, _D]),
            "orc_estimate_precision_matrix": (None, [_D, _SZ, C.c_double, C.c_int, _D, _D, _D, _D, _D]),
        }
        for name, (res, args) in sig.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _libs[path] = L
    return _libs[path]


def _d(a):
    return a.ctypes.data_as(_D)


def _arr(x):
    return np.ascontiguousarray(np.asarray(x, dtype=np.float64))


def _nan(x):
    return float("nan") if x is None else float(x)


def method_id(m) -> int:
    return m if isinstance(m, int) else M[m]


def set_threads(n: int) -> None:
    lib().orc_set_num_threads(int(n))


def num_threads() -> int:
    return int(lib().orc_num_threads())


# ----------------------------------------------------------------- exact --
def term(li, lj, eta):
    r, i = C.c_double(), C.c_double()
    lib().orc_term(li, lj, eta, C.byref(r), C.byref(i))
    return r.value, i.value


def naive_sum(x, ev, eta):
    ev = _arr(ev)
    r, i = C.c_double(), C.c_double()
    lib().orc_naive_sum(x, _d(ev), ev.size, eta, C.byref(r), C.byref(i))
    return r.value, i.value


def autovec_sum(x, ev, eta):
    ev = _arr(ev)
    r, i = C.c_double(), C.c_double()
    lib().orc_autovec_sum(x, _d(ev), ev.size, eta, C.byref(r), C.byref(i))
    return r.value, i.value


def symmetric_sweep(ev, eta):
    ev = _arr(ev)
    re, im = np.empty_like(ev), np.empty_like(ev)
    lib().orc_symmetric_sweep(_d(ev), ev.size, eta, _d(re), _d(im))
    return re, im


def tiled_full_square(ev, eta):
    ev = _arr(ev)
    re, im = np.empty_like(ev), np.empty_like(ev)
    lib().orc_tiled_full_square(_d(ev), ev.size, eta, _d(re), _d(im))
    return re, im


def tiled_targets(targets, ev, eta, shape="block", isa="v2"):
    """Parallel all-points route of the reference for a subset of targets (raw).

    shape "block": the reference's loop shape (32-target blocks x source
    quads, cacheblock.rs:1286-1424); "target": one accumulation chain per
    target.  Both give the same sums bit for bit.  isa "v3" runs the
    x86-64-v3 build (same results)."""
    t, ev = _arr(targets), _arr(ev)
    re, im = np.empty_like(t), np.empty_like(t)
    L = lib_v3() if isa == "v3" else lib()
    f = L.orc_tiled_targets_blocked if shape == "block" else L.orc_tiled_targets
    f(_d(t), t.size, _d(ev), ev.size, eta, _d(re), _d(im))
    return re, im


def compute_all(ev, eta, method="blocked", cutoff=None, parallel=False):
    """compute_all_stieltjes (src/stieltjes/mod.rs:601-790), scaled by 1/p."""
    ev = _arr(ev)
    re, im = np.empty_like(ev), np.empty_like(ev)
    st = lib().orc_compute_all(_d(ev), ev.size, eta, method_id(method), _nan(cutoff),
                               int(bool(parallel)), _d(re), _d(im))
    if st:
        raise NotImplementedError(f"oracle does not restate method {method!r}")
    return re, im


def compute_at_points(q, ev, eta, method="blocked", cutoff=None, parallel=False):
    """compute_stieltjes_at_points (src/stieltjes/mod.rs:394-494), raw sums."""
    q, ev = _arr(q), _arr(ev)
    re, im = np.empty_like(q), np.empty_like(q)
    st = lib().orc_compute_at_points(_d(q), q.size, _d(ev), ev.size, eta, method_id(method),
                                     _nan(cutoff), int(bool(parallel)), _d(re), _d(im))
    if st:
        raise NotImplementedError(f"oracle does not restate method {method!r}")
    return re, im


def all_f32(ev, eta):
    ev = np.ascontiguousarray(np.asarray(ev, dtype=np.float32))
    re, im = np.empty_like(ev), np.empty_like(ev)
    lib().orc_all_f32(ev.ctypes.data_as(_F), ev.size, np.float32(eta),
                      re.ctypes.data_as(_F), im.ctypes.data_as(_F))
    return re, im


def with_deriv(ev, eta):
    ev = _arr(ev)
    out = [np.empty_like(ev) for _ in range(4)]
    lib().orc_with_deriv(_d(ev), ev.size, eta, *[_d(o) for o in out])
    return tuple(out)


def truth_points(q, ev, eta):
    """Raw sums in double-double arithmetic (the error-statistics truth)."""
    q, ev = _arr(q), _arr(ev)
    re, im = np.empty_like(q), np.empty_like(q)
    lib().orc_truth_points(_d(q), q.size, _d(ev), ev.size, eta, _d(re), _d(im))
    return re, im


def adjoint_direct(ev, eta, w, v, idx=None):
    ev, w, v = _arr(ev), _arr(w), _arr(v)
    if idx is None:
        n, ip = ev.size, None
    else:
        idxa = np.ascontiguousarray(np.asarray(idx, dtype=np.int64))
        n, ip = idxa.size, idxa.ctypes.data_as(C.POINTER(C.c_long))
    g = np.empty(n)
    lib().orc_adjoint_direct(_d(ev), ev.size, eta, _d(w), _d(v), ip, n, _d(g))
    return g


# --------------------------------------------------------------- chebcode --
PRESETS = {  # src/stieltjes/chebcode.rs:939-972
    "chebcode": (0.5, 11, 32, False),
    "chebcode_fast": (1.0, 8, 32, True),
    "chebcode_xtreme": (0.25, 11, 16, False),
    "chebcode_balanced": (0.55, 11, 32, False),
}


def chebcode_points(q, ev, eta, theta, n, leaf_cap, f32, parallel=True):
    q, ev = _arr(q), _arr(ev)
    re, im = np.empty_like(q), np.empty_like(q)
    lib().orc_chebcode_points(_d(q), q.size, _d(ev), ev.size, eta, theta, n, leaf_cap,
                              int(f32), int(parallel), _d(re), _d(im))
    return re, im


def evaluate_many(ev, etas, theta, n, leaf_cap):
    """ChebCodeBatch::evaluate_many (src/stieltjes/chebcode.rs:1312-1361): RAW
    sums at every eigenvalue for each eta, as (n_eta, p) arrays."""
    ev = _arr(ev)
    et = _arr(etas)
    re = np.empty((et.size, ev.size))
    im = np.empty_like(re)
    lib().orc_evaluate_many(_d(ev), ev.size, _d(et), et.size, theta, n, leaf_cap, _d(re), _d(im))
    return re, im


def grid_leaf_cap(n, p, nq, preset_leaf):
    return int(lib().orc_grid_leaf_cap(n, p, nq, preset_leaf))


def chebtree(sorted_ev, n, theta, leaf_cap):
    s = _arr(sorted_ev)
    L = lib()
    nn = L.orc_chebtree_export(_d(s), s.size, n, theta, leaf_cap, None, None, None, None, None,
                               None, None)
    lo, hi = np.empty(nn), np.empty(nn)
    li, hi_i = np.empty(nn, np.int64), np.empty(nn, np.int64)
    right = np.empty(nn, np.int32)
    nodes, w = np.empty(nn * n), np.empty(nn * n)
    L.orc_chebtree_export(_d(s), s.size, n, theta, leaf_cap, _d(lo), _d(hi),
                          li.ctypes.data_as(_I64), hi_i.ctypes.data_as(_I64),
                          right.ctypes.data_as(C.POINTER(C.c_int32)), _d(nodes), _d(w))
    return dict(lo=lo, hi=hi, lo_idx=li, hi_idx=hi_i, right=right,
                nodes=nodes.reshape(nn, n), w=w.reshape(nn, n))


# ------------------------------------------------------------------ nufft --
def nufft_grid_size(raw_range, eta):
    return int(lib().orc_nufft_grid_size(raw_range, eta))


def nufft_points(q, ev, eta, parallel=False):
    q, ev = _arr(q), _arr(ev)
    re, im = np.empty_like(q), np.empty_like(q)
    lib().orc_nufft_points(_d(q), q.size, _d(ev), ev.size, eta, int(parallel), _d(re), _d(im))
    return re, im


def nufft_grid(ev, eta):
    ev = _arr(ev)
    L = lib()
    raw = float(ev[-1] - ev[0])
    m = nufft_grid_size(raw, eta)
    dens, packed = np.empty(m), np.empty(2 * m)
    lo, dx = C.c_double(), C.c_double()
    L.orc_nufft_grid(_d(ev), ev.size, eta, _d(dens), _d(packed), C.byref(lo), C.byref(dx))
    return dict(m=m, density=dens, packed=packed[0::2] + 1j * packed[1::2], lo=lo.value,
                dx=dx.value)


def nufft_geometry(first, last, eta):
    """nufft.rs:106-126: (m, lo, dx) of the grid of a spectrum whose first
    and last entries are first / last."""
    m, lo, dx = _SZ(), C.c_double(), C.c_double()
    lib().orc_nufft_geometry(float(first), float(last), float(eta), C.byref(m), C.byref(lo),
                             C.byref(dx))
    return int(m.value), lo.value, dx.value


def grid_density(ev, m, lo, dx, order=4):
    """The sequential order-N splat of ev on the grid (m, lo, dx)."""
    ev = _arr(ev)
    out = np.empty(int(m))
    lib().orc_grid_density(_d(ev), ev.size, int(m), float(lo), float(dx), int(order), _d(out))
    return out


def grid_eval(density, m, lo, dx, eta, q, order=4):
    """Convolution of a grid density and interpolation at q: RAW sums."""
    density, q = _arr(density), _arr(q)
    re, im = np.empty_like(q), np.empty_like(q)
    lib().orc_grid_eval(_d(density), int(m), float(lo), float(dx), float(eta), int(order), _d(q),
                        q.size, _d(re), _d(im))
    return re, im


# ------------------------------------------------------------------- fft5 --
def fft5_grid_size(ev, eta, pad_eta_mult=1000.0, pad_range_frac=0.75):
    ev = _arr(ev)
    return int(lib().orc_fft5_grid_size(float(ev[0]), float(ev[-1]), ev.size, eta, pad_eta_mult,
                                        pad_range_frac))


def fft5_points(q, ev, eta, order=8, m=None, pad_eta_mult=1000.0, pad_range_frac=0.75):
    """fft5.rs:559-625: RAW sums of the fft5 grid convolution at q."""
    q, ev = _arr(q), _arr(ev)
    re, im = np.empty_like(q), np.empty_like(q)
    st = lib().orc_fft5_points(_d(q), q.size, _d(ev), ev.size, eta, int(order), int(m or 0),
                               pad_eta_mult, pad_range_frac, _d(re), _d(im))
    if st:
        raise ValueError(f"fft5 oracle: status {st}")
    return re, im


def lagrange(n, t):
    w = np.empty(n)
    lib().orc_lagrange(int(n), float(t), _d(w))
    return w


def fft(x, sign=-1):
    a = np.ascontiguousarray(np.asarray(x, dtype=np.complex128)).copy()
    lib().orc_fft(a.view(np.float64).ctypes.data_as(_D), a.size, int(sign))
    return a


def lagrange4(t):
    w = np.empty(4)
    lib().orc_lagrange4(t, _d(w))
    return w


# -------------------------------------------------------------- consumers --
def shrinkage_factor(li, c, mr, mi):
    return lib().orc_shrinkage_factor(li, c, mr, mi)


def inverse_bbp(lh, gamma, sigma2=1.0):
    return lib().orc_inverse_bbp(lh, gamma, sigma2)


def bbp_threshold(gamma, sigma2):
    return lib().orc_bbp_threshold(gamma, sigma2)


def mp_median_factor(g):
    return lib().orc_mp_median_factor(g)


def bema(sorted_ev, gamma, margin=1.0):
    s = _arr(sorted_ev)
    idx = np.empty(max(s.size, 1), np.int64)
    edge, s2 = C.c_double(), C.c_double()
    k = lib().orc_bema(_d(s), s.size, gamma, margin, idx.ctypes.data_as(_I64), C.byref(edge),
                       C.byref(s2))
    return dict(k=int(k), spike_indices=idx[:k].copy(), bulk_edge=edge.value, sigma2=s2.value)


def ledoit_wolf(ev, c, method="blocked", parallel=False, eta=None):
    ev = _arr(ev)
    out = np.empty_like(ev)
    st = lib().orc_ledoit_wolf(_d(ev), ev.size, c, method_id(method), int(parallel), _nan(eta),
                               _d(out))
    if st:
        raise NotImplementedError(method)
    return out


def rie(ev, c, method="blocked", parallel=False):
    ev = _arr(ev)
    out = np.empty_like(ev)
    st = lib().orc_rie(_d(ev), ev.size, c, method_id(method), int(parallel), _d(out))
    if st:
        raise NotImplementedError(method)
    return out


_DECONV_KEYS = ["lambda_grid", "density", "w_re", "sample_stieltjes_real",
                "sample_stieltjes_imag", "population_stieltjes_real",
                "population_stieltjes_imag"]


def spectral_deconvolution(ev, c, n_points=200, eta=None, lmin=None, lmax=None,
                           method="blocked", parallel=False, cutoff=None):
    ev = _arr(ev)
    out = np.empty(7 * n_points)
    st = lib().orc_spectral_deconvolution(_d(ev), ev.size, c, n_points, _nan(eta), _nan(lmin),
                                          _nan(lmax), method_id(method), int(parallel),
                                          _nan(cutoff), _d(out))
    if st:
        raise NotImplementedError(method)
    o = out.reshape(7, n_points)
    return {k: o[i].copy() for i, k in enumerate(_DECONV_KEYS)}


def estimate_population_eigenvalues(ev, c, margin=1.0):
    ev = _arr(ev)
    p = ev.size
    k = C.c_size_t()
    sp, ss = np.empty(max(p, 1)), np.empty(max(p, 1))
    bp, bs = np.empty(max(p, 1)), np.empty(max(p, 1))
    edge, s2 = C.c_double(), C.c_double()
    st = lib().orc_estimate_population(_d(ev), p, c, margin, C.byref(k), _d(sp), _d(ss),
                                       C.byref(edge), C.byref(s2), _d(bp), _d(bs))
    assert st == 0
    kk = k.value
    return dict(k=kk, spikes=sp[:kk].copy(), spike_sample=ss[:kk].copy(), bulk_edge=edge.value,
                sigma2=s2.value, bulk_population=bp[:p - kk].copy(), bulk_sample=bs[:p - kk].copy())


def deconvolve_spiked(ev, c, n_points=200, eta=None, margin=1.0, method="auto", parallel=False,
                      cutoff=None):
    ev = _arr(ev)
    p = ev.size
    k = C.c_size_t()
    sp, ss = np.empty(max(p, 1)), np.empty(max(p, 1))
    edge, s2 = C.c_double(), C.c_double()
    out = np.empty(7 * n_points)
    st = lib().orc_deconvolve_spiked(_d(ev), p, c, n_points, _nan(eta), margin, method_id(method),
                                     int(parallel), _nan(cutoff), C.byref(k), _d(sp), _d(ss),
                                     C.byref(edge), C.byref(s2), _d(out))
    if st:
        raise NotImplementedError(method)
    kk = k.value
    o = out.reshape(7, n_points)
    return dict(k=kk, spikes=sp[:kk].copy(), spike_sample=ss[:kk].copy(), bulk_edge=edge.value,
                sigma2=s2.value, bulk={key: o[i].copy() for i, key in enumerate(_DECONV_KEYS)})


# ------------------------------------------------------- inverse shrinkage --
def scaled_ray(ev, scale):
    """compute_stieltjes_scaled_ray (src/stieltjes/mod.rs:304-319): RAW sums at
    z_i = ev_i (1 + i scale)."""
    ev = _arr(ev)
    re, im = np.empty_like(ev), np.empty_like(ev)
    lib().orc_scaled_ray(_d(ev), ev.size, scale, _d(re), _d(im))
    return re, im


INVERSE_METHODS = {"qis": 0, "lis": 1, "gis": 2}


def inverse_shrinkage(ev, c, method="qis"):
    """inverse_nonlinear_shrinkage (src/deconvolution/inverse.rs:156-269)."""
    ev = _arr(ev)
    out = [np.empty_like(ev) for _ in range(4)]
    h = C.c_double()
    lib().orc_inverse_shrinkage(_d(ev), ev.size, c, INVERSE_METHODS[method], *[_d(o) for o in out],
                                C.byref(h))
    return dict(precision_eigenvalues=out[0], covariance_eigenvalues=out[1], theta=out[2],
                htheta=out[3], smoothing=h.value)


# ---------------------------------------------------------- matrix front --
def _mat(m):
    return np.ascontiguousarray(np.asarray(m, dtype=np.float64))


def symmetric_eigh(m):
    """pipeline/mod.rs:502-585 (Jacobi): ascending eigenvalues, eigenvector columns."""
    m = _mat(m)
    p = m.shape[0]
    ev, vec = np.empty(p), np.empty((p, p))
    lib().orc_symmetric_eigh(_d(m), p, _d(ev), _d(vec))
    return ev, vec


def angular_overlaps(lambda_rie, c, sigma2):
    l = _arr(lambda_rie)
    out = np.empty_like(l)
    lib().orc_angular_overlaps(_d(l), l.size, c, sigma2, _d(out))
    return out


def _clean_out(p):
    return np.empty((p, p)), np.empty((p, p)), np.empty(p), np.empty(p), C.c_double()


def clean_eigensystem(eigenvectors, eigenvalues, c):
    """pipeline/mod.rs:197-242."""
    v, e = _mat(eigenvectors), _arr(eigenvalues)
    p = e.size
    cov, vec, l, a2, s2 = _clean_out(p)
    lib().orc_clean_eigensystem(_d(v), _d(e), p, c, _d(cov), _d(vec), _d(l), _d(a2), C.byref(s2))
    return dict(covariance=cov, eigenvectors=vec, eigenvalues=l, overlaps=a2, sigma2=s2.value)


def clean_matrix(m, c, renormalize=False):
    """pipeline/mod.rs:244-331 (+ python.rs:729-731)."""
    m = _mat(m)
    p = m.shape[0]
    cov, vec, l, a2, s2 = _clean_out(p)
    lib().orc_clean_matrix(_d(m), p, c, int(renormalize), _d(cov), _d(vec), _d(l), _d(a2),
                           C.byref(s2))
    return dict(covariance=cov, eigenvectors=vec, eigenvalues=l, overlaps=a2, sigma2=s2.value)


def renormalize_to_unit_diagonal(m):
    m = _mat(m)
    out = np.empty_like(m)
    lib().orc_renormalize(_d(m), m.shape[0], _d(out))
    return out


def _prec_out(p):
    return np.empty((p, p)), np.empty((p, p)), np.empty(p), np.empty(p), C.c_double()


def precision_from_eigensystem(eigenvectors, eigenvalues, c, method="qis"):
    """pipeline/mod.rs:409-464."""
    v, e = _mat(eigenvectors), _arr(eigenvalues)
    p = e.size
    om, vec, pe, ce, h = _prec_out(p)
    lib().orc_precision_from_eigensystem(_d(v), _d(e), p, c, INVERSE_METHODS[method], _d(om),
                                         _d(vec), _d(pe), _d(ce), C.byref(h))
    return dict(precision=om, eigenvectors=vec, precision_eigenvalues=pe,
                covariance_eigenvalues=ce, smoothing=h.value)


def estimate_precision_matrix(m, c, method="qis"):
    """pipeline/mod.rs:466-478."""
    m = _mat(m)
    p = m.shape[0]
    om, vec, pe, ce, h = _prec_out(p)
    lib().orc_estimate_precision_matrix(_d(m), p, c, INVERSE_METHODS[method], _d(om), _d(vec),
                                        _d(pe), _d(ce), C.byref(h))
    return dict(precision=om, eigenvectors=vec, precision_eigenvalues=pe,
                covariance_eigenvalues=ce, smoothing=h.value)
