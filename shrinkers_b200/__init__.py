"""shrinkers_b200 -- the shrinkers Stieltjes-transform hot path on NVIDIA B200.

A drop-in for the Python face of the ``shrinkers`` crate (its PyO3 module,
src/python.rs:1048-1071) restricted to the functions that run the empirical
Stieltjes transform and the estimators that consume it:

    stieltjes_transform, stieltjes_transform_with_deriv, deconvolve_spiked,
    estimate_population_eigenvalues, ledoit_wolf_shrinkage,
    shrink_eigenvalues, detect_spikes_bema, inverse_bbp

Same names, keyword arguments, defaults, return dictionaries and error
messages as the reference; the transforms run in hand-written sm_100a CUDA
kernels behind the C ABI of ``include/shrinkers_b200.h``.  Additions with no
reference counterpart: ``precision="mixed"`` (FP32 far field + FP64 near
field), :func:`stieltjes_transform_batched`, :func:`stieltjes_adjoint`, and
the PyTorch autograd binding in :mod:`shrinkers_b200.autograd`.
"""
from __future__ import annotations

import ctypes as C
import math
import numbers

import numpy as np

from . import _native

__version__ = "0.1.0"

__all__ = [
    "stieltjes_transform", "stieltjes_transform_with_deriv", "deconvolve_spiked",
    "estimate_population_eigenvalues", "ledoit_wolf_shrinkage", "shrink_eigenvalues",
    "detect_spikes_bema", "inverse_bbp", "stieltjes_at_points", "stieltjes_transform_batched",
    "stieltjes_adjoint", "parse_method", "method_name", "inverse_nonlinear_shrinkage",
    "stieltjes_scaled_ray", "chebcode_evaluate_many", "stieltjes_fft5_with_options",
    "clean_correlation_matrix", "clean_covariance_matrix", "estimate_precision_matrix",
    "clean_eigensystem", "precision_from_eigensystem", "renormalize_to_unit_diagonal",
    "symmetric_eigh", "stieltjes_fmm",
]

_D = C.POINTER(C.c_double)
_PREC = {"f64": 0, "mixed": 1}
_PAR_SEQ, _PAR_PAR, _PAR_AUTO = 0, 1, 2


def _lib():
    return _native.load()


def _dp(a: np.ndarray):
    """double* to a's data; the caller keeps `a` alive for the call (every
    call site passes a named array)."""
    return C.cast(a.ctypes.data, _D)


# ------------------------------------------------------------ parsing --
class _Inferred:
    pass


INFERRED = "inferred"


def _inferred_f64(value, what: str):
    """InferredF64 extraction (python.rs:97-134): float, None or "inferred"."""
    if isinstance(value, str):
        if value == "inferred":
            return None
        raise ValueError("expected a float, None, or the string 'inferred'")
    if value is None:
        return None
    try:
        return float(value)
    except (TypeError, ValueError):
        raise ValueError("expected a float, None, or the string 'inferred'") from None


def _require_positive_finite(v: float, what: str) -> float:
    """python.rs:146-153."""
    if not (math.isfinite(v) and v > 0.0):
        raise ValueError(f"{what} must be a positive finite number, got {_fmt(v)}")
    return v


def _fmt(v: float) -> str:
    if math.isnan(v):
        return "NaN"
    if math.isinf(v):
        return "inf" if v > 0 else "-inf"
    return repr(float(v))


def _owned_f64_vec(array, what: str = "eigenvalues") -> np.ndarray:
    """python.rs:186-191: a 1-D float64 ndarray, contiguous, copied."""
    if not isinstance(array, np.ndarray) or array.ndim != 1 or array.dtype != np.float64:
        raise TypeError(
            f"argument '{what}': expected a 1-D numpy.ndarray of float64, got "
            f"{type(array).__name__}"
            + (f" of dtype {array.dtype} and ndim {array.ndim}" if isinstance(array, np.ndarray) else ""))
    if not array.flags["C_CONTIGUOUS"]:
        raise ValueError(f"{what} must be contiguous")
    return np.array(array, dtype=np.float64, copy=True)


def _require_finite(ev: np.ndarray, what: str) -> None:
    """python.rs:135-144."""
    if not np.all(np.isfinite(ev)):
        raise ValueError(f"{what} must be finite (found NaN or infinity)")


def _sanitize_positive(ev: np.ndarray, what: str = "eigenvalues") -> None:
    """python.rs:292-308: clamp round-off dust, reject meaningful negatives."""
    if ev.size == 0:
        return
    # a finite sum means every entry is finite (a NaN or infinity makes it
    # non-finite); only an overflowing sum needs the element-wise check
    if not math.isfinite(float(ev.sum())):
        _require_finite(ev, what)
    if float(ev.min()) >= 0.0:
        return
    scale = max(1.0, float(np.max(np.abs(ev))))
    tol = 1e-10 * scale
    neg = np.nonzero(ev < 0.0)[0]
    for i in neg:
        v = float(ev[i])
        if v < -tol:
            raise ValueError(
                f"{what} must be non-negative (found {v}, tolerance {tol:.3e}); "
                "covariance eigenvalues cannot be significantly negative")
        ev[i] = 0.0


def _require_concentration(c) -> float:
    """python.rs:311-318."""
    c = float(c)
    if not math.isfinite(c) or c <= 0.0 or c > 1.0:
        raise ValueError(f"c (concentration ratio p/n) must satisfy 0 < c <= 1, got {_fmt(c)}")
    return c


def _owned_positive_spectrum(array, c) -> tuple[np.ndarray, float]:
    """python.rs:194-199."""
    ev = _owned_f64_vec(array, "eigenvalues")
    _sanitize_positive(ev, "eigenvalues")
    return ev, _require_concentration(c)


def _parse_parallel(parallel) -> int:
    """python.rs:367-373 (Option<bool>; anything else is a TypeError)."""
    if parallel is None:
        return _PAR_AUTO
    if isinstance(parallel, (bool, np.bool_)):
        return _PAR_PAR if bool(parallel) else _PAR_SEQ
    raise TypeError(f"argument 'parallel': '{type(parallel).__name__}' object cannot be "
                    "converted to 'PyBool'")


def parse_method(method: str) -> int:
    """python.rs:321-350 parse_method: every alias of the reference."""
    if not isinstance(method, str):
        raise TypeError(f"argument 'method': '{type(method).__name__}' object cannot be "
                        "converted to 'PyString'")
    out = C.c_int()
    st = _lib().shrk_parse_method(method.encode(), C.byref(out))
    if st != _native.SHRK_OK:
        raise ValueError(f"unknown method '{method}'")
    return out.value


def method_name(method_id: int) -> str:
    return _lib().shrk_method_name(int(method_id)).decode()


def _usize(v, what: str) -> int:
    if isinstance(v, (bool, np.bool_)) or not isinstance(v, numbers.Integral):
        raise TypeError(f"argument '{what}': '{type(v).__name__}' object cannot be "
                        "interpreted as an integer")
    v = int(v)
    if v < 0:
        raise OverflowError(f"argument '{what}': can't convert negative int to unsigned")
    return v


def _cutoff(cutoff) -> float:
    """python.rs:277-284: None/"inferred" disable it (NaN on the ABI)."""
    v = _inferred_f64(cutoff, "cutoff")
    if v is None:
        return float("nan")
    return _require_positive_finite(v, "cutoff ratio")


# --------------------------------------------------------- transforms --
def stieltjes_transform(eigenvalues, eta=INFERRED, method="blocked", precision="f64",
                        cutoff=INFERRED, parallel=False):
    """python.rs:783-837: S(lambda_i)/p for every eigenvalue.

    Returns {"real", "imag"} (float64; float32 for precision="f32"), Im > 0.
    ``precision="mixed"`` selects the B200 mixed-precision exact kernel.
    """
    ev = _owned_f64_vec(eigenvalues, "eigenvalues")
    _require_finite(ev, "eigenvalues")
    if ev.size == 0:
        raise ValueError("eigenvalues must be non-empty")
    p = ev.size
    eta_v = _inferred_f64(eta, "eta")
    eta_v = _require_positive_finite(0.1 / math.sqrt(p) if eta_v is None else eta_v, "eta")
    m = parse_method(method)
    par = _parse_parallel(parallel)
    cut = _cutoff(cutoff)
    L = _lib()
    if precision in ("f64", "mixed"):
        re, im = np.empty(p), np.empty(p)
        st = L.shrk_stieltjes_all(_dp(ev), p, eta_v, m, _PREC[precision], cut, par, _dp(re), _dp(im))
        _native.check(st, "stieltjes_transform")
        return {"real": re, "imag": im}
    if precision == "f32":
        ev32 = ev.astype(np.float32)
        re, im = np.empty(p, np.float32), np.empty(p, np.float32)
        fp = C.POINTER(C.c_float)
        st = L.shrk_stieltjes_all_f32(ev32.ctypes.data_as(fp), p, np.float32(eta_v), m, cut,
                                      re.ctypes.data_as(fp), im.ctypes.data_as(fp))
        _native.check(st, "stieltjes_transform(f32)")
        return {"real": re, "imag": im}
    raise ValueError(f"unknown precision '{precision}' (expected 'f64' or 'f32')")


def stieltjes_transform_with_deriv(eigenvalues, eta=INFERRED):
    """python.rs:758-781: raw value and analytic derivative at every eigenvalue."""
    ev = _owned_f64_vec(eigenvalues, "eigenvalues")
    _require_finite(ev, "eigenvalues")
    if ev.size == 0:
        raise ValueError("eigenvalues must be non-empty")
    p = ev.size
    eta_v = _inferred_f64(eta, "eta")
    eta_v = _require_positive_finite(0.1 / math.sqrt(p) if eta_v is None else eta_v, "eta")
    out = [np.empty(p) for _ in range(4)]
    st = _lib().shrk_stieltjes_with_deriv(_dp(ev), p, eta_v, *[_dp(o) for o in out])
    _native.check(st, "stieltjes_transform_with_deriv")
    return dict(zip(["real", "imag", "deriv_real", "deriv_imag"], out))


def stieltjes_at_points(query_points, eigenvalues, eta, method="blocked", precision="f64",
                        cutoff=None, parallel=False):
    """Raw sums at arbitrary query points (compute_stieltjes_at_points,
    src/stieltjes/mod.rs:394-494; not exported by the reference's module)."""
    q = np.ascontiguousarray(np.asarray(query_points, dtype=np.float64))
    ev = np.ascontiguousarray(np.asarray(eigenvalues, dtype=np.float64))
    re, im = np.empty(q.size), np.empty(q.size)
    st = _lib().shrk_stieltjes_at_points(_dp(q), q.size, _dp(ev), ev.size, float(eta),
                                         parse_method(method), _PREC[precision], _cutoff(cutoff),
                                         _parse_parallel(parallel), _dp(re), _dp(im))
    _native.check(st, "stieltjes_at_points")
    return {"real": re, "imag": im}


def stieltjes_transform_batched(spectra, eta=None, precision="mixed"):
    """Many spectra of uneven length in one persistent launch.

    ``spectra``: a sequence of 1-D float64 arrays, or a tuple
    ``(values, offsets)`` with spectrum s = values[offsets[s]:offsets[s+1]].
    ``eta``: None (1/sqrt(p_s) per spectrum), a float, or one value per
    spectrum.  Returns a list of {"real", "imag"} dicts scaled by 1/p_s.
    """
    if isinstance(spectra, tuple) and len(spectra) == 2 and np.ndim(spectra[1]) == 1 \
            and np.asarray(spectra[1]).dtype.kind in "iu":
        vals = np.ascontiguousarray(np.asarray(spectra[0], dtype=np.float64))
        offs = np.ascontiguousarray(np.asarray(spectra[1], dtype=np.int64))
    else:
        arrs = [np.asarray(s, dtype=np.float64).ravel() for s in spectra]
        offs = np.zeros(len(arrs) + 1, np.int64)
        offs[1:] = np.cumsum([a.size for a in arrs])
        vals = np.ascontiguousarray(np.concatenate(arrs) if arrs else np.empty(0))
    n = offs.size - 1
    sizes = np.diff(offs)
    if n <= 0:
        return []
    if np.any(sizes <= 0):
        raise ValueError("eigenvalues must be non-empty")
    _require_finite(vals, "eigenvalues")
    if eta is None:
        etas = 1.0 / np.sqrt(sizes.astype(np.float64))
    else:
        etas = np.broadcast_to(np.asarray(eta, dtype=np.float64), (n,)).copy()
    for e in etas:
        _require_positive_finite(float(e), "eta")
    etas = np.ascontiguousarray(etas)
    re, im = np.empty(vals.size), np.empty(vals.size)
    st = _lib().shrk_stieltjes_batched(_dp(vals), offs.ctypes.data_as(C.POINTER(C.c_int64)), n,
                                       _dp(etas), _PREC[precision], _dp(re), _dp(im))
    _native.check(st, "stieltjes_transform_batched")
    return [{"real": re[offs[s]:offs[s + 1]], "imag": im[offs[s]:offs[s + 1]]} for s in range(n)]


def stieltjes_adjoint(eigenvalues, g_real, g_imag, eta=None, precision="f64", method="exact"):
    """dL/d lambda for L = sum_j Re(conj(g_j) m_j), m_j = (1/p) sum_i 1/(lambda_i - z_j),
    z_j = lambda_j + i eta (eta default 1/sqrt(p)).  Includes the dependence
    of z_j on lambda_j.  ``method``: "exact" (every pair; ``precision`` f64 or
    mixed) or a ChebCode preset name ("chebcode", "chebcode_xtreme",
    "chebcode_balanced", "chebcode_fast"), whose tree evaluates the source
    sums in FP64."""
    ev = np.ascontiguousarray(np.asarray(eigenvalues, dtype=np.float64))
    gr = np.ascontiguousarray(np.asarray(g_real, dtype=np.float64))
    gi = np.ascontiguousarray(np.asarray(g_imag, dtype=np.float64))
    if ev.size == 0:
        raise ValueError("eigenvalues must be non-empty")
    if gr.shape != ev.shape or gi.shape != ev.shape:
        raise ValueError("cotangents must have the shape of eigenvalues")
    _require_finite(ev, "eigenvalues")
    eta_v = 1.0 / math.sqrt(ev.size) if eta is None else _require_positive_finite(float(eta), "eta")
    grad = np.empty(ev.size)
    if method == "exact":
        st = _lib().shrk_stieltjes_adjoint(_dp(ev), ev.size, eta_v, _dp(gr), _dp(gi),
                                           _PREC[precision], _dp(grad))
    else:
        st = _lib().shrk_stieltjes_adjoint_treecode(_dp(ev), ev.size, eta_v, _dp(gr), _dp(gi),
                                                    parse_method(method), _dp(grad))
    _native.check(st, "stieltjes_adjoint")
    return grad


# ---------------------------------------------------------- estimators --
_BULK_KEYS = ["lambda_grid", "density", "w_re", "sample_stieltjes_real",
              "sample_stieltjes_imag", "population_stieltjes_real",
              "population_stieltjes_imag"]


def deconvolve_spiked(eigenvalues, c, n_points=200, eta=INFERRED, margin=1.0, *, method="auto",
                      parallel=False, cutoff=INFERRED, precision="f64"):
    """python.rs:428-475 deconvolve_spiked (BEMA + inverse BBP + El Karoui)."""
    ev, c = _owned_positive_spectrum(eigenvalues, c)
    n_points = _usize(n_points, "n_points")
    if n_points == 0:
        raise ValueError("n_points must be >= 1")
    margin = _require_positive_finite(float(margin), "margin")
    eta_v = _inferred_f64(eta, "eta")
    eta_arg = float("nan") if eta_v is None else _require_positive_finite(eta_v, "eta")
    m = parse_method(method)
    par = _parse_parallel(parallel)
    cut = _cutoff(cutoff)
    p = ev.size
    k = C.c_size_t()
    sp, ss = np.empty(max(p, 1)), np.empty(max(p, 1))
    edge, s2 = C.c_double(), C.c_double()
    out = np.zeros(7 * n_points)
    st = _lib().shrk_deconvolve_spiked(_dp(ev), p, c, n_points, eta_arg, margin, m,
                                       _PREC[precision], par, cut, C.byref(k), _dp(sp), _dp(ss),
                                       C.byref(edge), C.byref(s2), _dp(out))
    _native.check(st, "deconvolve_spiked")
    kk = int(k.value)
    o = out.reshape(7, n_points)
    if p - kk == 0:
        o = np.zeros((7, 0))
    return {
        "k": kk,
        "spikes": sp[:kk].copy(),
        "spike_sample": ss[:kk].copy(),
        "bulk_edge": float(edge.value),
        "sigma2": float(s2.value),
        "bulk": {key: o[i].copy() for i, key in enumerate(_BULK_KEYS)},
    }


def estimate_population_eigenvalues(eigenvalues, c, margin=1.0, *, precision="f64"):
    """python.rs:974-1000 estimate_population_eigenvalues."""
    ev, c = _owned_positive_spectrum(eigenvalues, c)
    margin = _require_positive_finite(float(margin), "margin")
    p = ev.size
    k = C.c_size_t()
    sp, ss = np.empty(max(p, 1)), np.empty(max(p, 1))
    bp, bs = np.empty(max(p, 1)), np.empty(max(p, 1))
    edge, s2 = C.c_double(), C.c_double()
    st = _lib().shrk_estimate_population_eigenvalues(_dp(ev), p, c, margin, _PREC[precision],
                                                     C.byref(k), _dp(sp), _dp(ss), C.byref(edge),
                                                     C.byref(s2), _dp(bp), _dp(bs))
    _native.check(st, "estimate_population_eigenvalues")
    kk = int(k.value)
    return {
        "k": kk,
        "spikes": sp[:kk].copy(),
        "spike_sample": ss[:kk].copy(),
        "bulk_edge": float(edge.value),
        "sigma2": float(s2.value),
        "bulk_population": bp[:p - kk].copy(),
        "bulk_sample": bs[:p - kk].copy(),
    }


def ledoit_wolf_shrinkage(eigenvalues, c, *, precision="f64"):
    """python.rs:1007-1019: raw Ledoit-Wolf xi (RmtConfig::new: Blocked, sequential)."""
    ev, c = _owned_positive_spectrum(eigenvalues, c)
    out = np.empty(ev.size)
    if ev.size == 0:
        return out
    st = _lib().shrk_ledoit_wolf_shrinkage(_dp(ev), ev.size, c, 2, _PREC[precision], _PAR_SEQ,
                                           float("nan"), _dp(out))
    _native.check(st, "ledoit_wolf_shrinkage")
    return out


_INVERSE = {"qis": 0, "quadratic": 0, "quadratic_inverse": 0,
            "lis": 1, "linear": 1, "linear_inverse": 1,
            "gis": 2, "geometric": 2, "geometric_inverse": 2}


def _parse_inverse_method(method: str) -> int:
    """inverse.rs:98-105 InverseShrinkageMethod::parse (python.rs:353-359)."""
    key = method.lower() if isinstance(method, str) else None
    if key not in _INVERSE:
        raise ValueError(f"unknown inverse shrinkage method '{method}' "
                         "(expected 'qis', 'lis' or 'gis')")
    return _INVERSE[key]


def stieltjes_scaled_ray(eigenvalues, scale):
    """RAW sums at z_i = lambda_i (1 + i*scale) (mod.rs:304-319), as
    {"real", "imag"}; every point has its own eta_i = scale*lambda_i."""
    ev = _owned_f64_vec(eigenvalues, "eigenvalues")
    if ev.size == 0:
        raise ValueError("eigenvalues must be non-empty")
    _require_finite(ev, "eigenvalues")
    s = _require_positive_finite(float(scale), "scale")
    re, im = np.empty(ev.size), np.empty(ev.size)
    _native.check(_lib().shrk_stieltjes_scaled_ray(_dp(ev), ev.size, s, _dp(re), _dp(im)),
                  "stieltjes_scaled_ray")
    return {"real": re, "imag": im}


def stieltjes_fmm(eigenvalues, eta=INFERRED, order=16, m2l="fp64"):
    """The dyadic Chebyshev FMM (no reference counterpart; the reference's
    ChebCode treecode is method="chebcode*"): S(ev_i)/p at every eigenvalue
    as {"real", "imag"}.  order = Chebyshev points per box in [4, 16]; the
    error vs the exact sums goes from ~1e-9 (10) to FP64 round-off (16).
    m2l="tf32x3" runs the M2L stage on the tensor cores (~1e-7 relative)."""
    modes = {"fp64": 0, "tf32x3": 1}
    if m2l not in modes:
        raise ValueError(f"unknown m2l mode {m2l!r} (expected 'fp64' or 'tf32x3')")
    ev = _owned_f64_vec(eigenvalues, "eigenvalues")
    _require_finite(ev, "eigenvalues")
    if ev.size == 0:
        raise ValueError("eigenvalues must be non-empty")
    e = _inferred_f64(eta, "eta")
    e = 0.1 / math.sqrt(ev.size) if e is None else _require_positive_finite(e, "eta")
    re, im = np.empty(ev.size), np.empty(ev.size)
    _native.check(_lib().shrk_stieltjes_fmm(_dp(ev), ev.size, e, int(order), modes[m2l], _dp(re),
                                            _dp(im)), "stieltjes_fmm")
    return {"real": re, "imag": im}


_ORDER = {"linear": 2, "cubic": 4, "quintic": 6, "heptic": 8}


def stieltjes_fft5_with_options(eigenvalues, eta, order="heptic", grid_size=None,
                                pad_eta_mult=1000.0, pad_range_frac=0.75):
    """compute_all_stieltjes_fft5_with_options (fft5.rs:568-590): RAW sums at
    every eigenvalue from the fft5 grid convolution, as {"real", "imag"}.
    order: "linear" / "cubic" / "quintic" / "heptic" (or 2/4/6/8 nodes);
    grid_size: a forced grid of any length up to 2^21, or a power of two up
    to 2^22 (None = dx <= eta/8, m >= 8p);
    padding max(pad_eta_mult*eta, pad_range_frac*range).  The first and last
    entries bound the grid (ascending input expected, as in the reference)."""
    ev = _owned_f64_vec(eigenvalues, "eigenvalues")
    if ev.size == 0:
        raise ValueError("eigenvalues must be non-empty")
    _require_finite(ev, "eigenvalues")
    e = _require_positive_finite(float(eta), "eta")
    n = _ORDER.get(order, order) if isinstance(order, str) else int(order)
    if n not in (2, 4, 6, 8):
        raise ValueError(f"unknown order {order!r}")
    m = 0 if grid_size is None else int(grid_size)
    if m < 0:
        raise ValueError("grid_size must be positive")
    re, im = np.empty(ev.size), np.empty(ev.size)
    _native.check(_lib().shrk_stieltjes_fft5_with_options(_dp(ev), ev.size, e, n, m,
                                                          float(pad_eta_mult),
                                                          float(pad_range_frac), _dp(re),
                                                          _dp(im)),
                  "stieltjes_fft5_with_options")
    return {"real": re, "imag": im}


def chebcode_evaluate_many(eigenvalues, etas, method="chebcode"):
    """ChebCodeBatch::evaluate_many (chebcode.rs:1312-1361): one tree for the
    ChebCode preset ``method``, RAW sums at every eigenvalue for each eta.
    Returns {"real", "imag"} arrays of shape (len(etas), p), input order."""
    ev = _owned_f64_vec(eigenvalues, "eigenvalues")
    if ev.size == 0:
        raise ValueError("eigenvalues must be non-empty")
    _require_finite(ev, "eigenvalues")
    et = np.ascontiguousarray(np.asarray(etas, dtype=np.float64).ravel())
    for e in et:
        _require_positive_finite(float(e), "eta")
    re = np.empty((et.size, ev.size))
    im = np.empty_like(re)
    if et.size:
        _native.check(_lib().shrk_chebcode_evaluate_many(_dp(ev), ev.size, _dp(et), et.size,
                                                         parse_method(method), _dp(re), _dp(im)),
                      "chebcode_evaluate_many")
    return {"real": re, "imag": im}


def inverse_nonlinear_shrinkage(eigenvalues, c, *, method="qis", parallel=False):
    """python.rs:562-591 inverse_nonlinear_shrinkage (Ledoit & Wolf 2022):
    precision-matrix eigenvalues by QIS / LIS / GIS.  Returns
    {"precision_eigenvalues", "covariance_eigenvalues", "smoothing"}."""
    ev, c = _owned_positive_spectrum(eigenvalues, c)
    bad = ev[ev <= 0.0]
    if bad.size:
        raise ValueError("eigenvalues must be strictly positive for inverse shrinkage "
                         f"(found {_fmt(float(bad[0]))})")
    m = _parse_inverse_method(method)
    _parse_parallel(parallel)
    prec, cov = np.empty(ev.size), np.empty(ev.size)
    h = C.c_double()
    _native.check(_lib().shrk_inverse_nonlinear_shrinkage(_dp(ev), ev.size, c, m, _dp(prec),
                                                          _dp(cov), C.byref(h), None, None),
                  "inverse_nonlinear_shrinkage")
    return {"precision_eigenvalues": prec, "covariance_eigenvalues": cov, "smoothing": h.value}


def shrink_eigenvalues(eigenvalues, c, *, method="auto", parallel=False, precision="f64"):
    """python.rs:1021-1042: trace-preserving RIE shrinkage."""
    ev = _owned_f64_vec(eigenvalues, "eigenvalues")
    _require_finite(ev, "eigenvalues")
    c = _require_concentration(c)
    m = parse_method(method)
    par = _parse_parallel(parallel)
    out = np.empty(ev.size)
    if ev.size == 0:
        return out
    st = _lib().shrk_rie_shrinkage(_dp(ev), ev.size, c, m, _PREC[precision], par, _dp(out))
    _native.check(st, "shrink_eigenvalues")
    return out


def detect_spikes_bema(eigenvalues, c, margin=1.0):
    """python.rs:856-874 detect_spikes_bema (host arithmetic, bit-exact)."""
    ev, c = _owned_positive_spectrum(eigenvalues, c)
    ev = np.sort(ev, kind="stable")
    margin = _require_positive_finite(float(margin), "margin")
    k = C.c_size_t()
    idx = np.empty(max(ev.size, 1), np.int64)
    edge, s2 = C.c_double(), C.c_double()
    st = _lib().shrk_detect_spikes_bema(_dp(ev), ev.size, c, margin, C.byref(k),
                                        idx.ctypes.data_as(C.POINTER(C.c_int64)), C.byref(edge),
                                        C.byref(s2))
    _native.check(st, "detect_spikes_bema")
    kk = int(k.value)
    return {"k": kk, "spike_indices": idx[:kk].copy(), "bulk_edge": float(edge.value),
            "sigma2": float(s2.value)}


def _checked_lambda_hat(x: float) -> float:
    """python.rs:155-169."""
    if not math.isfinite(x):
        raise ValueError("lambda_hat must be finite (found NaN or infinity)")
    if x <= 0.0:
        raise ValueError("lambda_hat must be positive (sample spikes cannot be ≤ 0)")
    return x


def inverse_bbp(lambda_hat, c, sigma2=1.0):
    """python.rs:931-942: scalar -> float, 1-D array -> ndarray."""
    c = _require_concentration(c)
    sigma2 = _require_positive_finite(float(sigma2), "sigma2")
    L = _lib()
    if isinstance(lambda_hat, (numbers.Real, np.floating)) and not isinstance(lambda_hat, bool):
        return float(L.shrk_inverse_bbp(_checked_lambda_hat(float(lambda_hat)), c, sigma2))
    try:
        arr = [float(x) for x in np.asarray(lambda_hat, dtype=np.float64).ravel()]
    except (TypeError, ValueError):
        raise ValueError("expected a float or a 1-D array of floats") from None
    return np.array([L.shrk_inverse_bbp(_checked_lambda_hat(x), c, sigma2) for x in arr])


# ------------------------------------------------------- matrix front-end --
def _owned_symmetric_matrix(matrix, what: str) -> np.ndarray:
    """python.rs:220-249: a square, finite, symmetric float64 matrix (copied,
    row-major); symmetry within 1e-12 of the largest magnitude (at least 1)."""
    if not isinstance(matrix, np.ndarray) or matrix.ndim != 2 or matrix.dtype != np.float64:
        raise TypeError(f"argument '{what}': expected a 2-D numpy.ndarray of float64")
    rows, cols = matrix.shape
    if rows != cols:
        raise ValueError(f"{what} must be a square matrix")
    a = np.array(matrix, dtype=np.float64, order="C", copy=True)
    if not np.all(np.isfinite(a)):
        raise ValueError(f"{what} must contain only finite values")
    tol = 1e-12 * max(1.0, float(np.max(np.abs(a)))) if a.size else 0.0
    if np.any(np.abs(np.triu(a, 1) - np.triu(a.T, 1)) > tol):
        raise ValueError(f"{what} must be symmetric")
    if rows == 0:
        raise ValueError(f"{what} must be non-empty")
    return a


def _clean_dict(p):
    return (np.empty((p, p)), np.empty((p, p)), np.empty(p), np.empty(p), C.c_double())


def _clean_matrix(matrix, what, c, renormalize):
    a = _owned_symmetric_matrix(matrix, what)
    c = _require_concentration(c)
    p = a.shape[0]
    cov, vec, ev, ov, s2 = _clean_dict(p)
    _native.check(_lib().shrk_clean_covariance_matrix(_dp(a), p, c, int(bool(renormalize)),
                                                      _dp(cov), _dp(vec), _dp(ev), _dp(ov),
                                                      C.byref(s2)), f"clean {what}")
    return {"covariance": cov, "eigenvectors": vec, "eigenvalues": ev, "overlaps": ov,
            "sigma2": s2.value}


def clean_correlation_matrix(correlation, c, *, renormalize=False):
    """python.rs:683-741 clean_correlation_matrix (pipeline/mod.rs:308-329):
    RIE eigenvalue shrinkage + eigenvector angular-overlap correction.
    Returns {"covariance", "eigenvectors" (columns, descending), "eigenvalues"
    (RIE, descending), "overlaps", "sigma2"}; renormalize=True rescales the
    result to unit diagonal."""
    return _clean_matrix(correlation, "correlation", c, renormalize)


def clean_covariance_matrix(covariance, c):
    """python.rs:647-681 clean_covariance_matrix (pipeline/mod.rs:273-306):
    the same estimator as clean_correlation_matrix, in covariance units."""
    return _clean_matrix(covariance, "covariance", c, False)


def estimate_precision_matrix(covariance, c, *, method="qis", parallel=False):
    """python.rs:593-645 estimate_precision_matrix (pipeline/mod.rs:466-478):
    inverse nonlinear shrinkage of the eigenvalues, Omega = U diag(w) U^T.
    Returns {"precision", "eigenvectors", "precision_eigenvalues",
    "covariance_eigenvalues", "smoothing"}."""
    a = _owned_symmetric_matrix(covariance, "covariance")
    c = _require_concentration(c)
    m = _parse_inverse_method(method)
    _parse_parallel(parallel)
    p = a.shape[0]
    om, vec = np.empty((p, p)), np.empty((p, p))
    pe, ce, h = np.empty(p), np.empty(p), C.c_double()
    _native.check(_lib().shrk_estimate_precision_matrix(_dp(a), p, c, m, _dp(om), _dp(vec),
                                                        _dp(pe), _dp(ce), C.byref(h)),
                  "estimate_precision_matrix")
    return {"precision": om, "eigenvectors": vec, "precision_eigenvalues": pe,
            "covariance_eigenvalues": ce, "smoothing": h.value}


def _eigensystem(eigenvectors, eigenvalues):
    v = np.ascontiguousarray(np.asarray(eigenvectors, dtype=np.float64))
    e = np.ascontiguousarray(np.asarray(eigenvalues, dtype=np.float64).ravel())
    if v.ndim != 2 or v.shape != (e.size, e.size) or e.size == 0:
        raise ValueError("eigenvectors must be a non-empty p x p matrix parallel to eigenvalues")
    if not (np.all(np.isfinite(v)) and np.all(np.isfinite(e))):
        raise ValueError("eigensystem must contain only finite values")
    return v, e


def clean_eigensystem(eigenvectors, eigenvalues, c):
    """pipeline/mod.rs:197-242 clean_eigensystem (the reference's Rust entry
    point for an eigensystem computed elsewhere): same keys as
    clean_correlation_matrix."""
    v, e = _eigensystem(eigenvectors, eigenvalues)
    c = _require_concentration(c)
    p = e.size
    cov, vec, ev, ov, s2 = _clean_dict(p)
    _native.check(_lib().shrk_clean_eigensystem(_dp(v), _dp(e), p, c, _dp(cov), _dp(vec),
                                                _dp(ev), _dp(ov), C.byref(s2)),
                  "clean_eigensystem")
    return {"covariance": cov, "eigenvectors": vec, "eigenvalues": ev, "overlaps": ov,
            "sigma2": s2.value}


def precision_from_eigensystem(eigenvectors, eigenvalues, c, *, method="qis"):
    """pipeline/mod.rs:409-464 precision_from_eigensystem: same keys as
    estimate_precision_matrix."""
    v, e = _eigensystem(eigenvectors, eigenvalues)
    c = _require_concentration(c)
    m = _parse_inverse_method(method)
    p = e.size
    om, vec = np.empty((p, p)), np.empty((p, p))
    pe, ce, h = np.empty(p), np.empty(p), C.c_double()
    _native.check(_lib().shrk_precision_from_eigensystem(_dp(v), _dp(e), p, c, m, _dp(om),
                                                         _dp(vec), _dp(pe), _dp(ce), C.byref(h)),
                  "precision_from_eigensystem")
    return {"precision": om, "eigenvectors": vec, "precision_eigenvalues": pe,
            "covariance_eigenvalues": ce, "smoothing": h.value}


def renormalize_to_unit_diagonal(matrix):
    """pipeline/mod.rs:331-341: D^-1/2 S D^-1/2 (S unchanged when a diagonal
    entry is not positive)."""
    a = np.ascontiguousarray(np.asarray(matrix, dtype=np.float64))
    if a.ndim != 2 or a.shape[0] != a.shape[1] or a.shape[0] == 0:
        raise ValueError("matrix must be a non-empty square matrix")
    out = np.empty_like(a)
    _native.check(_lib().shrk_renormalize_to_unit_diagonal(_dp(a), a.shape[0], _dp(out)),
                  "renormalize_to_unit_diagonal")
    return out


def symmetric_eigh(matrix):
    """pipeline/mod.rs:502-585 symmetric_eigh on the GPU (this library's eigensolver):
    (ascending eigenvalues, eigenvectors as columns)."""
    a = _owned_symmetric_matrix(matrix, "matrix")
    p = a.shape[0]
    ev, vec = np.empty(p), np.empty((p, p))
    _native.check(_lib().shrk_symmetric_eigh(_dp(a), p, _dp(ev), _dp(vec)), "symmetric_eigh")
    return ev, vec
