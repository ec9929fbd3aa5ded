"""ctypes binding of libshrinkers_b200.so (the C ABI in include/shrinkers_b200.h).

The shared library is built in-tree by ``shrinkers_b200._build`` (nvcc,
sm_100a).  Loading it never touches the GPU; any compute call on a machine
without a usable CUDA device returns SHRK_ECUDA, which is raised as a
``RuntimeError`` -- there is no CPU fallback.  ``ctypes.CDLL`` releases the
GIL for the duration of every foreign call, which is what gives the module
the reference's GIL-release behaviour (python.rs ``py.detach``).
"""
from __future__ import annotations

import ctypes as C
import os

from . import _build

SHRK_OK, SHRK_EINVAL, SHRK_ECUDA, SHRK_ETIMEOUT, SHRK_ENOTIMPL, SHRK_ENOMEM = range(6)

_D = C.POINTER(C.c_double)
_F = C.POINTER(C.c_float)
_I64 = C.POINTER(C.c_int64)
_SZ = C.c_size_t
_ST = C.c_int
_P = C.c_void_p

# name -> (restype, argtypes).  Must list every symbol of include/shrinkers_b200.h and
# include/shrinkers_b200_diag.h.
SIGNATURES = {
    "shrk_last_error": (_SZ, [C.c_char_p, _SZ]),
    "shrk_version": (C.c_char_p, []),
    "shrk_device_count": (C.c_int, []),
    "shrk_parse_method": (_ST, [C.c_char_p, C.POINTER(C.c_int)]),
    "shrk_method_name": (C.c_char_p, [C.c_int]),
    "shrk_resolve_auto_method": (C.c_int, [C.c_int, C.c_int, _SZ]),
    "shrk_grid_appropriate": (C.c_int, [C.c_int, _SZ, _SZ]),
    "shrk_mixed_near_k": (C.c_double, []),
    "shrk_stream_check": (_ST, [_P]),
    "shrk_stream_release": (_ST, [_P]),
    "shrk_stieltjes_all": (_ST, [_D, _SZ, C.c_double, C.c_int, C.c_int, C.c_double, C.c_int, _D, _D]),
    "shrk_stieltjes_all_dev": (_ST, [_P, _SZ, C.c_double, C.c_int, C.c_int, C.c_double, C.c_int, _P, _P, _P]),
    "shrk_stieltjes_all_f32": (_ST, [_F, _SZ, C.c_float, C.c_int, C.c_double, _F, _F]),
    "shrk_stieltjes_at_points": (_ST, [_D, _SZ, _D, _SZ, C.c_double, C.c_int, C.c_int, C.c_double, C.c_int, _D, _D]),
    "shrk_stieltjes_at_points_dev": (_ST, [_P, _SZ, _P, _SZ, C.c_double, C.c_int, C.c_int, C.c_double, C.c_int, _P, _P, _P]),
    "shrk_stieltjes_at_points_noalloc": (_ST, [_P, _SZ, _P, _SZ, C.c_double, C.c_int, _P, _P, _P]),
    "shrk_stieltjes_with_deriv": (_ST, [_D, _SZ, C.c_double, _D, _D, _D, _D]),
    "shrk_stieltjes_batched": (_ST, [_D, _I64, _SZ, _D, C.c_int, _D, _D]),
    "shrk_stieltjes_batched_dev": (_ST, [_P, _P, _SZ, _P, C.c_int, _P, _P, _P]),
    "shrk_batched_autotune": (_ST, [C.c_int, C.c_int, C.POINTER(C.c_int32)]),
    "shrk_batched_set_tune": (_ST, [C.c_int, C.POINTER(C.c_int32)]),
    "shrk_stieltjes_adjoint": (_ST, [_D, _SZ, C.c_double, _D, _D, C.c_int, _D]),
    "shrk_stieltjes_adjoint_dev": (_ST, [_P, _SZ, C.c_double, _P, _P, C.c_int, _P, _P]),
    "shrk_stieltjes_adjoint_treecode": (_ST, [_D, _SZ, C.c_double, _D, _D, C.c_int, _D]),
    "shrk_stieltjes_adjoint_treecode_dev": (_ST, [_P, _SZ, C.c_double, _P, _P, C.c_int, _P, _P]),
    "shrk_chebcode_evaluate_many": (_ST, [_D, _SZ, _D, _SZ, C.c_int, _D, _D]),
    "shrk_chebcode_evaluate_many_dev": (_ST, [_P, _SZ, _P, _SZ, C.c_int, _P, _P, _P]),
    "shrk_stieltjes_scaled_ray": (_ST, [_D, _SZ, C.c_double, _D, _D]),
    "shrk_stieltjes_scaled_ray_dev": (_ST, [_P, _SZ, C.c_double, _P, _P, _P]),
    "shrk_stieltjes_fmm": (_ST, [_D, _SZ, C.c_double, C.c_int, C.c_int, _D, _D]),
    "shrk_stieltjes_fmm_dev": (_ST, [_P, _SZ, C.c_double, C.c_int, C.c_int, _P, _P, _P]),
    "shrk_stieltjes_fft5_with_options": (_ST, [_D, _SZ, C.c_double, C.c_int, _SZ, C.c_double, C.c_double, _D, _D]),
    "shrk_stieltjes_fft5_with_options_dev": (_ST, [_P, _SZ, C.c_double, C.c_int, _SZ, C.c_double, C.c_double, _P, _P, _P]),
    "shrk_stieltjes_shard_dev": (_ST, [_P, _SZ, _SZ, C.c_int, _P, _SZ, C.c_double, C.c_int, C.c_int,
                                       C.c_double, C.c_int, _P, _P, _P]),
    "shrk_nufft_grid": (_ST, [C.c_double, C.c_double, C.c_double, _I64, _D, _D]),
    "shrk_nufft_density_dev": (_ST, [_P, _SZ, C.c_int64, C.c_double, C.c_double, _P, _P]),
    "shrk_nufft_eval_dev": (_ST, [_P, C.c_int64, C.c_double, C.c_double, C.c_double, _P, _SZ, _P,
                                  _P, _P]),
    "shrk_inverse_nonlinear_shrinkage": (_ST, [_D, _SZ, C.c_double, C.c_int, _D, _D, _D, _D, _D]),
    "shrk_symmetric_eigh": (_ST, [_D, _SZ, _D, _D]),
    "shrk_symmetric_eigh_dev": (_ST, [_P, _SZ, _P, _P, _P]),
    "shrk_clean_covariance_matrix_dev": (_ST, [_P, _SZ, C.c_double, C.c_int, _P, _P, _P, _P, _D,
                                               _P]),
    "shrk_estimate_precision_matrix_dev": (_ST, [_P, _SZ, C.c_double, C.c_int, _P, _P, _P, _P,
                                                 _D, _P]),
    "shrk_clean_eigensystem": (_ST, [_D, _D, _SZ, C.c_double, _D, _D, _D, _D, _D]),
    "shrk_clean_covariance_matrix": (_ST, [_D, _SZ, C.c_double, C.c_int, _D, _D, _D, _D, _D]),
    "shrk_renormalize_to_unit_diagonal": (_ST, [_D, _SZ, _D]),
    "shrk_precision_from_eigensystem": (_ST, [_D, _D, _SZ, C.c_double, C.c_int, _D, _D, _D, _D, _D]),
    "shrk_estimate_precision_matrix": (_ST, [_D, _SZ, C.c_double, C.c_int, _D, _D, _D, _D, _D]),
    "shrk_shrinkage_factor": (C.c_double, [C.c_double] * 4),
    "shrk_inverse_bbp": (C.c_double, [C.c_double] * 3),
    "shrk_bbp_threshold": (C.c_double, [C.c_double] * 2),
    "shrk_mp_median_factor": (C.c_double, [C.c_double]),
    "shrk_detect_spikes_bema": (_ST, [_D, _SZ, C.c_double, C.c_double, C.POINTER(_SZ), _I64, _D, _D]),
    "shrk_ledoit_wolf_shrinkage": (_ST, [_D, _SZ, C.c_double, C.c_int, C.c_int, C.c_int, C.c_double, _D]),
    "shrk_rie_shrinkage": (_ST, [_D, _SZ, C.c_double, C.c_int, C.c_int, C.c_int, _D]),
    "shrk_spectral_deconvolution": (_ST, [_D, _SZ, C.c_double, _SZ, C.c_double, C.c_double, C.c_double, C.c_int, C.c_int, C.c_int, C.c_double, _D]),
    "shrk_estimate_population_eigenvalues": (_ST, [_D, _SZ, C.c_double, C.c_double, C.c_int, C.POINTER(_SZ), _D, _D, _D, _D, _D, _D]),
    "shrk_deconvolve_spiked": (_ST, [_D, _SZ, C.c_double, _SZ, C.c_double, C.c_double, C.c_int, C.c_int, C.c_int, C.c_double, C.POINTER(_SZ), _D, _D, _D, _D, _D]),
    "shrk_timing_enable": (None, [C.c_int]),
    "shrk_timing_reset": (None, []),
    "shrk_timing_read": (_ST, [C.c_char_p, _I64, _D]),
    "shrk_launch_count": (C.c_int64, []),
    "shrk_measure_pipe_rates": (_ST, [_D, _D]),
    "shrk_measure_rcp_bias": (_ST, [_D, _D]),
    "shrk_diag_set_wait_limit": (C.c_longlong, [C.c_longlong]),
    "shrk_diag_dgemm": (_ST, [C.c_int, C.c_int, C.c_int64, C.c_int64, C.c_int64, C.c_double, _P,
                              C.c_int64, _P, C.c_int64, C.c_double, _P, C.c_int64, _P]),
}

_lib = None


def lib_path() -> str:
    return _build.LIB


def load(build_if_missing: bool = True):
    """Load (building first if absent or stale) and bind the library."""
    global _lib
    if _lib is not None:
        return _lib
    path = _build.LIB
    if not os.path.exists(path):
        if not build_if_missing:
            raise RuntimeError(f"libshrinkers_b200.so is missing at {path}")
        _build.build()
    L = C.CDLL(path)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _lib = L
    return L


def last_error() -> str:
    L = load()
    buf = C.create_string_buffer(4096)
    L.shrk_last_error(buf, len(buf))
    return buf.value.decode(errors="replace")


def check(status: int, what: str = "") -> None:
    """Map a shrk_status to the Python exception the reference would raise."""
    if status == SHRK_OK:
        return
    msg = last_error() or what
    if status == SHRK_EINVAL:
        raise ValueError(msg)
    if status == SHRK_ENOTIMPL:
        raise NotImplementedError(msg)
    if status == SHRK_ENOMEM:
        raise MemoryError(msg)
    raise RuntimeError(f"shrinkers_b200 CUDA failure ({what}): {msg}")
