"""PyTorch autograd over the GPU transform and its hand-written adjoint.

``stieltjes_m(ev, eta=None, precision="f64", method="exact")`` returns

    m_j = (1/p) sum_i 1/(ev_i - z_j),   z_j = ev_j + i*eta,

as a complex128 CUDA tensor, differentiable with respect to ``ev``
(including the dependence of z_j on ev_j).  The forward pass is the
all-points transform (``shrk_stieltjes_all_dev``; m = -conj(S)/p in terms of
the reference's raw sum S(x) = sum_i 1/((x - ev_i) - i*eta), term.rs:26-31);
the backward pass is the adjoint kernel (``shrk_stieltjes_adjoint_dev``),
which recomputes the pair terms instead of storing them.  With a ChebCode
preset as ``method`` both passes use that preset's tree (forward:
``shrk_stieltjes_all_dev`` with the preset; backward:
``shrk_stieltjes_adjoint_treecode_dev``); the gradient is then the treecode
evaluation of the exact adjoint, to the preset's accuracy.  Both run on the
caller's current CUDA stream with device pointers: no host copies.

For a real loss L, PyTorch hands backward the cotangent
g_j = dL/dRe(m_j) + i dL/dIm(m_j); the adjoint returns
dL/dev_k = sum_j (Re g_j dRe m_j/dev_k + Im g_j dIm m_j/dev_k).

There is no CPU path: CPU tensors raise ``ValueError``.
"""
from __future__ import annotations

import math

import torch

from . import _native

_PREC = {"f64": 0, "mixed": 1}
_BLOCKED = 2  # StieltjesMethod::Blocked
_CHEB = {"chebcode": 13, "chebcode_fast": 14, "chebcode_xtreme": 15, "chebcode_balanced": 16}


def _check_input(ev: torch.Tensor) -> None:
    if not isinstance(ev, torch.Tensor):
        raise TypeError("eigenvalues must be a torch.Tensor")
    if not ev.is_cuda:
        raise ValueError("eigenvalues must be a CUDA tensor (there is no CPU path)")
    if ev.dtype != torch.float64:
        raise ValueError("eigenvalues must be float64")
    if ev.dim() != 1 or ev.numel() == 0:
        raise ValueError("eigenvalues must be a non-empty 1-D tensor")


class StieltjesTransform(torch.autograd.Function):
    """m(z_j) at z_j = ev_j + i*eta for every j (see the module docstring)."""

    @staticmethod
    def forward(ctx, ev: torch.Tensor, eta: float, precision: str, method: str = "exact"):
        L = _native.load()
        prec = _PREC[precision]
        mid = _BLOCKED if method == "exact" else _CHEB[method]
        ev_c = ev.detach().contiguous()
        p = ev_c.numel()
        re = torch.empty_like(ev_c)
        im = torch.empty_like(ev_c)
        with torch.cuda.device(ev_c.device):
            stream = torch.cuda.current_stream(ev_c.device).cuda_stream
            st = L.shrk_stieltjes_all_dev(ev_c.data_ptr(), p, eta, mid, prec, float("nan"), 0,
                                          re.data_ptr(), im.data_ptr(), stream)
        _native.check(st, "stieltjes_all_dev")
        ctx.save_for_backward(ev_c)
        ctx.eta = eta
        ctx.prec = prec
        ctx.method = mid
        # S/p -> m = -conj(S)/p
        return torch.complex(-re, im)

    @staticmethod
    def backward(ctx, grad_m: torch.Tensor):
        (ev,) = ctx.saved_tensors
        L = _native.load()
        g = grad_m.to(torch.complex128)
        g_re = g.real.contiguous()
        g_im = g.imag.contiguous()
        grad = torch.empty_like(ev)
        with torch.cuda.device(ev.device):
            stream = torch.cuda.current_stream(ev.device).cuda_stream
            if ctx.method == _BLOCKED:
                st = L.shrk_stieltjes_adjoint_dev(ev.data_ptr(), ev.numel(), ctx.eta,
                                                  g_re.data_ptr(), g_im.data_ptr(), ctx.prec,
                                                  grad.data_ptr(), stream)
            else:
                st = L.shrk_stieltjes_adjoint_treecode_dev(ev.data_ptr(), ev.numel(), ctx.eta,
                                                           g_re.data_ptr(), g_im.data_ptr(),
                                                           ctx.method, grad.data_ptr(), stream)
        _native.check(st, "stieltjes_adjoint_dev")
        return grad, None, None, None


def stieltjes_m(ev: torch.Tensor, eta: float | None = None, precision: str = "f64",
                method: str = "exact") -> torch.Tensor:
    """Differentiable m(z_j), z_j = ev_j + i*eta (eta default 1/sqrt(p));
    method "exact" or a ChebCode preset name."""
    _check_input(ev)
    if precision not in _PREC:
        raise ValueError(f"unknown precision '{precision}' (expected 'f64' or 'mixed')")
    if method != "exact" and method not in _CHEB:
        raise ValueError(f"unknown method '{method}' (expected 'exact' or a chebcode preset)")
    eta_v = 1.0 / math.sqrt(ev.numel()) if eta is None else float(eta)
    if not (math.isfinite(eta_v) and eta_v > 0.0):
        raise ValueError("eta must be a positive finite number")
    return StieltjesTransform.apply(ev, eta_v, precision, method)
