"""Differentiable RMSD for PyTorch (CUDA tensors only).

``rmsd(coords, reference)`` returns per-frame RMSD (float64) of
``coords[F, N, 3]`` against ``reference[N_sel, 3]`` after optimal
superposition, through a ``torch.autograd.Function`` whose backward is the
library's hand-written kernel: dRMSD/dx_k = (x_k - x_bar - R^T (y_k - y_bar)) /
(n RMSD), with R re-derived from the QCP eigenvector of the covariance saved by
the forward (16 doubles per frame) rather than stored.  The reference plan has
no gradient; this is an addition.  Calls are issued on torch's current stream.
"""
from __future__ import annotations

from typing import Optional

import torch

from . import _native as N


def _stream() -> int:
    return torch.cuda.current_stream().cuda_stream


class _RefCache:
    """Keeps uploaded references alive per (device, data_ptr, version)."""

    def __init__(self):
        self._key = None
        self._ref = None

    def get(self, ctx: N.Context, ref: torch.Tensor) -> N.Reference:
        key = (ctx.device, ref.data_ptr(), ref._version, tuple(ref.shape))
        if key != self._key:
            r = ref.detach().to(torch.float32).contiguous()
            self._ref = N.Reference(ctx, r.data_ptr(), r.shape[0], r.shape[1], keepalive=r)
            self._key = key
        return self._ref


_cache = _RefCache()


class RmsdFunction(torch.autograd.Function):
    @staticmethod
    def forward(ctx_, coords: torch.Tensor, reference: torch.Tensor, selection: Optional[torch.Tensor]):
        if not coords.is_cuda:
            raise N.WarpMdError(N.WMD_ERR_INVALID_ARG, "coords must be a CUDA tensor")
        if coords.dtype != torch.float32 or coords.dim() != 3 or coords.shape[2] != 3:
            raise N.WarpMdError(N.WMD_ERR_INVALID_ARG, "coords must be float32 with shape (frames, atoms, 3)")
        x = coords.contiguous()
        dev = x.device.index or 0
        ctx = N.context(dev)
        ref = _cache.get(ctx, reference.to(x.device))
        F, n_atoms = x.shape[0], x.shape[1]
        sel = None
        n_sel = ref.n_sel
        if selection is not None:
            sel = selection.to(device=x.device, dtype=torch.int32).contiguous()
            if sel.numel() != n_sel:
                raise N.WarpMdError(N.WMD_ERR_MISMATCH, "selection and reference lengths differ")
        out = torch.empty(F, dtype=torch.float64, device=x.device)
        stats = torch.empty(F, N.FRAME_STATS, dtype=torch.float64, device=x.device)
        ctx.check(ctx.lib.wmd_rmsd_forward(ctx.handle, x.data_ptr(), F, n_atoms, 3,
                                           None if sel is None else sel.data_ptr(), n_sel, ref.handle,
                                           out.data_ptr(), stats.data_ptr(), _stream()))
        ctx_.save_for_backward(x, stats, sel if sel is not None else torch.empty(0, device=x.device))
        ctx_.ref = ref
        ctx_.has_sel = sel is not None
        return out

    @staticmethod
    def backward(ctx_, grad_out: torch.Tensor):
        x, stats, sel = ctx_.saved_tensors
        ref = ctx_.ref
        ctx = N.context(x.device.index or 0)
        F, n_atoms = x.shape[0], x.shape[1]
        # dL/drmsd goes to the kernel as it is (float64, any stride: the
        # broadcast ones of rmsd.sum() have stride 0), without a copy
        g = grad_out
        if g.dtype != torch.float64 or g.device != x.device or g.dim() != 1:
            g = g.to(device=x.device, dtype=torch.float64).reshape(-1)
        # the kernel writes every selected atom of every frame; only atoms
        # outside the selection need zeros
        covers_all = not ctx_.has_sel and ref.n_sel == n_atoms
        grad = torch.empty_like(x) if covers_all else torch.zeros_like(x)
        ctx.check(ctx.lib.wmd_rmsd_backward_f64(ctx.handle, x.data_ptr(), F, n_atoms, 3,
                                                sel.data_ptr() if ctx_.has_sel else None, ref.n_sel, ref.handle,
                                                stats.data_ptr(), g.data_ptr(), g.stride(0), grad.data_ptr(),
                                                _stream()))
        return grad, None, None


def rmsd(coords: torch.Tensor, reference: torch.Tensor, selection: Optional[torch.Tensor] = None) -> torch.Tensor:
    """Per-frame aligned RMSD (float64), differentiable w.r.t. ``coords``."""
    return RmsdFunction.apply(coords, reference, selection)


def rmsd_value_and_grad(coords: torch.Tensor, reference: torch.Tensor, weights: Optional[torch.Tensor] = None,
                        selection: Optional[torch.Tensor] = None, out: Optional[torch.Tensor] = None,
                        grad: Optional[torch.Tensor] = None):
    """Per-frame aligned RMSD (float64) and the gradient of
    sum_f weights[f] * rmsd[f] w.r.t. ``coords`` (float32, shaped like it;
    weights default to 1) in one call, outside autograd.  For dense packed
    frames this is one kernel that reads each frame from DRAM once.  ``out``
    and ``grad`` may be given (contiguous, right shape and dtype) to be
    filled in place, e.g. inside a captured CUDA graph."""
    if not coords.is_cuda or coords.dtype != torch.float32 or coords.dim() != 3 or coords.shape[2] != 3:
        raise N.WarpMdError(N.WMD_ERR_INVALID_ARG, "coords must be a CUDA float32 tensor (frames, atoms, 3)")
    x = coords.detach().contiguous()
    ctx = N.context(x.device.index or 0)
    ref = _cache.get(ctx, reference.to(x.device))
    F, n_atoms = x.shape[0], x.shape[1]
    sel = None
    if selection is not None:
        sel = selection.to(device=x.device, dtype=torch.int32).contiguous()
        if sel.numel() != ref.n_sel:
            raise N.WarpMdError(N.WMD_ERR_MISMATCH, "selection and reference lengths differ")
    w = None
    if weights is not None:
        w = weights.to(device=x.device, dtype=torch.float64)
        if w.dim() != 1 or w.shape[0] != F:
            raise N.WarpMdError(N.WMD_ERR_MISMATCH, "weights must have one entry per frame")
    if out is None:
        out = torch.empty(F, dtype=torch.float64, device=x.device)
    elif out.shape != (F,) or out.dtype != torch.float64 or not out.is_contiguous() or out.device != x.device:
        raise N.WarpMdError(N.WMD_ERR_MISMATCH, "out must be a contiguous float64 vector of one entry per frame")
    covers_all = sel is None and ref.n_sel == n_atoms
    if grad is None:
        grad = torch.empty_like(x) if covers_all else torch.zeros_like(x)
    elif grad.shape != x.shape or grad.dtype != torch.float32 or not grad.is_contiguous() or grad.device != x.device:
        raise N.WarpMdError(N.WMD_ERR_MISMATCH, "grad must be a contiguous float32 tensor shaped like coords")
    elif not covers_all:
        grad.zero_()  # rows of atoms outside the selection are not written
    ctx.check(ctx.lib.wmd_rmsd_value_and_grad(ctx.handle, x.data_ptr(), F, n_atoms, 3,
                                              None if sel is None else sel.data_ptr(), ref.n_sel, ref.handle,
                                              None if w is None else w.data_ptr(), 0 if w is None else w.stride(0),
                                              out.data_ptr(), grad.data_ptr(), _stream()))
    return out, grad


def pairwise(coords: torch.Tensor, metric: str = "rms", mode: str = "i8x3") -> torch.Tensor:
    """All-pairs RMSD matrix of CUDA float32 frames (F, N, 3) -> (F, F) float32."""
    from .plans import _PAIR_MODES

    x = coords.contiguous()
    ctx = N.context(x.device.index or 0)
    F = x.shape[0]
    out = torch.empty(F, F, dtype=torch.float32, device=x.device)
    m = N.PAIR_RMS if metric == "rms" else N.PAIR_NOFIT
    ctx.check(ctx.lib.wmd_pairwise_rmsd(ctx.handle, x.data_ptr(), F, x.shape[1], 3, None, x.shape[1], m,
                                        _PAIR_MODES[mode], out.data_ptr(), _stream()))
    return out
