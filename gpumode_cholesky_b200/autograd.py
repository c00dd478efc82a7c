"""Differentiable Cholesky with the library's hand-written adjoint.

``CholeskyFunction.apply(A, mode)`` factors with :func:`cholesky` and, in
backward, maps Lbar = dLoss/dL to Abar = dLoss/dA with
``b2p_potrf_backward``:

    P = Phi(L^T Lbar),   Abar = 1/2 (S + S^T),   S = L^{-T} P L^{-1}

(Phi keeps the lower triangle and halves the diagonal) -- the same adjoint
torch.linalg.cholesky's autograd uses, computed here by the library's
tensor-core products.  The reference has no backward; this is an extension.
"""

from __future__ import annotations

import torch

from . import _lib
from .potrf import _stream_ptr, cholesky, resolve_mode, workspace


def potrf_backward(l: torch.Tensor, lbar: torch.Tensor, mode: str | int = "bf16x3") -> torch.Tensor:
    """Abar for a batch of factors ``l`` and output gradients ``lbar`` (both (batch, n, n) FP32 CUDA)."""
    if l.shape != lbar.shape or l.dim() != 3 or l.shape[-1] != l.shape[-2]:
        raise ValueError("l and lbar must both have shape (batch, n, n)")
    if l.dtype != torch.float32 or lbar.dtype != torch.float32:
        raise TypeError("l and lbar must be float32")
    if not (l.is_cuda and lbar.is_cuda):
        raise RuntimeError("l and lbar must be CUDA tensors: this library has no CPU path")
    l = l.contiguous()
    lbar = lbar.contiguous()
    batch, n, _ = l.shape
    code = resolve_mode(mode, n)
    abar = torch.empty_like(l)
    lib = _lib.load()
    with torch.cuda.device(l.device):
        ws_bytes = lib.b2p_potrf_backward_workspace_size(batch, n)
        ws = workspace(l.device, ws_bytes).data_ptr() if ws_bytes else None
        st = lib.b2p_potrf_backward(
            l.data_ptr(), lbar.data_ptr(), abar.data_ptr(), batch, n, code, ws, ws_bytes, _stream_ptr(l.device)
        )
    _lib.check(st, "b2p_potrf_backward")
    return abar


class CholeskyFunction(torch.autograd.Function):
    """L = chol(A) with the library's forward and hand-written adjoint."""

    @staticmethod
    def forward(ctx, a: torch.Tensor, mode: str | int | None = None, bwd_mode: str | int = "bf16x3"):
        l = cholesky(a, mode=mode)
        ctx.save_for_backward(l)
        ctx.bwd_mode = bwd_mode
        return l

    @staticmethod
    def backward(ctx, lbar: torch.Tensor):
        (l,) = ctx.saved_tensors
        return potrf_backward(l, lbar, ctx.bwd_mode), None, None


def cholesky_differentiable(a: torch.Tensor, mode: str | int | None = None, bwd_mode: str | int = "bf16x3"):
    """Differentiable factorization: ``L`` with gradients through the hand-written adjoint."""
    return CholeskyFunction.apply(a, mode, bwd_mode)
