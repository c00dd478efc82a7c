"""Gaussian-process negative log-likelihood through the library's Cholesky.

    loss(A, y) = 1/2 y^T A^{-1} y + sum_i log L_ii,   A = L L^T

per batch item (the constant n/2 log 2 pi is omitted).  Forward: the
factorization, then ``b2p_gp_nll_forward`` (alpha = L^{-1} y and the loss in
one launch).  Backward: ``b2p_gp_nll_backward`` gives beta = L^{-T} alpha
(= A^{-1} y, so dLoss/dy = beta) and Lbar = dLoss/dL =
tril(-beta alpha^T) + diag(1 / L_ii); the hand-written Cholesky adjoint
(``b2p_potrf_backward``) maps Lbar to dLoss/dA.  No torch solver or
elementwise op runs on this path.
"""

from __future__ import annotations

import torch

from . import _lib
from .autograd import potrf_backward
from .potrf import _stream_ptr, cholesky


def _check(l: torch.Tensor, v: torch.Tensor) -> None:
    if l.dim() != 3 or l.shape[-1] != l.shape[-2] or v.shape != l.shape[:2]:
        raise ValueError("expected l (batch, n, n) and a vector (batch, n)")
    if l.dtype != torch.float32 or v.dtype != torch.float32:
        raise TypeError("expected float32 tensors")
    if not (l.is_cuda and v.is_cuda):
        raise RuntimeError("CUDA tensors required: this library has no CPU path")


def trsv(l: torch.Tensor, b: torch.Tensor, trans: bool = False) -> torch.Tensor:
    """x = L^{-1} b (or L^{-T} b) for a batch of lower factors ``l`` and vectors ``b``."""
    _check(l, b)
    l, b = l.contiguous(), b.contiguous()
    x = torch.empty_like(b)
    with torch.cuda.device(l.device):
        st = _lib.load().b2p_trsv_batched(
            l.data_ptr(), b.data_ptr(), x.data_ptr(), l.shape[0], l.shape[-1], int(trans), _stream_ptr(l.device)
        )
    _lib.check(st, "b2p_trsv_batched")
    return x


def gp_nll_from_factor(l: torch.Tensor, y: torch.Tensor) -> tuple[torch.Tensor, torch.Tensor]:
    """(loss, alpha) from the factor: loss (batch,), alpha = L^{-1} y (batch, n)."""
    _check(l, y)
    l, y = l.contiguous(), y.contiguous()
    alpha = torch.empty_like(y)
    loss = torch.empty(y.shape[0], dtype=torch.float32, device=y.device)
    with torch.cuda.device(l.device):
        st = _lib.load().b2p_gp_nll_forward(
            l.data_ptr(), y.data_ptr(), alpha.data_ptr(), loss.data_ptr(), l.shape[0], l.shape[-1],
            _stream_ptr(l.device),
        )
    _lib.check(st, "b2p_gp_nll_forward")
    return loss, alpha


def gp_nll_lbar(l: torch.Tensor, alpha: torch.Tensor, gloss: torch.Tensor) -> tuple[torch.Tensor, torch.Tensor]:
    """(beta, Lbar) for upstream gradients ``gloss`` (batch,)."""
    _check(l, alpha)
    gloss = gloss.to(torch.float32).contiguous()
    beta = torch.empty_like(alpha)
    lbar = torch.empty_like(l)
    with torch.cuda.device(l.device):
        st = _lib.load().b2p_gp_nll_backward(
            l.data_ptr(), alpha.data_ptr(), gloss.data_ptr(), beta.data_ptr(), lbar.data_ptr(), l.shape[0],
            l.shape[-1], _stream_ptr(l.device),
        )
    _lib.check(st, "b2p_gp_nll_backward")
    return beta, lbar


class GPNLLFunction(torch.autograd.Function):
    """loss(A, y) with the library's factorization, GP kernels and Cholesky adjoint."""

    @staticmethod
    def forward(ctx, a: torch.Tensor, y: torch.Tensor, mode, bwd_mode):
        l = cholesky(a, mode=mode)
        loss, alpha = gp_nll_from_factor(l, y.to(torch.float32))
        ctx.save_for_backward(l, alpha)
        ctx.bwd_mode = bwd_mode
        return loss

    @staticmethod
    def backward(ctx, gloss: torch.Tensor):
        l, alpha = ctx.saved_tensors
        beta, lbar = gp_nll_lbar(l, alpha, gloss)
        abar = potrf_backward(l, lbar, ctx.bwd_mode) if ctx.needs_input_grad[0] else None
        ybar = gloss.to(beta.dtype).unsqueeze(-1) * beta if ctx.needs_input_grad[1] else None
        return abar, ybar, None, None


def gp_nll(a: torch.Tensor, y: torch.Tensor, mode: str | int | None = "fp32", bwd_mode: str | int = "bf16x3"):
    """Per-item loss of a batch: ``a`` (batch, n, n) SPD, ``y`` (batch, n); returns (batch,).

    ``mode`` is the factorization's precision, FP32 by default: kernel
    matrices with a small jitter are ill-conditioned (RBF over 2048 points
    in [0,1]^3 with 1e-4 jitter: condition numbers 2e6-9e6), and the 16-bit
    operand split of BF16x3 ("auto") cannot factor some of them where FP32
    can.  Differentiable in ``a`` and ``y``.
    """
    return GPNLLFunction.apply(a, y, mode, bwd_mode)


def gp_nll_grad_closed_form(a: torch.Tensor, y: torch.Tensor) -> torch.Tensor:
    """dLoss/dA = 1/2 (A^{-1} - A^{-1} y y^T A^{-1}) in FP64 (reference values for tests)."""
    ad = a.double()
    ainv = torch.linalg.inv(ad)
    v = ainv @ y.double().unsqueeze(-1)
    return 0.5 * (ainv - v @ v.transpose(-1, -2))
