"""Gaussian-process negative log-likelihood through the library's Cholesky.

    loss(A, y) = 1/2 y^T A^{-1} y + sum_i log L_ii,   A = L L^T

per batch item (the constant n/2 log 2 pi is omitted).  L comes from
:class:`~gpumode_cholesky_b200.autograd.CholeskyFunction`, so dLoss/dA flows
through the hand-written adjoint; the triangular solve for alpha = L^{-1} y
and the log-diagonal are ordinary differentiable torch operations.
"""

from __future__ import annotations

import torch

from .autograd import cholesky_differentiable


def gp_nll(a: torch.Tensor, y: torch.Tensor, mode: str | int | None = "auto", bwd_mode: str | int = "bf16x3"):
    """Per-item loss of a batch: ``a`` (batch, n, n) SPD, ``y`` (batch, n); returns (batch,).

    ``mode`` is the forward precision (default "auto": BF16x3 for n > 128).
    """
    l = cholesky_differentiable(a, mode, bwd_mode)
    alpha = torch.linalg.solve_triangular(l, y.unsqueeze(-1), upper=False).squeeze(-1)
    return 0.5 * (alpha * alpha).sum(-1) + torch.log(torch.diagonal(l, dim1=-2, dim2=-1)).sum(-1)


def gp_nll_grad_closed_form(a: torch.Tensor, y: torch.Tensor) -> torch.Tensor:
    """dLoss/dA = 1/2 (A^{-1} - A^{-1} y y^T A^{-1}) in FP64 (reference values for tests)."""
    ad = a.double()
    ainv = torch.linalg.inv(ad)
    v = ainv @ y.double().unsqueeze(-1)
    return 0.5 * (ainv - v @ v.transpose(-1, -2))
