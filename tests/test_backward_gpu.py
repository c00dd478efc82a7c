"""GPU: the hand-written Cholesky adjoint.

Checks b2p_potrf_backward against (1) the golden FP64 torch-autograd
gradients, (2) the FP64 oracle adjoint, (3) torch.linalg.cholesky autograd
on the same inputs and (4) the closed-form GP gradient.  Tolerance: relative
Frobenius error <= 5e-4 for BF16x3 products (the adjoint amplifies operand
rounding by the condition of L) and <= 5e-3 for TF32.
"""

from __future__ import annotations

import numpy as np
import pytest
import torch

import oracle
from gpumode_cholesky_b200 import cholesky, cholesky_differentiable, gp_nll, inputs, potrf_backward
from gpumode_cholesky_b200.gp import gp_nll_grad_closed_form

pytestmark = pytest.mark.gpu

TOL = {"bf16x3": 5e-4, "tf32": 5e-3}


def _rel(x, y):
    x = np.asarray(x, dtype=np.float64)
    y = np.asarray(y, dtype=np.float64)
    return float(np.linalg.norm(x - y) / max(np.linalg.norm(y), 1e-30))


@pytest.mark.parametrize("mode", ["bf16x3", "tf32"])
def test_adjoint_matches_golden_autograd(golden_backward, mode):
    for g in golden_backward:
        l = torch.from_numpy(g["l"]).float().cuda()
        lbar = torch.from_numpy(g["lbar"]).float().cuda()
        abar = potrf_backward(l, lbar, mode).cpu().numpy()
        assert np.isfinite(abar).all()
        assert _rel(abar, g["abar"]) <= TOL[mode], (g["l"].shape, _rel(abar, g["abar"]))


@pytest.mark.parametrize("batch,n", [(5, 17), (4, 64), (3, 100), (2, 127), (2, 257), (2, 512)])
def test_adjoint_matches_oracle(batch, n):
    a = inputs.well_conditioned(batch, n, seed=n, device="cpu")
    l = cholesky(a.cuda())
    g = torch.Generator().manual_seed(n)
    lbar = torch.randn((batch, n, n), generator=g).tril()
    abar = potrf_backward(l, lbar.cuda()).cpu().numpy()
    want = oracle.potrf_backward_f64(l.cpu().numpy().astype(np.float64), lbar.numpy().astype(np.float64))
    assert _rel(abar, want) <= TOL["bf16x3"]
    assert np.allclose(abar, np.swapaxes(abar, -1, -2), atol=1e-6 * np.abs(abar).max())


def test_autograd_function_matches_torch():
    a = inputs.well_conditioned(3, 96, seed=4, device="cuda").requires_grad_(True)
    w = torch.randn(3, 96, 96, device="cuda")
    (ours,) = torch.autograd.grad((cholesky_differentiable(a) * w).sum(), a)
    a2 = a.detach().double().requires_grad_(True)
    (ref,) = torch.autograd.grad((torch.linalg.cholesky(a2) * w.double()).sum(), a2)
    assert _rel(ours.cpu(), ref.cpu()) <= TOL["bf16x3"]


@pytest.mark.parametrize("batch,n", [(16, 128), (2, 512)])
def test_gp_loss_gradient(batch, n):
    a, y = inputs.rbf_kernel_batch(batch, n, seed=11, device="cuda")
    a.requires_grad_(True)
    loss = gp_nll(a, y).sum()
    (grad,) = torch.autograd.grad(loss, a)
    want = gp_nll_grad_closed_form(a.detach(), y)
    # The RBF matrices are ill-conditioned (jitter 1e-4), so compare against
    # torch's own FP32 autograd as well, not only the FP64 closed form.
    a32 = a.detach().clone().requires_grad_(True)
    l32 = torch.linalg.cholesky(a32)
    alpha = torch.linalg.solve_triangular(l32, y.unsqueeze(-1), upper=False).squeeze(-1)
    loss32 = (0.5 * (alpha * alpha).sum(-1) + torch.log(torch.diagonal(l32, dim1=-2, dim2=-1)).sum(-1)).sum()
    (g32,) = torch.autograd.grad(loss32, a32)
    e_ours = _rel(grad.cpu(), want.cpu())
    e_torch = _rel(g32.cpu(), want.cpu())
    assert e_ours <= max(10 * e_torch, 1e-3), (e_ours, e_torch)


def test_adjoint_finite_difference():
    """<Abar, dA> == d<Lbar, L>/dt by central differences of the FP64 oracle factor."""
    n = 40
    a = inputs.well_conditioned(1, n, seed=2, device="cpu").double()
    rng = np.random.default_rng(0)
    lbar = np.tril(rng.standard_normal((1, n, n)))
    da = rng.standard_normal((1, n, n))
    da = 0.5 * (da + np.swapaxes(da, -1, -2))
    h = 1e-6
    lp, _ = oracle.potrf_f64(a.numpy() + h * da)
    lm, _ = oracle.potrf_f64(a.numpy() - h * da)
    fd = float(np.sum(lbar * (lp - lm)) / (2 * h))
    l = cholesky(a.float().cuda())
    abar = potrf_backward(l, torch.from_numpy(lbar).float().cuda()).cpu().double().numpy()
    assert float(np.sum(abar * da)) == pytest.approx(fd, rel=1e-3)
