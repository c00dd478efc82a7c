"""GPU: batched triangular solves and the Gaussian-process loss kernels.

Oracle: torch's FP64 solve_triangular / inverse on the same factor, and the
FP64 closed-form gradient of the loss; bars are relative errors against the
FP64 values, held to what torch's own FP32 route achieves (x10) or 1e-5.
"""

from __future__ import annotations

import pytest
import torch

from gpumode_cholesky_b200 import cholesky, gp_nll, inputs
from gpumode_cholesky_b200.gp import gp_nll_from_factor, gp_nll_grad_closed_form, gp_nll_lbar, trsv

pytestmark = pytest.mark.gpu


def _rel(x: torch.Tensor, ref: torch.Tensor) -> float:
    return (torch.linalg.norm((x.double() - ref).flatten()) / torch.linalg.norm(ref.flatten())).item()


@pytest.mark.parametrize("trans", [False, True])
@pytest.mark.parametrize("batch,n", [(3, 1), (4, 5), (2, 31), (2, 32), (2, 33), (5, 100), (3, 129), (2, 500), (2, 2048)])
def test_trsv_against_fp64(trans, batch, n):
    a = inputs.well_conditioned(batch, n, seed=n + 1, device="cuda")
    l = cholesky(a, mode="fp32")
    b = torch.randn(batch, n, device="cuda", generator=torch.Generator("cuda").manual_seed(n))
    x = trsv(l, b, trans=trans)
    ref = torch.linalg.solve_triangular(
        l.double().transpose(-1, -2) if trans else l.double(), b.double().unsqueeze(-1), upper=trans
    ).squeeze(-1)
    t32 = torch.linalg.solve_triangular(l.transpose(-1, -2) if trans else l, b.unsqueeze(-1), upper=trans).squeeze(-1)
    assert _rel(x, ref) <= max(10 * _rel(t32, ref), 1e-5)


def test_trsv_in_place_and_rejects():
    a = inputs.well_conditioned(2, 70, seed=3, device="cuda")
    l = cholesky(a, mode="fp32")
    b = torch.randn(2, 70, device="cuda")
    want = trsv(l, b)
    from gpumode_cholesky_b200 import _lib

    lib = _lib.load()
    st = lib.b2p_trsv_batched(l.data_ptr(), b.data_ptr(), b.data_ptr(), 2, 70, 0, None)
    torch.cuda.synchronize()
    assert st == _lib.B2P_OK and torch.equal(b, want)
    assert lib.b2p_trsv_batched(l.data_ptr(), b.data_ptr(), b.data_ptr(), 2, 40000, 0, None) == _lib.B2P_ERR_INVALID_ARG
    assert lib.b2p_trsv_batched(None, b.data_ptr(), b.data_ptr(), 2, 70, 0, None) == _lib.B2P_ERR_INVALID_ARG


@pytest.mark.parametrize("batch,n", [(256, 128), (8, 2048), (3, 77)])
def test_gp_forward_and_lbar_against_fp64(batch, n):
    """Loss and alpha from the factor; beta = A^{-1} y and Lbar against FP64 on the same factor."""
    a, y = inputs.rbf_kernel_batch(batch, n, seed=5, device="cuda")
    l = cholesky(a, mode="fp32")
    loss, alpha = gp_nll_from_factor(l, y)
    ld = l.double()
    a64 = torch.linalg.solve_triangular(ld, y.double().unsqueeze(-1), upper=False).squeeze(-1)
    loss64 = 0.5 * (a64 * a64).sum(-1) + torch.log(torch.diagonal(ld, dim1=-2, dim2=-1)).sum(-1)
    a32 = torch.linalg.solve_triangular(l, y.unsqueeze(-1), upper=False).squeeze(-1)
    assert _rel(alpha, a64) <= max(10 * _rel(a32, a64), 1e-5)
    assert torch.allclose(loss.double(), loss64, rtol=1e-4, atol=1e-3 * n)
    g = torch.rand(batch, device="cuda") + 0.5
    beta, lbar = gp_nll_lbar(l, alpha, g)
    b64 = torch.linalg.solve_triangular(ld.transpose(-1, -2), a64.unsqueeze(-1), upper=True).squeeze(-1)
    b32 = torch.linalg.solve_triangular(l.transpose(-1, -2), a32.unsqueeze(-1), upper=True).squeeze(-1)
    assert _rel(beta, b64) <= max(10 * _rel(b32, b64), 1e-5)
    want = g.double()[:, None, None] * (
        torch.tril(-b64.unsqueeze(-1) * a64.unsqueeze(-2)) + torch.diag_embed(1.0 / torch.diagonal(ld, dim1=-2, dim2=-1))
    )
    assert _rel(lbar, want) <= max(10 * _rel(b32, b64), 1e-5)
    assert (torch.triu(lbar, 1) == 0).all()


@pytest.mark.parametrize("batch,n", [(16, 128), (2, 512), (2, 2048)])
def test_gp_loss_gradients_in_a_and_y(batch, n):
    a, y = inputs.rbf_kernel_batch(batch, n, seed=13, device="cuda")
    a.requires_grad_(True)
    y.requires_grad_(True)
    (ga, gy) = torch.autograd.grad(gp_nll(a, y).sum(), (a, y))
    want_a = gp_nll_grad_closed_form(a.detach(), y.detach())
    want_y = torch.linalg.solve(a.detach().double(), y.detach().double().unsqueeze(-1)).squeeze(-1)
    # torch's own FP32 route as the yardstick for these ill-conditioned (jitter 1e-4) matrices
    a32 = a.detach().clone().requires_grad_(True)
    y32 = y.detach().clone().requires_grad_(True)
    l32 = torch.linalg.cholesky(a32)
    al = torch.linalg.solve_triangular(l32, y32.unsqueeze(-1), upper=False).squeeze(-1)
    loss32 = (0.5 * (al * al).sum(-1) + torch.log(torch.diagonal(l32, dim1=-2, dim2=-1)).sum(-1)).sum()
    (ta, ty) = torch.autograd.grad(loss32, (a32, y32))
    assert _rel(ga, want_a) <= max(10 * _rel(ta, want_a), 1e-3)
    assert _rel(gy, want_y) <= max(10 * _rel(ty, want_y), 1e-4)
