"""GPU: the FP8 mode (B2P_MODE_FP8, "fp8") on the split path.

The trailing updates run as a BF16 product of the operands' high halves plus
the two cross terms hi*lo and lo*hi in E4M3 with a power-of-two scale per
64-row block (panel_copy.cuh), accumulated in FP32; the diagonal blocks and
the panel solves stay FP32.  Bars (the stated tolerance of the FP8 path):
  * relative residual ||A - L L^T||_F / ||A||_F <= 1e-4, in FP64 on the
    device, and the reference checker's verdict;
  * forward error against the FP64 oracle (n <= 1024) or cuSOLVER's FP64
    factor: at most 1e-2 relative (the cross terms' E4M3 rounding is about
    2^-12 of each product);
  * info = 0, finite, exact zeros above the diagonal, positive diagonal;
    a negative pivot gives info = its index + 1; bitwise repeats.
The CPU emulation of the same scheme (BF16 hi products plus scaled E4M3
cross terms) gives a relative residual of 2.7e-5 at orders 1024 and 2048 on
G G^T / n + 0.1 I; pure per-32-block E4M3 products give 1.2e-2.
"""

from __future__ import annotations

import numpy as np
import pytest
import torch

import oracle
from gpumode_cholesky_b200 import checker, cholesky, inputs

pytestmark = pytest.mark.gpu


def _residual(l: torch.Tensor, a: torch.Tensor) -> torch.Tensor:
    ld, ad = l.double(), a.double()
    r = ld @ ld.transpose(-1, -2)
    r -= ad
    return torch.linalg.matrix_norm(r) / torch.linalg.matrix_norm(ad)


def _common(a: torch.Tensor, l: torch.Tensor, info: torch.Tensor) -> None:
    assert (info == 0).all()
    assert torch.isfinite(l).all()
    assert (torch.triu(l, 1) == 0).all()
    assert (torch.diagonal(l, dim1=-2, dim2=-1) > 0).all()
    res = _residual(l, a)
    assert (res <= 1e-4).all(), res.tolist()
    ok, msg = checker.check(a, l)
    assert ok, msg


@pytest.mark.parametrize("batch,n", [(3, 1024), (2, 2048), (1, 4096)])
@pytest.mark.parametrize("gen", ["gram", "well"])
def test_fp8_split_orders(batch, n, gen):
    if gen == "gram":
        a = torch.stack([inputs.large_gram(n, seed=n + i, device="cuda")[0] for i in range(batch)])
    else:
        a = inputs.well_conditioned(batch, n, seed=n + 1, device="cuda")
    info = torch.full((batch,), -9, dtype=torch.int32, device="cuda")
    l = cholesky(a, mode="fp8", info=info)
    torch.cuda.synchronize()
    _common(a, l, info)
    if n <= 1024:
        l64, _ = oracle.potrf_f64(a.cpu().numpy())
        err = np.linalg.norm((l.cpu().numpy() - l64).reshape(batch, -1), axis=1) / np.linalg.norm(
            l64.reshape(batch, -1), axis=1
        )
    else:
        l64 = torch.linalg.cholesky(a.double())
        err = (torch.linalg.matrix_norm(l.double() - l64) / torch.linalg.matrix_norm(l64)).cpu().numpy()
    assert (err <= 1e-2).all(), err
    assert torch.equal(l, cholesky(a, mode="fp8"))
    bad = a.clone()
    j = n - 100
    bad[batch - 1, j, j] = -1.0
    cholesky(bad, mode="fp8", info=info)
    torch.cuda.synchronize()
    assert info[batch - 1].item() == j + 1


@pytest.mark.parametrize("n", [16384, 32768])
def test_fp8_config3_large_orders(n):
    a = inputs.large_gram(n, seed=n + 7, device="cuda")
    info = torch.full((1,), -9, dtype=torch.int32, device="cuda")
    l = cholesky(a, mode="fp8", info=info)
    torch.cuda.synchronize()
    _common(a, l, info)
    assert torch.equal(l, cholesky(a, mode="fp8"))
