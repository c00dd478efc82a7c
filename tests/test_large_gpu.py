"""GPU: the large single matrices of the benchmark suite, 1 x 16384 and 1 x 32768.

A = G G^T / n + 0.1 I with G ~ N(0, 1) (the benchmark's generator), factored
on the split path with the outer-block update, in BF16x3 and in the drop-in's
"auto" mode (BF16x3 with the pivot guard).  Held to:
  * info = 0, finite, exact zeros above the diagonal, positive diagonal;
  * relative residual ||A - L L^T||_F / ||A||_F (FP64, on the device) at
    most 1e-5, or twice that of cuSOLVER's FP32 factor where that is larger
    (FP32 rounding itself grows like sqrt(n) eps at these orders);
  * the reference checker's verdict (reference/reference.py:137-188);
  * forward error against cuSOLVER's FP64 factor within the mixed modes'
    bound of the parity tests: 64 x that of cuSOLVER's FP32 factor + 1e-6;
  * a negative pivot deep in the matrix gives info = its index + 1 (the
    leading block is SPD);
  * bitwise-identical repeats.
Sizes are beyond what the CPU oracle factors in seconds, so the checks are
these size-independent properties; the oracle covers the same kernels at
orders up to 4096 in test_paths_gpu.py.
"""

from __future__ import annotations

import pytest
import torch

from gpumode_cholesky_b200 import checker, cholesky, inputs

pytestmark = pytest.mark.gpu


def _residual(l: torch.Tensor, a: torch.Tensor) -> float:
    ld = l.double()
    r = ld @ ld.transpose(-1, -2)
    del ld
    r -= a.double()
    out = (torch.linalg.matrix_norm(r) / torch.linalg.matrix_norm(a.double())).max().item()
    del r
    return out


def _rel(x: torch.Tensor, y: torch.Tensor) -> float:
    return (torch.linalg.matrix_norm(x.double() - y) / torch.linalg.matrix_norm(y)).max().item()


@pytest.mark.parametrize("mode", ["bf16x3", "auto"])
@pytest.mark.parametrize("n", [16384, 32768])
def test_config3_large_orders(n, mode):
    a = inputs.large_gram(n, seed=n + 7, device="cuda")
    info = torch.full((1,), -9, dtype=torch.int32, device="cuda")
    l = cholesky(a, mode=mode, info=info)
    torch.cuda.synchronize()
    assert info.item() == 0
    assert torch.isfinite(l).all()
    assert (torch.triu(l, 1) == 0).all()
    assert (torch.diagonal(l, dim1=-2, dim2=-1) > 0).all()

    ref32 = torch.linalg.cholesky(a)
    res, res32 = _residual(l, a), _residual(ref32, a)
    assert res <= max(1e-5, 2.0 * res32), (res, res32)
    ok, msg = checker.check(a, l)
    assert ok, msg

    l64 = torch.linalg.cholesky(a.double())
    fwd, fwd32 = _rel(l, l64), _rel(ref32, l64)
    del l64, ref32
    assert fwd <= 64.0 * fwd32 + 1e-6, (fwd, fwd32)

    again = cholesky(a, mode=mode)
    assert torch.equal(again, l)
    del again, l

    j = n - 1000
    a[0, j, j] = -1.0
    cholesky(a, mode=mode, info=info)
    torch.cuda.synchronize()
    assert info.item() == j + 1
