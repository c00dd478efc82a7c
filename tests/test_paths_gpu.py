"""GPU: every n > 128 algorithm forced through b2p_potrf_batched_path.

Each path (blocked right-looking, fused one-CTA-per-matrix, its
warp-specialized form, and the multi-CTA split path) is checked on its own
against the same bars as the automatic dispatch:
  * relative residual ||A - L L^T||_F / ||A||_F <= 1e-5 (BF16x3), <= 1e-3
    (TF32), computed in FP64;
  * exact zeros above the diagonal and a positive diagonal;
  * info equal to the FP64 oracle's for a matrix with a negative pivot;
  * agreement between paths: relative Frobenius distance of the factors
    <= 1e-5 (BF16x3) / 2e-3 (TF32).
"""

from __future__ import annotations

import pytest
import torch

import oracle
from gpumode_cholesky_b200 import cholesky, inputs

pytestmark = pytest.mark.gpu

TOL_FACTOR = {"tf32": 1e-3, "bf16x3": 1e-5}
TOL_AGREE = {"tf32": 2e-3, "bf16x3": 1e-5}


def _residual(l: torch.Tensor, a: torch.Tensor) -> float:
    ld, ad = l.double(), a.double()
    r = torch.linalg.matrix_norm(ld @ ld.transpose(-1, -2) - ad) / torch.linalg.matrix_norm(ad)
    return r.max().item()


def _check_factor(l: torch.Tensor, a: torch.Tensor, mode: str) -> None:
    assert torch.isfinite(l).all()
    assert (torch.triu(l, 1) == 0).all()
    assert (torch.diagonal(l, dim1=-2, dim2=-1) > 0).all()
    assert _residual(l, a) <= TOL_FACTOR[mode]


@pytest.mark.parametrize("mode", ["tf32", "bf16x3"])
@pytest.mark.parametrize(
    "batch,n",
    [(3, 192), (2, 320), (5, 512), (2, 1024), (3, 1536), (2, 2048), (1, 4096)],
)
def test_split_path(mode, batch, n):
    # TF32 operands (~1e-3 relative) cannot factor the spectrum [1, 1e6]
    # half of the mixed batch; BF16x3 must.
    if mode == "tf32":
        a = inputs.well_conditioned(batch, n, seed=n + 3, device="cuda")
    else:
        a = inputs.mixed_batch(batch, n, seed=n + 3, device="cuda")
    info = torch.full((batch,), -9, dtype=torch.int32, device="cuda")
    l = cholesky(a, mode=mode, info=info, path="split")
    assert (info == 0).all()
    _check_factor(l, a, mode)


@pytest.mark.parametrize("mode", ["tf32", "bf16x3"])
@pytest.mark.parametrize("batch,n", [(1, 8192), (2, 12288), (1, 12352)])
def test_split_path_large_orders(mode, batch, n):
    """n >= 12288: the panels older than the previous 512-column outer block
    are applied by the wide update (12352 ends in a partial outer block);
    8192 runs without it.  Factor bars as above; a negative pivot deep in the
    matrix gives the oracle's info; the result is bitwise reproducible."""
    a = torch.stack([inputs.large_gram(n, seed=n + i, device="cuda")[0] for i in range(batch)])
    info = torch.full((batch,), -9, dtype=torch.int32, device="cuda")
    l = cholesky(a, mode=mode, info=info, path="split")
    assert (info == 0).all()
    assert torch.isfinite(l).all()
    assert (torch.triu(l, 1) == 0).all()
    assert (torch.diagonal(l, dim1=-2, dim2=-1) > 0).all()
    # Above n ~ 1e4 an FP32 factorization itself leaves a relative residual
    # above 1e-5 (rounding grows like sqrt(n) eps), so BF16x3 is held to
    # 1e-5 or twice the residual of the FP32 library factor, whichever is larger.
    bar = TOL_FACTOR[mode]
    if mode == "bf16x3":
        bar = max(bar, 2.0 * _residual(torch.linalg.cholesky(a), a))
    assert _residual(l, a) <= bar
    again = cholesky(a, mode=mode, path="split")
    assert torch.equal(l, again)
    j = n - 700
    a[batch - 1, j, j] = -1.0
    cholesky(a, mode=mode, info=info, path="split")
    assert info[batch - 1].item() == j + 1
    if batch > 1:
        assert (info[: batch - 1] == 0).all()


@pytest.mark.parametrize("path", ["fused", "fused_ws", "split", "blocked"])
@pytest.mark.parametrize("mode", ["tf32", "bf16x3"])
def test_paths_agree(path, mode):
    a = inputs.well_conditioned(6, 640, seed=21, device="cuda")
    l = cholesky(a, mode=mode, path=path)
    _check_factor(l, a, mode)
    ref = cholesky(a, mode="fp32", path="blocked").double()
    d = torch.linalg.norm((l.double() - ref).flatten()) / torch.linalg.norm(ref.flatten())
    assert d.item() <= TOL_AGREE[mode]


@pytest.mark.parametrize("path", ["fused", "fused_ws", "split", "blocked"])
@pytest.mark.parametrize("col", [5, 40, 64, 200, 447])
def test_paths_nonspd_info(path, col):
    a = inputs.generate_input(3, 448, 2, 91, "dense", device="cpu")
    a[1, col, col] = -5.0
    _, ref = oracle.potrf_f64(a.numpy())
    info = torch.full((3,), -9, dtype=torch.int32, device="cuda")
    l = cholesky(a.cuda(), mode="bf16x3", info=info, path=path)
    assert info.cpu().tolist() == ref.tolist()
    assert torch.isfinite(l[0]).all() and torch.isfinite(l[2]).all()
    assert torch.isnan(l[1]).any()


@pytest.mark.parametrize("batch,n", [(3, 1024), (5, 768), (16, 512), (40, 576), (150, 256)])
def test_fused_ws_cluster_and_single(batch, n):
    """Small batches run 8, 4 or 2 CTAs per matrix; batches above half the SM count one."""
    a = inputs.mixed_batch(batch, n, seed=batch + n, device="cuda")
    info = torch.full((batch,), -9, dtype=torch.int32, device="cuda")
    l = cholesky(a, mode="bf16x3", info=info, path="fused_ws")
    assert (info == 0).all()
    _check_factor(l, a, "bf16x3")
    # Same arithmetic as the one-CTA-per-matrix kernel.
    ref = cholesky(a, mode="bf16x3", path="fused").double()
    d = torch.linalg.norm((l.double() - ref).flatten()) / torch.linalg.norm(ref.flatten())
    assert d.item() <= TOL_AGREE["bf16x3"]


def test_split_repeat_bitwise():
    a = inputs.well_conditioned(2, 1536, seed=4, device="cuda")
    assert torch.equal(cholesky(a, mode="bf16x3", path="split"), cholesky(a, mode="bf16x3", path="split"))


def test_split_passes_reference_checker():
    a = inputs.generate_input(2, 1024, 2, 123, "dense", device="cpu")
    l = cholesky(a.cuda(), mode="bf16x3", path="split").cpu().numpy()
    ok, msg = oracle.check_implementation(a.numpy(), l)
    assert ok, msg


def test_unsupported_path_raises():
    a = inputs.well_conditioned(1, 2048, seed=1, device="cuda")
    with pytest.raises(Exception, match="unsupported"):
        cholesky(a, mode="bf16x3", path="fused")
    with pytest.raises(Exception, match="unsupported"):
        cholesky(a, mode="bf16x3", path="fused_ws")
    with pytest.raises(Exception, match="unsupported"):
        cholesky(a, mode="fp32", path="split")
