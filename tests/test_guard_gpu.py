"""GPU: the pivot guard of the mixed modes (B2P_FLAG_GUARD, mode suffix "+guard").

After each 64-wide block column's diagonal block is factored, the guard
checks every pivot against the error the mixed update may carry; a failing
column, and every later column of that matrix, is recomputed with its
update in FP32.  The tests hold it to:
  * no effect where nothing fails: bitwise equal to the unguarded mode, and
    fp32_from = -1, on well-conditioned inputs, on every guarded path;
  * a known trigger: A = G G^T / r + 3e-5 I with G of rank r = 200 has
    pivots near 3e-5 A_jj from column 200 on, under the BF16x3 bound at block
    column 3 (columns 192..255), so fp32_from = 3 on every path; the factor
    is then as accurate as the plain FP32 one (relative residual in FP64 at
    most twice FP32's plus 1e-7, forward error against the FP64 oracle at
    most twice FP32's plus 1e-6) and passes the reference checker;
  * non-SPD input: the oracle's info (the guard recomputes the failing
    column in FP32 and the pivot is still negative there);
  * Gaussian-process kernels (config 5 inputs, order 2048), where plain
    BF16x3 can produce NaN pivots: finite, positive diagonal, residual
    within twice the FP32 factor's.
"""

from __future__ import annotations

import numpy as np
import pytest
import torch

import oracle
from gpumode_cholesky_b200 import cholesky, custom_kernel, inputs

pytestmark = pytest.mark.gpu

PATHS = ["fused", "fused_ws", "split"]


def _rel_residual(a: torch.Tensor, l: torch.Tensor) -> torch.Tensor:
    ld, ad = l.double(), a.double()
    return torch.linalg.matrix_norm(ld @ ld.transpose(-1, -2) - ad) / torch.linalg.matrix_norm(ad)


def _low_rank_plus_jitter(batch: int, n: int, r: int, jitter: float, seed: int) -> torch.Tensor:
    g = torch.Generator().manual_seed(seed)
    m = torch.randn(batch, n, r, generator=g, dtype=torch.float64)
    a = m @ m.transpose(-1, -2) / r + jitter * torch.eye(n, dtype=torch.float64)
    return a.float()


@pytest.mark.parametrize("path", PATHS)
@pytest.mark.parametrize("mode", ["bf16x3", "tf32"])
def test_guard_is_silent_on_well_conditioned_input(path, mode):
    batch, n = (6, 512) if path != "split" else (2, 1024)
    a = inputs.well_conditioned(batch, n, seed=77 + n, device="cuda")
    want = cholesky(a, mode=mode, path=path)
    fp = torch.full((batch,), 99, dtype=torch.int32, device="cuda")
    got = cholesky(a, mode=mode + "+guard", path=path, fp32_from=fp)
    torch.cuda.synchronize()
    assert torch.equal(got, want)
    assert (fp == -1).all()


@pytest.mark.parametrize("path", PATHS + ["auto"])
def test_guard_recomputes_from_the_failing_column(path):
    batch, n, r = 4, 512, 200
    a = _low_rank_plus_jitter(batch, n, r, 3e-5, seed=5).cuda()
    fp = torch.full((batch,), 99, dtype=torch.int32, device="cuda")
    info = torch.full((batch,), 7, dtype=torch.int32, device="cuda")
    got = cholesky(a, mode="bf16x3+guard", path=path, fp32_from=fp, info=info)
    plain = cholesky(a, mode="fp32")
    torch.cuda.synchronize()
    assert fp.tolist() == [r // 64] * batch
    assert (info == 0).all()
    assert torch.isfinite(got).all()
    assert (torch.triu(got, 1) == 0).all()
    res, res32 = _rel_residual(a, got), _rel_residual(a, plain)
    assert (res <= 2 * res32 + 1e-7).all(), (res.tolist(), res32.tolist())
    an = a.cpu().numpy()
    l64, _ = oracle.potrf_f64(an)
    err = np.linalg.norm((got.cpu().numpy() - l64).reshape(batch, -1), axis=1)
    err32 = np.linalg.norm((plain.cpu().numpy() - l64).reshape(batch, -1), axis=1)
    assert (err <= 2 * err32 + 1e-6 * np.linalg.norm(l64.reshape(batch, -1), axis=1)).all(), (err, err32)
    ok, msg = oracle.check_implementation(an, got.cpu().numpy())
    assert ok, msg
    # Bitwise repeatable, like every other path.
    assert torch.equal(got, cholesky(a, mode="bf16x3+guard", path=path))


def test_guard_split_large_order():
    """The split path's step kernels carry the guard state across launches."""
    batch, n, r = 1, 2048, 1000
    a = _low_rank_plus_jitter(batch, n, r, 3e-5, seed=6).cuda()
    fp = torch.full((batch,), 99, dtype=torch.int32, device="cuda")
    got = cholesky(a, mode="bf16x3+guard", path="split", fp32_from=fp)
    plain = cholesky(a, mode="fp32")
    torch.cuda.synchronize()
    assert 0 <= fp.item() <= r // 64
    assert torch.isfinite(got).all()
    assert (_rel_residual(a, got) <= 2 * _rel_residual(a, plain) + 1e-7).all()


@pytest.mark.parametrize("path", PATHS)
def test_guard_keeps_the_oracle_info_on_non_spd_input(path):
    batch, n = 2, 512
    a = inputs.generate_input(batch, n, 2, 91, "dense", device="cpu")
    j = 300
    a[1, j, j] = -5.0
    _, want = oracle.potrf_f64(a.numpy())
    info = torch.zeros(batch, dtype=torch.int32, device="cuda")
    fp = torch.zeros(batch, dtype=torch.int32, device="cuda")
    cholesky(a.cuda(), mode="bf16x3+guard", path=path, info=info, fp32_from=fp)
    torch.cuda.synchronize()
    assert info.cpu().tolist() == want.tolist()
    assert fp.cpu().tolist() == [-1, j // 64]


def test_guard_gp_kernels():
    a, _ = inputs.rbf_kernel_batch(2, 2048, seed=52048, device="cuda")
    fp = torch.full((2,), 99, dtype=torch.int32, device="cuda")
    got = cholesky(a, mode="bf16x3+guard", fp32_from=fp)
    plain = cholesky(a, mode="fp32")
    torch.cuda.synchronize()
    assert torch.isfinite(got).all()
    assert (torch.diagonal(got, dim1=-2, dim2=-1) > 0).all()
    assert (_rel_residual(a, got) <= 2 * _rel_residual(a, plain) + 1e-7).all()


def test_custom_kernel_runs_the_guarded_mixed_mode():
    """The drop-in is bitwise the explicit "bf16x3+guard" call for orders that are multiples of 64."""
    a = inputs.well_conditioned(8, 512, seed=3, device="cuda")
    assert torch.equal(custom_kernel(a), cholesky(a, mode="bf16x3+guard"))
    b = inputs.well_conditioned(8, 300, seed=3, device="cuda")
    assert torch.equal(custom_kernel(b), cholesky(b, mode="fp32"))
