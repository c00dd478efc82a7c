"""GPU: the pivot guard of the mixed modes (B2P_FLAG_GUARD, mode suffix "+guard").

After each 64-wide block column's diagonal block is factored, the guard
checks every pivot against the error the mixed update may carry and records
the first failing column per matrix (fp32_from); the matrices that trip are
then refactored from their first column in FP32 by the rescue kernel.  The
tests hold it to:
  * no effect where nothing trips: bitwise equal to the unguarded mode and
    fp32_from = -1 on well-conditioned inputs, on every guarded path;
  * a known trigger: A = G G^T / r + 1e-5 I with G of rank r has pivots of
    1e-5 A_jj from column r on and well above the bound before, so the guard
    trips at block column r // 64 or, since the mixed update biases the
    computed pivots upwards (it drops the always-positive lo*lo products and
    its accumulator truncates), within two block columns after it; the
    rescued factor is as accurate as the plain FP32 path's (relative
    residual in FP64 at most twice FP32's plus 1e-7; forward error against
    the FP64 oracle at most four times FP32's plus 1e-6 of the factor's norm,
    the rescue being left-looking where the FP32 path is right-looking) and
    passes the reference checker;
  * TF32, whose bound (about 2e-3) the prescribed-spectrum matrices of the
    mid workload fall under: those trip and come out at FP32 accuracy, the
    well-conditioned half does not trip;
  * non-SPD input: the oracle's info (the rescue meets the negative pivot in
    FP32), fp32_from at the failing column;
  * Gaussian-process kernels (config 5 inputs, order 2048), where plain
    BF16x3 can produce NaN pivots: finite, positive diagonal, residual
    within twice the FP32 factor's (or the mixed modes' 1e-5 where a matrix
    did not trip).
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


def _fp32_accuracy(a: torch.Tensor, got: torch.Tensor, idx: list[int]) -> None:
    """Matrices idx of `got` are as accurate as the plain FP32 path's factors."""
    if not idx:
        return
    a, got = a[idx], got[idx]
    plain = cholesky(a, mode="fp32")
    res, res32 = _rel_residual(a, got), _rel_residual(a, plain)
    assert (res <= 2 * res32 + 1e-7).all(), (res.tolist(), res32.tolist())
    an = a.cpu().numpy()
    l64, _ = oracle.potrf_f64(an)
    b = len(idx)
    err = np.linalg.norm((got.cpu().numpy() - l64).reshape(b, -1), axis=1)
    err32 = np.linalg.norm((plain.cpu().numpy() - l64).reshape(b, -1), axis=1)
    assert (err <= 4 * err32 + 1e-6 * np.linalg.norm(l64.reshape(b, -1), axis=1)).all(), (err, err32)
    ok, msg = oracle.check_implementation(an, got.cpu().numpy())
    assert ok, msg


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
def test_guard_rescues_from_the_failing_column(path):
    batch, n, r = 4, 512, 200
    a = _low_rank_plus_jitter(batch, n, r, 1e-5, seed=5).cuda()
    fp = torch.full((batch,), 99, dtype=torch.int32, device="cuda")
    info = torch.full((batch,), 7, dtype=torch.int32, device="cuda")
    got = cholesky(a, mode="bf16x3+guard", path=path, fp32_from=fp, info=info)
    torch.cuda.synchronize()
    assert all(r // 64 <= t <= r // 64 + 2 for t in fp.tolist()), fp.tolist()
    assert (info == 0).all()
    assert torch.isfinite(got).all()
    assert (torch.triu(got, 1) == 0).all()
    _fp32_accuracy(a, got, list(range(batch)))
    # Bitwise repeatable, like every other path.
    assert torch.equal(got, cholesky(a, mode="bf16x3+guard", path=path))


def test_guard_split_large_order():
    """The split path's step kernels carry the guard state across launches."""
    batch, n, r = 1, 2048, 1000
    a = _low_rank_plus_jitter(batch, n, r, 1e-5, seed=6).cuda()
    fp = torch.full((batch,), 99, dtype=torch.int32, device="cuda")
    got = cholesky(a, mode="bf16x3+guard", path="split", fp32_from=fp)
    torch.cuda.synchronize()
    assert r // 64 <= fp.item() <= r // 64 + 2, fp.item()
    assert torch.isfinite(got).all()
    _fp32_accuracy(a, got, [0])


@pytest.mark.parametrize("path", PATHS)
def test_guard_makes_tf32_safe_on_the_spectrum_matrices(path):
    batch, n = 4, 512
    a = inputs.mixed_batch(batch, n, 510512, device="cuda")  # the last half: spectrum [1, 1e6]
    fp = torch.full((batch,), 99, dtype=torch.int32, device="cuda")
    got = cholesky(a, mode="tf32+guard", path=path, fp32_from=fp)
    torch.cuda.synchronize()
    trips = fp.tolist()
    assert trips[0] == -1 and trips[1] == -1, trips
    assert trips[2] >= 1 and trips[3] >= 1, trips
    _fp32_accuracy(a, got, [2, 3])
    assert (_rel_residual(a[:2], got[:2]) <= 1e-3).all()


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
    res, res32 = _rel_residual(a, got), _rel_residual(a, plain)
    tripped = torch.tensor([t >= 0 for t in fp.tolist()], device=res.device)
    bound = torch.where(tripped, 2 * res32 + 1e-7, torch.full_like(res32, 1e-5))
    assert (res <= bound).all(), (fp.tolist(), res.tolist(), res32.tolist())


def test_custom_kernel_runs_the_guarded_mixed_mode():
    """The drop-in is bitwise the explicit "bf16x3+guard" call for orders that are multiples of 64."""
    a = inputs.well_conditioned(8, 512, seed=3, device="cuda")
    assert torch.equal(custom_kernel(a), cholesky(a, mode="bf16x3+guard"))
    b = inputs.well_conditioned(8, 300, seed=3, device="cuda")
    assert torch.equal(custom_kernel(b), cholesky(b, mode="fp32"))
