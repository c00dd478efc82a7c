"""cholesky_checked: the residual-checked FP32 refactor of mixed-precision factors.

CPU: the randomized residual estimate tracks the oracle's exact FP64
relative residual.  GPU: the refactor pass replaces exactly the matrices that
fail, with the FP32 path's own factors.
"""

from __future__ import annotations

import numpy as np
import pytest
import torch

import oracle
from gpumode_cholesky_b200 import inputs
from gpumode_cholesky_b200.potrf import residual_estimate
from tests.conftest import GOLDEN_CASES


def test_residual_estimate_tracks_exact_residual_cpu():
    for c in GOLDEN_CASES[:10]:
        a, l = torch.from_numpy(c["a"]), torch.from_numpy(c["l"])
        exact = oracle.residuals(c["a"], c["l"])["rel_fro"]
        est = residual_estimate(a, l, probes=32, seed=1).numpy()
        ok = exact > 1e-12  # exact zeros (n = 1, 2) give a zero estimate too
        assert np.all(est[~ok] < 1e-12)
        ratio = est[ok] / exact[ok]
        assert np.all((ratio > 0.5) & (ratio < 2.0)), ratio
        np.testing.assert_allclose(residual_estimate(a, l, probes=0).numpy(), exact, rtol=1e-6, atol=1e-300)


def test_residual_estimate_flags_bad_factors_cpu():
    a = inputs.well_conditioned(3, 40, seed=2)
    l = torch.linalg.cholesky(a)
    good = residual_estimate(a, l)
    assert (good < 1e-5).all()
    l2 = l.clone()
    l2[1, 30, 3] += 1e-2  # one wrong entry: a residual far above 1e-5
    l2[2, 5, 5] = float("nan")
    est = residual_estimate(a, l2)
    assert est[0] < 1e-5 and est[1] > 1e-4 and torch.isinf(est[2])


@pytest.mark.gpu
def test_checked_tolerance_extremes_gpu():
    from gpumode_cholesky_b200 import cholesky, cholesky_checked

    a = inputs.well_conditioned(12, 512, seed=4, device="cuda")
    l, redone = cholesky_checked(a, mode="bf16x3", tol=float("inf"))
    assert not redone.any()
    assert torch.equal(l, cholesky(a, mode="bf16x3"))
    l, redone = cholesky_checked(a, mode="bf16x3", tol=0.0)
    assert redone.all()
    assert torch.equal(l, cholesky(a, mode="fp32"))


@pytest.mark.gpu
def test_checked_refactors_only_failures_gpu():
    from gpumode_cholesky_b200 import cholesky, cholesky_checked

    a = inputs.well_conditioned(10, 256, seed=8, device="cuda")
    a[6] = -a[6]  # not SPD in any precision
    info = torch.full((10,), -3, dtype=torch.int32, device="cuda")
    l, redone = cholesky_checked(a, mode="bf16x3", info=info)
    assert redone.cpu().tolist() == [i == 6 for i in range(10)]
    _, want = oracle.potrf_f64(a.cpu().numpy())
    assert info.cpu().tolist() == want.tolist()
    plain = cholesky(a, mode="bf16x3")
    keep = [i for i in range(10) if i != 6]
    assert torch.equal(l[keep], plain[keep])


@pytest.mark.gpu
def test_checked_gp_kernels_meet_tolerance_gpu():
    from gpumode_cholesky_b200 import checker, cholesky_checked

    a, _ = inputs.rbf_kernel_batch(4, 2048, seed=21, device="cuda")
    # probes=0: the exact FP64 check, so every kept factor meets the bound itself
    l, redone = cholesky_checked(a, mode="bf16x3", tol=1e-5, probes=0)
    assert torch.isfinite(l).all()
    rel = checker.residual_norms(a, l, precision="fp64")["rel_fro"]
    assert (rel <= 1e-5).all(), (rel.tolist(), redone.tolist())
