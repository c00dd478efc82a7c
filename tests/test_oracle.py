"""CPU: pin the oracle and the input generators against the reference's golden vectors."""

from __future__ import annotations

import numpy as np
import pytest
import torch

import oracle
from gpumode_cholesky_b200 import inputs
from tests.conftest import GOLDEN_CASES, case_id


@pytest.mark.parametrize("c", GOLDEN_CASES, ids=case_id)
def test_generator_reproduces_reference_inputs(c):
    """inputs.generate_input == reference generate_input, bit for bit, on CPU."""
    a = inputs.generate_input(c["batch"], c["n"], c["cond"], c["seed"], c["case"], device="cpu")
    assert np.array_equal(a.numpy(), c["a"])


@pytest.mark.parametrize("c", GOLDEN_CASES, ids=case_id)
def test_checker_restatement_matches_reference(c):
    """oracle.check_implementation gives the reference checker's verdict and residual."""
    ok, msg = oracle.check_implementation(c["a"], c["l"])
    assert ok == c["ok"]
    ref = oracle.scaled_residual(c["message"])
    got = oracle.scaled_residual(msg)
    # Same formula; FP32 summation order differs between torch and numpy.
    assert got == pytest.approx(ref, rel=0.15, abs=0.01)


@pytest.mark.parametrize("c", GOLDEN_CASES, ids=case_id)
def test_oracle_fp64_close_to_reference(c):
    """FP64 oracle factor vs the reference's FP32 LAPACK factor (rounding-level difference)."""
    l64, info = oracle.potrf_f64(c["a"])
    assert np.array_equal(info, c["info"])
    err = np.linalg.norm((l64 - c["l"]).reshape(c["batch"], -1), axis=1) / np.linalg.norm(
        l64.reshape(c["batch"], -1), axis=1
    )
    # condition-dependent bound: eps32 * n * kappa^(1/2)-ish; generous and family-aware
    bound = {"dense": 2e-5, "diagonal": 1e-6, "tridiagonal": 2e-5}.get(c["case"], 5e-3)
    assert err.max() < bound, err.max()
    # The FP64 oracle itself reconstructs A to FP32 input precision.
    r = oracle.residuals(c["a"], l64.astype(np.float32))
    assert r["rel_fro"].max() < 1e-5


@pytest.mark.parametrize("c", GOLDEN_CASES[:6], ids=case_id)
def test_oracle_fp32_passes_reference_checker(c):
    l32, info = oracle.potrf_f32(c["a"])
    ok, msg = oracle.check_implementation(c["a"], l32)
    assert ok, msg
    assert np.array_equal(info, c["info"])


def test_oracle_nonspd_info(golden_nonspd):
    a, info = golden_nonspd
    _, got = oracle.potrf_f64(a)
    assert np.array_equal(got, info)
    l32, got32 = oracle.potrf_f32(a)
    assert np.array_equal(got32, info)
    assert np.isnan(l32[1]).any() and np.isfinite(l32[0]).all()


def test_checker_rejects_bad_outputs(golden_cases):
    """The restated checker fails the same way the reference does on planted faults."""
    c = golden_cases[0]
    a, l = c["a"], c["l"].copy()
    bad = l.copy()
    bad[0, 0, 5] = 1.0  # upper triangle
    assert not oracle.check_implementation(a, bad)[0]
    bad = l.copy()
    bad[0, 3, 3] = -bad[0, 3, 3]  # negative diagonal
    assert not oracle.check_implementation(a, bad)[0]
    bad = l.copy()
    bad[0, 10, 2] += 1e-2  # reconstruction
    assert not oracle.check_implementation(a, bad)[0]
    bad = l.copy()
    bad[0, 1, 0] = np.nan
    assert oracle.check_implementation(a, bad) == (False, "output contains NaN or Inf")
    assert not oracle.check_implementation(a, l[:1])[0]


def test_oracle_backward_matches_torch_autograd(golden_backward):
    for g in golden_backward:
        got = oracle.potrf_backward_f64(g["l"], g["lbar"])
        np.testing.assert_allclose(got, g["abar"], rtol=1e-9, atol=1e-10)


def test_oracle_backward_finite_difference():
    """Adjoint identity <Abar, dA> = <Lbar, dL> by central differences (FP64)."""
    rng = np.random.default_rng(7)
    n = 12
    m = rng.standard_normal((n, n))
    a = m @ m.T / n + np.eye(n)
    lbar = np.tril(rng.standard_normal((n, n)))
    da = rng.standard_normal((n, n))
    da = 0.5 * (da + da.T)
    h = 1e-6
    lp, _ = oracle.potrf_f64(a + h * da)
    lm, _ = oracle.potrf_f64(a - h * da)
    fd = np.sum(lbar * (lp[0] - lm[0])) / (2 * h)
    l, _ = oracle.potrf_f64(a)
    abar = oracle.potrf_backward_f64(l, lbar)[0]
    assert np.sum(abar * da) == pytest.approx(fd, rel=1e-6)


def test_ref_kernel_cpu_is_reference_route(golden_cases):
    c = golden_cases[1]
    l = oracle.ref_kernel_cpu(torch.from_numpy(c["a"]))
    assert np.array_equal(l.numpy(), c["l"])
