"""The device-side checker (gpumode_cholesky_b200.checker) against the reference's verdicts.

CPU: the same torch code on CPU tensors gives the golden cases' verdicts, and
scaled residuals within 15 % of the reference's own (the bound the oracle's
restatement is held to: FP32 accumulation order differs between BLAS
libraries); the FP64 norms equal the oracle's FP64 norms.  GPU: the same on
device tensors, and a full-size factor from this library passes.
"""

from __future__ import annotations

import numpy as np
import pytest
import torch

import oracle
from gpumode_cholesky_b200 import checker
from tests.conftest import GOLDEN_CASES, case_id


def _verdict_matches(c, device):
    a = torch.from_numpy(c["a"]).to(device)
    l = torch.from_numpy(c["l"]).to(device)
    ok, msg = checker.check(a, l)
    assert ok == c["ok"], msg
    if ok:
        got = oracle.scaled_residual(msg)
        ref = oracle.scaled_residual(c["message"])
        assert got == pytest.approx(ref, rel=0.15, abs=0.01)
        assert msg.endswith(f"; batch={c['batch']}; n={c['a'].shape[-1]}")


@pytest.mark.parametrize("c", GOLDEN_CASES, ids=case_id)
def test_checker_matches_reference_verdicts_cpu(c):
    _verdict_matches(c, "cpu")


def test_fp64_norms_equal_oracle_cpu():
    for c in GOLDEN_CASES[:8]:
        nrm = checker.residual_norms(torch.from_numpy(c["a"]), torch.from_numpy(c["l"]), precision="fp64")
        ref = oracle.residuals(c["a"], c["l"])
        for key in ("a_l1", "upper_l1", "resid_l1", "rel_fro"):
            np.testing.assert_allclose(nrm[key].numpy(), ref[key], rtol=1e-6, atol=1e-300)


def test_checker_rejects_bad_outputs_cpu():
    c = GOLDEN_CASES[0]
    a = torch.from_numpy(c["a"])
    l = torch.from_numpy(c["l"]).clone()
    assert checker.check(a, l)[0]
    bad = l.clone()
    bad[0, 0, 1] = 1.0
    assert checker.check(a, bad)[1].startswith("output is not lower triangular enough")
    bad = l.clone()
    bad[0, 1, 1] = -bad[0, 1, 1]
    assert checker.check(a, bad) == (False, "output diagonal must be strictly positive")
    bad = l.clone()
    bad[0, -1, 0] += 1.0
    assert checker.check(a, bad)[1].startswith("L @ L.T does not reconstruct A")
    bad = l.clone()
    bad[0, 2, 1] = float("nan")
    assert checker.check(a, bad) == (False, "output contains NaN or Inf")
    assert not checker.check(a, l[:1])[0]
    assert not checker.check(a, l.double())[0]
    with pytest.raises(ValueError):
        checker.residual_norms(a, l, precision="bf16")


@pytest.mark.gpu
@pytest.mark.parametrize("c", GOLDEN_CASES, ids=case_id)
def test_checker_matches_reference_verdicts_gpu(c):
    _verdict_matches(c, "cuda")


@pytest.mark.gpu
def test_checker_full_size_factor_gpu():
    from gpumode_cholesky_b200 import cholesky, inputs

    a = inputs.well_conditioned(1, 8192, seed=3, device="cuda")
    l = cholesky(a, mode="auto")
    ok, msg = checker.check(a, l)
    assert ok, msg
    nrm = checker.residual_norms(a, l, precision="fp64")
    ld, ad = l.double(), a.double()
    rel = torch.linalg.matrix_norm(ld @ ld.transpose(-1, -2) - ad) / torch.linalg.matrix_norm(ad)
    assert nrm["rel_fro"].item() == pytest.approx(rel.item(), rel=1e-6)
    assert nrm["rel_fro"].item() <= 1e-5
