"""GPU: the tcgen05 tensor-core path (TF32 and BF16x3 trailing updates).

Tolerances:
  * the diagnostic tile GEMM against an FP64 product: relative Frobenius
    error <= 2e-3 for TF32 (10-bit mantissa operands), <= 2e-5 for BF16x3;
  * factorizations: relative residual ||A - L L^T||_F / ||A||_F <= 1e-5 for
    BF16x3 (the stated mixed-precision target) and <= 1e-3 for TF32, plus the
    restated reference checker on the well-conditioned inputs for BF16x3.
"""

from __future__ import annotations

import ctypes

import numpy as np
import pytest
import torch

import oracle
from gpumode_cholesky_b200 import _lib, cholesky, inputs

pytestmark = pytest.mark.gpu

TOL_GEMM = {"tf32": 2e-3, "bf16x3": 2e-5}
TOL_FACTOR = {"tf32": 1e-3, "bf16x3": 1e-5}


def _rel_fro(x: torch.Tensor, y: torch.Tensor) -> float:
    return float((torch.linalg.norm((x - y).flatten()) / torch.linalg.norm(y.flatten())).item())


@pytest.mark.parametrize("mode", ["tf32", "bf16x3"])
def test_tile_gemm_matches_fp64(mode):
    g = torch.Generator(device="cpu").manual_seed(3)
    count = 5
    a = torch.randn((count, 128, 64), generator=g).cuda()
    b = torch.randn((count, 128, 64), generator=g).cuda()
    d = torch.full((count, 128, 128), float("nan"), device="cuda")
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    lib = _lib.load()
    st = lib.b2p_debug_tc_gemm(
        a.data_ptr(), b.data_ptr(), d.data_ptr(), count, _lib.MODES[mode], err.data_ptr(),
        ctypes.c_void_p(torch.cuda.current_stream().cuda_stream),
    )
    assert st == 0, lib.b2p_last_error()
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    want = a.double() @ b.double().transpose(-1, -2)
    assert torch.isfinite(d).all()
    assert _rel_fro(d.double(), want) <= TOL_GEMM[mode]


@pytest.mark.parametrize("mode", ["tf32", "bf16x3"])
@pytest.mark.parametrize("batch,n", [(6, 200), (3, 384), (2, 700), (20, 512), (4, 1024)])
def test_factor_residual(mode, batch, n):
    a = inputs.well_conditioned(batch, n, seed=n + 1, device="cuda")
    info = torch.full((batch,), -9, dtype=torch.int32, device="cuda")
    l = cholesky(a, mode=mode, info=info)
    assert (info == 0).all()
    assert (torch.triu(l, 1) == 0).all()
    assert (torch.diagonal(l, dim1=-2, dim2=-1) > 0).all()
    ld, ad = l.double(), a.double()
    r = torch.linalg.matrix_norm(ld @ ld.transpose(-1, -2) - ad) / torch.linalg.matrix_norm(ad)
    assert r.max().item() <= TOL_FACTOR[mode]


@pytest.mark.parametrize("batch,n", [(6, 200), (4, 512)])
def test_bf16x3_passes_reference_checker(batch, n):
    a = inputs.generate_input(batch, n, 2, 77 + n, "dense", device="cpu")
    l = cholesky(a.cuda(), mode="bf16x3").cpu().numpy()
    ok, msg = oracle.check_implementation(a.numpy(), l)
    assert ok, msg


def test_bf16x3_close_to_fp32_mode():
    a = inputs.mixed_batch(8, 512, seed=5, device="cuda")
    l32 = cholesky(a, mode="fp32")
    lbf = cholesky(a, mode="bf16x3")
    assert _rel_fro(lbf.double(), l32.double()) < 1e-3
    l64, _ = oracle.potrf_f64(a[:4].cpu().numpy())
    e32 = np.linalg.norm(l32[:4].cpu().numpy() - l64) / np.linalg.norm(l64)
    ebf = np.linalg.norm(lbf[:4].cpu().numpy() - l64) / np.linalg.norm(l64)
    assert ebf < 50 * e32 + 1e-6


@pytest.mark.parametrize("mode", ["tf32", "bf16x3"])
def test_tensor_modes_repeat_bitwise(mode):
    a = inputs.well_conditioned(10, 320, seed=9, device="cuda")
    assert torch.equal(cholesky(a, mode=mode), cholesky(a, mode=mode))
