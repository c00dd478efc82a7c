"""GPU: the error path of the bounded device-side waits.

Every wait in the library's kernels (mbarrier phases of the tensor-core
pipelines, progress counters, grid barriers) gives up after a bounded
number of polls, reports B2P_ERR_TIMEOUT (or info = -1), lets whatever it
issued finish, releases its tensor memory and returns.  The diagnostic
b2p_debug_tc_gemm_stall makes such a wait run out on purpose -- a wait on an
mbarrier that nothing arrives on, bounded by the caller -- so the test sees:
  * the status in the caller's error word;
  * the work done before the wait (each CTA's first 128x64 pair) is correct;
  * the context stays usable: the same kernel without the stall and a
    factorization give correct results right after.
No fault, trap or endless loop is involved.
"""

from __future__ import annotations

import ctypes

import pytest
import torch

from gpumode_cholesky_b200 import _lib, cholesky, inputs

pytestmark = pytest.mark.gpu


def _stream() -> ctypes.c_void_p:
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


@pytest.mark.parametrize("mode", [_lib.MODE_BF16X3, _lib.MODE_TF32])
def test_bounded_wait_runs_out_and_reports_timeout(mode):
    lib = _lib.load()
    count = 4  # fewer pairs than SMs: every CTA computes one pair, then stalls
    g = torch.Generator(device="cuda").manual_seed(3)
    a = torch.randn(count, 128, 64, device="cuda", generator=g)
    b = torch.randn(count, 128, 64, device="cuda", generator=g)
    want = (a.double() @ b.double().transpose(-1, -2)).float()
    tol = 1e-5 if mode == _lib.MODE_BF16X3 else 2e-3

    d = torch.full((count, 128, 128), float("nan"), device="cuda")
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    st = lib.b2p_debug_tc_gemm_stall(a.data_ptr(), b.data_ptr(), d.data_ptr(), count, mode, 1000, err.data_ptr(), _stream())
    assert st == _lib.B2P_OK, lib.b2p_last_error()
    torch.cuda.synchronize()
    assert err.item() == _lib.B2P_ERR_TIMEOUT
    assert (torch.linalg.matrix_norm(d - want) / torch.linalg.matrix_norm(want)).max().item() <= tol

    # The context is intact: the kernel without the stall, then a factorization.
    d.fill_(float("nan"))
    err.zero_()
    st = lib.b2p_debug_tc_gemm(a.data_ptr(), b.data_ptr(), d.data_ptr(), count, mode, err.data_ptr(), _stream())
    assert st == _lib.B2P_OK
    torch.cuda.synchronize()
    assert err.item() == 0
    assert (torch.linalg.matrix_norm(d - want) / torch.linalg.matrix_norm(want)).max().item() <= tol
    m = inputs.well_conditioned(4, 512, seed=9, device="cuda")
    l = cholesky(m, mode="bf16x3")
    r = torch.linalg.matrix_norm(l.double() @ l.double().transpose(-1, -2) - m.double()) / torch.linalg.matrix_norm(m.double())
    assert r.max().item() <= 1e-5
