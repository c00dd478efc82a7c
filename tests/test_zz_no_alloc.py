"""GPU: the allocation-free entry point against the regular one.

b2p_potrf_batched_noalloc serves callers that cannot allocate device memory
(allocator-free host loops, plugins whose host owns all device memory,
serving processes that forbid allocation after start-up): it keeps its
scratch in a fixed 16 MiB device array inside the library instead of a
caller-provided workspace.  This file is collected last so that a failure
here stops a `-x` run only after every other test has run.
"""

from __future__ import annotations

import ctypes

import pytest
import torch

from gpumode_cholesky_b200 import _lib, cholesky, inputs

pytestmark = pytest.mark.gpu

# Same tolerance as the other parity tests: relative Frobenius difference.
REL_TOL = 2e-5


def _call_noalloc(a: torch.Tensor, out: torch.Tensor, info: torch.Tensor, mode: int = _lib.MODE_FP32) -> int:
    lib = _lib.load()
    return lib.b2p_potrf_batched_noalloc(
        a.data_ptr(),
        out.data_ptr(),
        a.shape[0],
        a.shape[1],
        mode,
        info.data_ptr(),
        ctypes.c_void_p(torch.cuda.current_stream().cuda_stream),
    )


def _rel(x: torch.Tensor, y: torch.Tensor) -> float:
    return float((torch.linalg.matrix_norm(x - y) / torch.linalg.matrix_norm(y)).max())


# FP32: the blocked path (48x320, 5x1000) and the one-CTA kernel (128x64,
# no scratch).  BF16x3 at orders that are multiples of 64: the fused kernel
# whose last, small wave goes to the warp-specialized kernel at an offset
# into the scratch (300x192), the warp-specialized kernel alone (8x512,
# 2x1024) and the split path (1x2048).
CASES = [
    (48, 320, "fp32"),
    (5, 1000, "fp32"),
    (128, 64, "fp32"),
    (300, 192, "bf16x3"),
    (8, 512, "bf16x3"),
    (2, 1024, "bf16x3"),
    (1, 2048, "bf16x3"),
]


@pytest.mark.parametrize("batch,n,mode", CASES)
def test_noalloc_matches_regular_entry_point_twice(batch, n, mode):
    torch.cuda.set_device(0)
    for call, seed in enumerate((11 + n, 23 + n)):  # two calls in a row, different inputs
        a = inputs.generate_input(batch, n, 2, seed, "dense", device="cpu").cuda()
        want = cholesky(a, mode=mode)
        got = torch.full_like(a, float("nan"))
        info = torch.full((batch,), -1, dtype=torch.int32, device="cuda")
        st = _call_noalloc(a, got, info, _lib.MODES[mode])
        assert st == _lib.B2P_OK, _lib.load().b2p_last_error()
        torch.cuda.synchronize()
        assert torch.isfinite(got).all(), f"call {call}"
        assert _rel(got, want) <= REL_TOL, f"call {call}"
        assert (info == 0).all()


def test_noalloc_rejects_batches_beyond_its_scratch():
    lib = _lib.load()
    cap = lib.b2p_noalloc_scratch_bytes()
    assert cap == 16 << 20
    max_batch = cap // (64 * 64 * 4)
    a = torch.empty((1, 200, 200), device="cuda")
    st = lib.b2p_potrf_batched_noalloc(a.data_ptr(), a.data_ptr(), max_batch + 1, 200, 0, None, None)
    assert st == _lib.B2P_ERR_WORKSPACE
    assert b"allocation-free" in lib.b2p_last_error()
    assert b"at most 1024 matrices" in lib.b2p_last_error()
    # Tensor modes keep every panel's operand copy: 40 matrices of order 512
    # need more than the scratch holds, and the message names the 36 that fit.
    st = lib.b2p_potrf_batched_noalloc(a.data_ptr(), a.data_ptr(), 40, 512, _lib.MODE_BF16X3, None, None)
    assert st == _lib.B2P_ERR_WORKSPACE
    assert b"at most 36 matrices" in lib.b2p_last_error()
