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


def _call_noalloc(a: torch.Tensor, out: torch.Tensor, info: torch.Tensor) -> int:
    lib = _lib.load()
    return lib.b2p_potrf_batched_noalloc(
        a.data_ptr(),
        out.data_ptr(),
        a.shape[0],
        a.shape[1],
        _lib.MODE_FP32,
        info.data_ptr(),
        ctypes.c_void_p(torch.cuda.current_stream().cuda_stream),
    )


def _rel(x: torch.Tensor, y: torch.Tensor) -> float:
    return float((torch.linalg.matrix_norm(x - y) / torch.linalg.matrix_norm(y)).max())


@pytest.mark.parametrize("batch,n", [(48, 320), (5, 1000), (128, 64)])
def test_noalloc_matches_regular_entry_point_twice(batch, n):
    torch.cuda.set_device(0)
    for call, seed in enumerate((11 + n, 23 + n)):  # two calls in a row, different inputs
        a = inputs.generate_input(batch, n, 2, seed, "dense", device="cpu").cuda()
        want = cholesky(a)
        got = torch.full_like(a, float("nan"))
        info = torch.full((batch,), -1, dtype=torch.int32, device="cuda")
        st = _call_noalloc(a, got, info)
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
