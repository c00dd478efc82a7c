"""GPU: the host-buffer entry point (cholesky_host / b2p_potrf_batched_host).

Each chunk is one b2p_potrf_batched call with the chunk's own batch size, so
the host result must equal, bit for bit, device calls over the same chunks;
it must also pass the restated reference checker (scaled residual <= 20).
"""

from __future__ import annotations

import numpy as np
import pytest
import torch

import oracle
from gpumode_cholesky_b200 import cholesky, cholesky_host, inputs

pytestmark = pytest.mark.gpu


def _device_by_chunks(a: torch.Tensor, mode, chunk: int) -> torch.Tensor:
    d = a.cuda()
    out = torch.empty_like(d)
    for c0 in range(0, d.shape[0], chunk):
        cholesky(d[c0 : c0 + chunk], mode=mode, out=out[c0 : c0 + chunk])
    return out.cpu()


@pytest.mark.parametrize(
    "batch,n,mode,chunk",
    [
        (300, 32, None, 64),  # warp kernel, ragged last chunk
        (40, 100, None, 16),  # one CTA per matrix
        (37, 256, "auto", 5),  # tensor-core path, last chunk of 2
        (9, 1024, "auto", 4),  # clustered CTAs per matrix
        (20, 300, "fp32", 6),  # blocked FP32, n not a multiple of 64
        (3, 2048, "auto", 1),  # multi-CTA split path, one matrix per chunk
    ],
)
def test_chunks_match_device_calls(batch, n, mode, chunk):
    a = inputs.generate_input(batch, n, 2, 4000 + n, "dense", device="cpu").pin_memory()
    l = cholesky_host(a, mode=mode, chunk=chunk)
    assert l.is_pinned() and not l.is_cuda
    ref = _device_by_chunks(a, mode, min(chunk, batch))
    assert torch.equal(l, ref)
    ok, msg = oracle.check_implementation(a.numpy(), l.numpy())
    assert ok, msg


def test_default_chunking_and_pageable_buffers():
    a = inputs.generate_input(96, 512, 2, 77, "dense", device="cpu")
    # 96 MB: the default takes four chunks of 24 matrices.
    pinned = cholesky_host(a.pin_memory(), mode="auto")
    assert torch.equal(pinned, _device_by_chunks(a, "auto", 24))
    out = torch.empty_like(a)  # pageable input and output: copies serialise, same result
    pageable = cholesky_host(a, mode="auto", out=out)
    assert pageable.data_ptr() == out.data_ptr()
    assert torch.equal(pageable, pinned)


def test_info_offsets_and_non_blocking():
    batch, n, chunk = 12, 256, 5
    a = inputs.generate_input(batch, n, 2, 91, "dense", device="cpu")
    a[7] = -a[7]  # not SPD: fails at the first pivot, in the second chunk
    a = a.pin_memory()
    info = torch.full((batch,), -9, dtype=torch.int32, device="cuda")
    out = torch.empty_like(a).pin_memory()
    cholesky_host(a, mode="auto", out=out, info=info, chunk=chunk, non_blocking=True)
    torch.cuda.current_stream().synchronize()
    _, want = oracle.potrf_f64(a.numpy())
    assert want[7] > 0 and np.array_equal(info.cpu().numpy(), want)
    good = [i for i in range(batch) if i != 7]
    ref = _device_by_chunks(a, "auto", chunk)
    assert torch.equal(out[good], ref[good])


def test_back_to_back_calls_share_the_workspace():
    # Two calls enqueued without a host sync in between, different shapes:
    # the second's copies start after the first's, on the same workspace.
    a1 = inputs.generate_input(50, 512, 2, 5, "dense", device="cpu").pin_memory()
    a2 = inputs.generate_input(6, 1024, 2, 6, "dense", device="cpu").pin_memory()
    o1 = torch.empty_like(a1).pin_memory()
    o2 = torch.empty_like(a2).pin_memory()
    cholesky_host(a1, mode="auto", out=o1, chunk=8, non_blocking=True)
    cholesky_host(a2, mode="auto", out=o2, chunk=2, non_blocking=True)
    torch.cuda.current_stream().synchronize()
    assert torch.equal(o1, _device_by_chunks(a1, "auto", 8))
    assert torch.equal(o2, _device_by_chunks(a2, "auto", 2))
