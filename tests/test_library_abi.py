"""CPU: the C-ABI library builds, loads and exports every declared symbol.

No compute call is made here (there is no GPU); only entry points that
return before touching the device are exercised.
"""

from __future__ import annotations

import ctypes
import re
import subprocess
from pathlib import Path

import pytest

from gpumode_cholesky_b200 import _lib, build
from gpumode_cholesky_b200.potrf import resolve_mode

ROOT = Path(__file__).resolve().parent.parent


def _declared_symbols() -> set[str]:
    names = set()
    for h in (ROOT / "include").glob("*.h"):
        names |= set(re.findall(r"B2P_API\s+[\w\s\*]+?\b(b2p_\w+)\s*\(", h.read_text()))
    return names


def test_header_declares_entry_points():
    names = _declared_symbols()
    assert {"b2p_potrf_batched", "b2p_potrf_ragged", "b2p_potrf_backward", "b2p_potrf_workspace_size"} <= names


def test_library_exports_every_declared_symbol():
    build.build()
    out = subprocess.run(["nm", "-D", "--defined-only", str(build.LIB_PATH)], capture_output=True, text=True, check=True)
    exported = {line.split()[-1] for line in out.stdout.splitlines() if " T " in line}
    missing = _declared_symbols() - exported
    assert not missing, f"declared but not exported: {sorted(missing)}"
    assert set(_lib.SIGNATURES) == _declared_symbols()


def test_library_loads_and_reports_version():
    lib = _lib.load()
    assert lib.b2p_version() >= 100
    assert lib.b2p_status_string(_lib.B2P_OK) == b"ok"
    assert lib.b2p_status_string(_lib.B2P_ERR_WORKSPACE).startswith(b"workspace")
    assert lib.b2p_status_string(99) == b"unknown status"


def test_argument_validation_without_device():
    lib = _lib.load()
    # empty batch: nothing to do, no device call
    assert lib.b2p_potrf_batched(None, None, 0, 32, 0, None, 0, None, None) == _lib.B2P_OK
    # negative sizes and unknown modes are rejected before any CUDA call
    assert lib.b2p_potrf_batched(None, None, -1, 32, 0, None, 0, None, None) == _lib.B2P_ERR_INVALID_ARG
    assert lib.b2p_potrf_batched(None, None, 1, -3, 0, None, 0, None, None) == _lib.B2P_ERR_INVALID_ARG
    assert lib.b2p_potrf_batched(None, None, 1, 32, 0x77, None, 0, None, None) == _lib.B2P_ERR_INVALID_ARG
    assert b"mode" in lib.b2p_last_error()
    assert lib.b2p_potrf_batched(None, None, 1, 32, 0, None, 0, None, None) == _lib.B2P_ERR_INVALID_ARG
    # misaligned pointers
    assert lib.b2p_potrf_batched(ctypes.c_void_p(8), ctypes.c_void_p(4096), 1, 32, 0, None, 0, None, None) == _lib.B2P_ERR_INVALID_ARG
    # overlapping buffers
    assert lib.b2p_potrf_batched(ctypes.c_void_p(4096), ctypes.c_void_p(4096 + 64), 1, 32, 0, None, 0, None, None) == _lib.B2P_ERR_INVALID_ARG
    assert b"overlap" in lib.b2p_last_error()


def test_host_entry_layout_and_validation_without_device():
    """b2p_potrf_batched_host: chunk layout and the checks made before any CUDA call."""
    lib = _lib.load()
    bf = _lib.MODE_BF16X3
    mib = 1 << 20
    # One chunk (3 small matrices): one input and one output buffer, no factorization workspace.
    assert lib.b2p_potrf_host_workspace_size(3, 16, 0, 0) == 2 * 3 * 16 * 16 * 4
    # 640 x 512 by default: 32 MiB chunks of 32 matrices, two buffers per direction,
    # plus the factorization's workspace for one chunk.
    ws = lib.b2p_potrf_host_workspace_size(640, 512, bf, 0)
    assert ws == 4 * 32 * mib + lib.b2p_potrf_workspace_size(32, 512, bf)
    # An explicit chunk that does not divide the batch: the larger of the two chunk workspaces.
    ws7 = lib.b2p_potrf_host_workspace_size(20, 256, bf, 7)
    need = max(lib.b2p_potrf_workspace_size(7, 256, bf), lib.b2p_potrf_workspace_size(6, 256, bf))
    assert ws7 == 4 * 7 * 256 * 256 * 4 + (need + 255) // 256 * 256
    # A chunk at least the batch is one chunk.
    assert lib.b2p_potrf_host_workspace_size(4, 64, 0, 100) == 2 * 4 * 64 * 64 * 4
    assert lib.b2p_potrf_host_workspace_size(0, 64, 0, 0) == 0
    assert lib.b2p_potrf_host_workspace_size(4, 64, 0, -1) == 0

    host = ctypes.create_string_buffer(2 * 4 * 64 * 64 * 4 + 512)
    base = (ctypes.addressof(host) + 255) // 256 * 256
    a, l = ctypes.c_void_p(base), ctypes.c_void_p(base + 4 * 64 * 64 * 4)
    call = lib.b2p_potrf_batched_host
    assert call(None, None, 0, 64, 0, 0, None, 0, None, None) == _lib.B2P_OK
    assert call(a, l, 4, 64, 0, -2, None, 0, None, None) == _lib.B2P_ERR_INVALID_ARG
    assert call(a, l, 4, 64, 0x77, 0, None, 0, None, None) == _lib.B2P_ERR_INVALID_ARG
    assert call(None, l, 4, 64, 0, 0, None, 0, None, None) == _lib.B2P_ERR_INVALID_ARG
    assert call(a, ctypes.c_void_p(base + 64), 4, 64, 0, 0, None, 0, None, None) == _lib.B2P_ERR_INVALID_ARG
    assert b"overlap" in lib.b2p_last_error()
    assert call(a, l, 4, 64, 0, 0, None, 0, None, None) == _lib.B2P_ERR_WORKSPACE
    assert str(2 * 4 * 64 * 64 * 4).encode() in lib.b2p_last_error()
    assert call(a, l, 4, 64, 0, 0, ctypes.c_void_p(base + 16), 1 << 20, None, None) == _lib.B2P_ERR_INVALID_ARG
    assert b"256-byte" in lib.b2p_last_error()


def test_host_workspace_matches_the_chunk_model():
    """The host entry's workspace: 2 buffers per direction (1 for one chunk) + one chunk's factor workspace."""
    import random

    lib = _lib.load()
    rng = random.Random(3)
    mib = 1 << 20
    for _ in range(300):
        n = rng.choice([1, 8, 32, 33, 64, 100, 128, 129, 256, 512, 640, 1024, 2048])
        batch = rng.randint(1, 3000)
        mode = rng.choice([_lib.MODE_FP32, _lib.MODE_TF32, _lib.MODE_BF16X3])
        chunk = rng.choice([0, 0, 1, 5, 64, 5000])
        mat = n * n * 4
        c = chunk
        if c == 0:
            c = max(1, max(4 * mib, min(32 * mib, batch * mat // 4)) // mat)
        c = min(c, batch)
        nchunks = -(-batch // c)
        nbuf = 2 if nchunks > 1 else 1
        buf = -(-c * mat // 256) * 256
        last = batch - (nchunks - 1) * c
        fw = max(lib.b2p_potrf_workspace_size(c, n, mode), lib.b2p_potrf_workspace_size(last, n, mode))
        want = 2 * nbuf * buf + -(-fw // 256) * 256
        assert lib.b2p_potrf_host_workspace_size(batch, n, mode, chunk) == want, (batch, n, mode, chunk)


def test_cholesky_host_rejects_device_and_bad_arguments():
    import torch

    from gpumode_cholesky_b200 import cholesky_host

    with pytest.raises(TypeError):
        cholesky_host(torch.zeros(2, 8, 8, dtype=torch.float64))
    with pytest.raises(ValueError):
        cholesky_host(torch.zeros(2, 8, 7))
    with pytest.raises(ValueError):
        cholesky_host(torch.zeros(2, 8, 8), chunk=-1)
    with pytest.raises(ValueError):
        cholesky_host(torch.zeros(2, 8, 8), out=torch.zeros(2, 8, 8, dtype=torch.float64))


def test_workspace_sizes_are_host_only():
    lib = _lib.load()
    assert lib.b2p_potrf_workspace_size(4096, 32, 0) == 0
    assert lib.b2p_potrf_workspace_size(256, 128, 0) == 0
    assert lib.b2p_potrf_workspace_size(640, 512, 0) >= 640 * 64 * 64 * 4
    assert lib.b2p_potrf_workspace_size(0, 512, 0) == 0


def test_path_workspace_sizes():
    """Forced paths: a path that cannot run (n, mode) reports 0 bytes."""
    lib = _lib.load()
    p = _lib.PATHS
    bf = _lib.MODE_BF16X3
    assert lib.b2p_potrf_path_workspace_size(4, 2048, bf, p["fused"]) == 0  # one CTA per matrix stops at 1024
    assert lib.b2p_potrf_path_workspace_size(4, 200, bf, p["split"]) == 0  # needs n % 64 == 0
    assert lib.b2p_potrf_path_workspace_size(4, 512, _lib.MODE_FP32, p["split"]) == 0  # tensor modes only
    assert lib.b2p_potrf_path_workspace_size(4, 512, bf, p["blocked"]) > 0
    assert lib.b2p_potrf_path_workspace_size(4, 512, bf, p["split"]) > lib.b2p_potrf_path_workspace_size(4, 512, bf, p["fused"])
    assert lib.b2p_potrf_path_workspace_size(4, 64, bf, p["split"]) == 0  # n <= 128 needs none
    # an unknown path is rejected before any device work
    assert lib.b2p_potrf_batched_path(ctypes.c_void_p(4096), ctypes.c_void_p(1 << 30), 1, 512, bf, 9, None, 0, None, None) == _lib.B2P_ERR_INVALID_ARG


def test_error_raises_python_exception():
    with pytest.raises(_lib.PotrfError) as ei:
        _lib.check(_lib.B2P_ERR_UNSUPPORTED, "call")
    assert ei.value.status == _lib.B2P_ERR_UNSUPPORTED


def test_mode_names():
    assert resolve_mode(None, 512) == _lib.MODE_FP32
    assert resolve_mode("bf16x3", 512) == _lib.MODE_BF16X3
    # auto: BF16x3 with the pivot guard where the guarded paths run (orders
    # > 128, multiples of 64), FP32 elsewhere.
    assert resolve_mode("auto", 512) == _lib.MODE_BF16X3 | _lib.FLAG_GUARD
    assert resolve_mode("auto", 300) == _lib.MODE_FP32
    assert resolve_mode("auto", 128) == _lib.MODE_FP32
    assert resolve_mode("tf32+fp64diag", 512) == _lib.MODE_TF32 | _lib.FLAG_FP64_DIAG
    assert resolve_mode("bf16x3+guard", 512) == _lib.MODE_BF16X3 | _lib.FLAG_GUARD
    assert resolve_mode("tf32+guard+fp64diag", 512) == _lib.MODE_TF32 | _lib.FLAG_GUARD | _lib.FLAG_FP64_DIAG
    with pytest.raises(ValueError):
        resolve_mode("int8", 512)
    with pytest.raises(ValueError):
        resolve_mode("bf16x3+fast", 512)


def test_custom_kernel_rejects_cpu_input():
    import torch

    from gpumode_cholesky_b200 import custom_kernel

    with pytest.raises(RuntimeError, match="no CPU path"):
        custom_kernel(torch.eye(4).expand(2, 4, 4).contiguous())
    with pytest.raises(TypeError):
        custom_kernel(torch.eye(4, dtype=torch.float64).expand(2, 4, 4).contiguous())


def test_trsv_and_gp_argument_validation_without_device():
    """The triangular-solve and GP entry points reject bad shapes and null
    pointers before any launch, and accept empty batches."""
    lib = _lib.load()
    fake = ctypes.c_void_p(16)  # never dereferenced: every call below returns first
    assert lib.b2p_trsv_batched(fake, fake, fake, 2, 40000, 0, None) == _lib.B2P_ERR_INVALID_ARG
    assert lib.b2p_trsv_batched(fake, fake, fake, -1, 8, 0, None) == _lib.B2P_ERR_INVALID_ARG
    assert lib.b2p_trsv_batched(None, fake, fake, 2, 8, 0, None) == _lib.B2P_ERR_INVALID_ARG
    assert lib.b2p_trsv_batched(None, None, None, 0, 8, 1, None) == _lib.B2P_OK
    assert lib.b2p_trsv_batched(None, None, None, 4, 0, 1, None) == _lib.B2P_OK
    assert lib.b2p_gp_nll_forward(fake, fake, fake, None, 2, 8, None) == _lib.B2P_ERR_INVALID_ARG
    assert lib.b2p_gp_nll_forward(fake, fake, fake, fake, 2, 32769, None) == _lib.B2P_ERR_INVALID_ARG
    assert lib.b2p_gp_nll_forward(None, None, None, None, 0, 8, None) == _lib.B2P_OK
    assert lib.b2p_gp_nll_backward(fake, fake, None, fake, fake, 2, 8, None) == _lib.B2P_ERR_INVALID_ARG
    assert lib.b2p_gp_nll_backward(fake, fake, fake, fake, None, 2, 8, None) == _lib.B2P_ERR_INVALID_ARG
    assert lib.b2p_gp_nll_backward(None, None, None, None, None, 0, 8, None) == _lib.B2P_OK
    assert lib.b2p_gp_nll_backward(fake, fake, fake, fake, None, 2, 8, None) == _lib.B2P_ERR_INVALID_ARG
    assert b"null" in lib.b2p_last_error()


def test_fp64_diag_flag_routes_to_blocked_workspace():
    """A flagged tensor-mode call takes the blocked path: its workspace is the
    blocked path's (one 64 x 64 FP32 inverse per matrix), not the panel copies."""
    lib = _lib.load()
    plain = lib.b2p_potrf_workspace_size(8, 512, _lib.MODE_BF16X3)
    flagged = lib.b2p_potrf_workspace_size(8, 512, _lib.MODE_BF16X3 | _lib.FLAG_FP64_DIAG)
    assert flagged == 8 * 64 * 64 * 4
    assert plain != flagged
    assert lib.b2p_potrf_workspace_size(8, 512, _lib.MODE_FP32 | _lib.FLAG_FP64_DIAG) == 8 * 64 * 64 * 4
