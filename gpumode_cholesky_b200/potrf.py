"""Host side of the batched Cholesky: the reference-facing ``custom_kernel``.

``custom_kernel(data) -> output`` keeps the reference's contract
(submission.py:4101-4268, reference/task.py:6-7, reference/eval.py:107-113):
``data`` is a (batch, n, n) FP32 CUDA tensor of SPD matrices, never mutated;
the result is a fresh tensor of the same shape, dtype and device holding L
(lower triangle, positive diagonal, exact zeros above).  Unlike the reference
there is no CPU path and no cuSOLVER fallback: a non-CUDA or non-FP32 input
raises, and a failing library call raises :class:`PotrfError`.
"""

from __future__ import annotations

import torch

from . import _lib

_WS: dict[tuple[int, int], torch.Tensor] = {}


def _stream_ptr(device: torch.device) -> int:
    return torch.cuda.current_stream(device).cuda_stream


def workspace(device: torch.device, nbytes: int) -> torch.Tensor:
    """Per-(device, stream) scratch buffer grown on demand, 256-byte aligned.

    Calls that share a stream are ordered by it, so one buffer per stream is
    safe; callers running several streams get one buffer each.
    """
    key = (device.index if device.index is not None else torch.cuda.current_device(), _stream_ptr(device))
    buf = _WS.get(key)
    if buf is None or buf.numel() < nbytes:
        buf = torch.empty(max(nbytes, 256), dtype=torch.uint8, device=device)
        _WS[key] = buf
    return buf


def resolve_mode(mode: str | int | None, n: int) -> int:
    """Precision mode code for order n; None picks the library default (FP32).

    A name is a mode ("fp32", "tf32", "bf16x3", "fp8") optionally followed by
    flags ("+fp64diag", "+guard").  "auto" is BF16x3 trailing updates with
    the pivot guard for n > 128 when n is a multiple of 64 (the mixed form
    that meets the 1e-5 relative residual; the guard recomputes in FP32 the
    columns whose pivots the mixed update cannot resolve), and FP32
    otherwise (orders <= 128 have no blocked update; other orders take the
    blocked path, which has no guard).
    """
    if mode is None:
        return _lib.MODE_FP32
    if isinstance(mode, int):
        return mode
    name, *flags = mode.lower().split("+")
    if name == "auto" and not flags:
        return (_lib.MODE_BF16X3 | _lib.FLAG_GUARD) if n > 128 and n % 64 == 0 else _lib.MODE_FP32
    if name not in _lib.MODES:
        raise ValueError(f"unknown precision mode {mode!r}; expected one of {sorted(_lib.MODES)}")
    code = _lib.MODES[name]
    for f in flags:
        if f not in _lib.FLAGS:
            raise ValueError(f"unknown mode flag {f!r} in {mode!r}; expected one of {sorted(_lib.FLAGS)}")
        code |= _lib.FLAGS[f]
    return code


def _check_input(a: torch.Tensor) -> None:
    if not isinstance(a, torch.Tensor):
        raise TypeError("input must be a torch.Tensor")
    if a.dim() != 3 or a.shape[-1] != a.shape[-2]:
        raise ValueError(f"input must have shape (batch, n, n), got {tuple(a.shape)}")
    if a.dtype != torch.float32:
        raise TypeError(f"input dtype must be torch.float32, got {a.dtype}")
    if not a.is_cuda:
        raise RuntimeError("input must be a CUDA tensor: this library has no CPU path")


def cholesky(
    a: torch.Tensor,
    mode: str | int | None = None,
    out: torch.Tensor | None = None,
    info: torch.Tensor | None = None,
    path: str = "auto",
    fp32_from: torch.Tensor | None = None,
) -> torch.Tensor:
    """Factor a batch of SPD matrices: returns L with A = L L^T.

    ``mode`` selects the trailing-update arithmetic ("fp32", "tf32",
    "bf16x3", "fp8", optionally suffixed "+fp64diag" and/or "+guard"; "auto"
    is "bf16x3+guard" for orders > 128 that are multiples of 64, else
    "fp32").  ``info`` may be an int32 CUDA tensor of shape (batch,) that
    receives 0 or the 1-based index of the first non-positive pivot.
    ``fp32_from`` may be an int32 CUDA tensor of shape (batch,) that receives
    the first 64-wide block column the pivot guard recomputed in FP32, or -1.
    ``path`` forces the algorithm for n > 128 ("blocked", "fused",
    "fused_ws", "split"; default "auto").
    """
    if path not in _lib.PATHS:
        raise ValueError(f"unknown path {path!r}; expected one of {sorted(_lib.PATHS)}")
    pcode = _lib.PATHS[path]
    _check_input(a)
    a = a.contiguous()
    batch, n, _ = a.shape
    code = resolve_mode(mode, n)
    if out is None:
        out = torch.empty_like(a)
    elif out.shape != a.shape or out.dtype != torch.float32 or not out.is_contiguous() or out.device != a.device:
        raise ValueError("out must be a contiguous float32 tensor shaped like the input, on the same device")
    lib = _lib.load()
    with torch.cuda.device(a.device):
        ws_bytes = lib.b2p_potrf_path_workspace_size(batch, n, code, pcode)
        ws_ptr = workspace(a.device, ws_bytes).data_ptr() if ws_bytes else None
        info_ptr = None
        if info is not None:
            if info.dtype != torch.int32 or info.numel() < batch or not info.is_cuda:
                raise ValueError("info must be an int32 CUDA tensor with at least batch elements")
            info_ptr = info.data_ptr()
        from_ptr = None
        if fp32_from is not None:
            if fp32_from.dtype != torch.int32 or fp32_from.numel() < batch or not fp32_from.is_cuda:
                raise ValueError("fp32_from must be an int32 CUDA tensor with at least batch elements")
            from_ptr = fp32_from.data_ptr()
        st = lib.b2p_potrf_batched_ex(
            a.data_ptr(), out.data_ptr(), batch, n, code, pcode, ws_ptr, ws_bytes, info_ptr, from_ptr,
            _stream_ptr(a.device),
        )
    _lib.check(st, "b2p_potrf_batched_ex")
    return out


def cholesky_host(
    a: torch.Tensor,
    mode: str | int | None = None,
    out: torch.Tensor | None = None,
    info: torch.Tensor | None = None,
    chunk: int = 0,
    non_blocking: bool = False,
) -> torch.Tensor:
    """Factor a batch held in host memory into host memory on the current GPU.

    The batch streams through the device in chunks of ``chunk`` matrices
    (0: about 32 MiB each, at least four): the copy in of the next chunk, the
    factorization of this one and the copy out of the previous one overlap
    (``b2p_potrf_batched_host``).  ``a`` and ``out`` should be pinned
    (``pin_memory()``) for the copies to overlap; ``out`` defaults to a new
    pinned tensor.  ``info`` is an optional int32 CUDA tensor as for
    :func:`cholesky`.  With ``non_blocking`` the call only enqueues, like
    ``Tensor.copy_(..., non_blocking=True)``: ``out`` holds L once the
    current stream is synchronised, and ``a`` and ``out`` must be kept
    alive until then.
    """
    if not isinstance(a, torch.Tensor):
        raise TypeError("input must be a torch.Tensor")
    if a.dim() != 3 or a.shape[-1] != a.shape[-2]:
        raise ValueError(f"input must have shape (batch, n, n), got {tuple(a.shape)}")
    if a.dtype != torch.float32:
        raise TypeError(f"input dtype must be torch.float32, got {a.dtype}")
    if a.is_cuda:
        raise ValueError("cholesky_host takes a host tensor; use cholesky() for a CUDA tensor")
    if chunk < 0:
        raise ValueError("chunk must be >= 0")
    a = a.contiguous()
    batch, n, _ = a.shape
    code = resolve_mode(mode, n)
    if out is None:
        out = torch.empty(a.shape, dtype=torch.float32, pin_memory=True)
    elif out.shape != a.shape or out.dtype != torch.float32 or not out.is_contiguous() or out.is_cuda:
        raise ValueError("out must be a contiguous float32 host tensor shaped like the input")
    device = torch.device("cuda", torch.cuda.current_device())
    info_ptr = None
    if info is not None:
        if info.dtype != torch.int32 or info.numel() < batch or not info.is_cuda:
            raise ValueError("info must be an int32 CUDA tensor with at least batch elements")
        info_ptr = info.data_ptr()
    lib = _lib.load()
    ws_bytes = lib.b2p_potrf_host_workspace_size(batch, n, code, chunk)
    ws_ptr = workspace(device, ws_bytes).data_ptr() if ws_bytes else None
    st = lib.b2p_potrf_batched_host(
        a.data_ptr(), out.data_ptr(), batch, n, code, chunk, ws_ptr, ws_bytes, info_ptr, _stream_ptr(device)
    )
    _lib.check(st, "b2p_potrf_batched_host")
    if not non_blocking:
        torch.cuda.current_stream(device).synchronize()
    return out


def residual_estimate(a: torch.Tensor, l: torch.Tensor, probes: int = 4, seed: int = 0) -> torch.Tensor:
    """Per-matrix estimate of ||L L^T - A||_F / ||A||_F from random probes, in FP64.

    For V with ``probes`` N(0, 1) columns, E[||(L L^T - A) V||_F^2] equals
    probes * ||L L^T - A||_F^2, so ||L (L^T V) - A V||_F / (sqrt(probes)
    ||A||_F) estimates the relative residual at O(probes * n^2) per matrix
    instead of the n^3 of forming L L^T.  A non-finite factor gives inf.
    ``probes=0`` forms L L^T exactly in FP64 instead.
    """
    if probes == 0:
        from .checker import residual_norms

        return residual_norms(a, l, precision="fp64")["rel_fro"]
    batch, n, _ = a.shape
    gen = torch.Generator(device=a.device)
    gen.manual_seed(seed)
    out = torch.empty(batch, dtype=torch.float64, device=a.device)
    step = max(1, (1 << 28) // max(1, n * n))  # slices of about 2 GiB of FP64 factor
    for b0 in range(0, batch, step):
        ld = l[b0 : b0 + step].double()
        ad = a[b0 : b0 + step].double()
        v = torch.randn((ld.shape[0], n, probes), dtype=torch.float64, device=a.device, generator=gen)
        r = torch.matmul(ld, torch.matmul(ld.transpose(-1, -2), v)) - torch.matmul(ad, v)
        est = torch.linalg.matrix_norm(r) / (probes**0.5 * torch.linalg.matrix_norm(ad).clamp_min(1e-300))
        out[b0 : b0 + ld.shape[0]] = torch.where(torch.isfinite(est), est, torch.full_like(est, float("inf")))
    return out


def cholesky_checked(
    a: torch.Tensor,
    mode: str | int | None = "bf16x3",
    tol: float = 1.0e-5,
    probes: int = 4,
    info: torch.Tensor | None = None,
    out: torch.Tensor | None = None,
) -> tuple[torch.Tensor, torch.Tensor]:
    """Factor in ``mode``, then refactor in FP32 every matrix whose factor fails a residual check.

    A matrix is refactored when its pivot check fails (``info`` != 0) or its
    relative residual (:func:`residual_estimate`, ``probes`` random vectors;
    0 for the exact FP64 check) exceeds ``tol`` or is not finite.  The
    mixed modes keep their speed on the matrices they factor well, and
    ill-conditioned ones fall back to the FP32 path of this library, not to
    a CPU or vendor routine.  Returns (L, redone): ``redone`` is a bool CUDA
    tensor marking the refactored matrices.  Synchronises the host once, to
    learn whether any matrix needs the FP32 pass.
    """
    _check_input(a)
    a = a.contiguous()
    batch = a.shape[0]
    own_info = torch.zeros(batch, dtype=torch.int32, device=a.device)
    l = cholesky(a, mode=mode, out=out, info=own_info)
    est = residual_estimate(a, l, probes=probes)
    redone = (own_info != 0) | ~(est <= tol)
    idx = redone.nonzero().flatten()
    if idx.numel() > 0:
        sub_info = torch.zeros(idx.numel(), dtype=torch.int32, device=a.device)
        sub = cholesky(a.index_select(0, idx), mode="fp32", info=sub_info)
        l.index_copy_(0, idx, sub)
        own_info.index_copy_(0, idx, sub_info)
    if info is not None:
        if info.dtype != torch.int32 or info.numel() < batch or not info.is_cuda:
            raise ValueError("info must be an int32 CUDA tensor with at least batch elements")
        info[:batch].copy_(own_info)
    return l, redone


def custom_kernel(data: torch.Tensor) -> torch.Tensor:
    """Drop-in for the reference entry point ``custom_kernel`` (submission.py:4101).

    One library call on the current stream, no host synchronisation, in the
    "auto" mode: BF16x3 trailing updates with the pivot guard for orders
    > 128 that are multiples of 64 (the reference likewise routes its
    benchmark shapes to mixed TF32/FP16/FP8 products), plain FP32 otherwise.
    ``cholesky(data, mode="fp32")`` is the plain FP32 method.
    """
    return cholesky(data, mode="auto")
