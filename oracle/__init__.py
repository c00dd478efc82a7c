"""CPU oracle for the batched Cholesky hot path -- TEST INFRASTRUCTURE ONLY.

Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` may import this package, and only as the checker or the timed
CPU baseline; the library (``gpumode_cholesky_b200``) never uses it.

Contents
  * :func:`potrf_f64` / :func:`potrf_f32` -- the reference's ``ref_kernel``
    (``torch.linalg.cholesky_ex(data).L``, reference/reference.py:129-130)
    restated in C as LAPACK's column Cholesky (``potrf_oracle.c``).
  * :func:`check_implementation` -- numpy restatement of the reference
    checker (reference/reference.py:137-188), same gates and message.
  * :func:`residuals` -- FP64 L1/Frobenius residuals per matrix.
  * :func:`potrf_backward_f64` -- FP64 Cholesky adjoint (no reference
    counterpart; pinned against torch autograd in the tests).
  * :func:`ref_kernel_cpu` -- the reference's CPU route itself
    (``torch.linalg.cholesky_ex`` in FP32), the timed CPU baseline.

Parity pin: ``tests/test_oracle.py`` checks these against the golden vectors
in ``tests/golden/`` that ``tests/golden/make_golden.py`` produced by running
the reference's own ``generate_input``/``ref_kernel``/``check_implementation``.
"""

from __future__ import annotations

import ctypes
import subprocess
import threading
from pathlib import Path

import numpy as np

_DIR = Path(__file__).resolve().parent
_LIB_PATH = _DIR / "liboracle_potrf.so"
_lock = threading.Lock()
_lib = None

_RECON_RTOL_FACTOR = 20.0  # reference/reference.py:6
_TRIANGULAR_RTOL_FACTOR = 8.0  # reference/reference.py:7
_EPS32 = float(np.finfo(np.float32).eps)
_TINY32 = float(np.finfo(np.float32).tiny)


def build() -> Path:
    """Compile the C restatement with gcc (``make -C oracle``)."""
    src = _DIR / "potrf_oracle.c"
    if _LIB_PATH.exists() and _LIB_PATH.stat().st_mtime >= src.stat().st_mtime:
        return _LIB_PATH
    res = subprocess.run(["make", "-C", str(_DIR)], capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"oracle build failed:\n{res.stdout}\n{res.stderr}")
    return _LIB_PATH


def _load():
    global _lib
    with _lock:
        if _lib is None:
            build()
            lib = ctypes.CDLL(str(_LIB_PATH))
            p, i64 = ctypes.c_void_p, ctypes.c_int64
            for name in ("oracle_potrf_f64", "oracle_potrf_f32"):
                fn = getattr(lib, name)
                fn.restype = ctypes.c_int
                fn.argtypes = [p, p, i64, i64, p]
            lib.oracle_residuals.restype = ctypes.c_int
            lib.oracle_residuals.argtypes = [p, p, i64, i64, p]
            lib.oracle_potrf_backward_f64.restype = ctypes.c_int
            lib.oracle_potrf_backward_f64.argtypes = [p, p, p, i64, i64]
            _lib = lib
        return _lib


def _as3(a: np.ndarray, dtype) -> np.ndarray:
    a = np.ascontiguousarray(a, dtype=dtype)
    if a.ndim == 2:
        a = a[None]
    if a.ndim != 3 or a.shape[1] != a.shape[2]:
        raise ValueError(f"expected (batch, n, n), got {a.shape}")
    return a


def potrf_f64(a: np.ndarray) -> tuple[np.ndarray, np.ndarray]:
    """FP64 lower Cholesky factor and LAPACK-style info per matrix."""
    a = _as3(a, np.float64)
    out = np.empty_like(a)
    info = np.zeros(a.shape[0], dtype=np.int32)
    _load().oracle_potrf_f64(a.ctypes.data, out.ctypes.data, a.shape[0], a.shape[1], info.ctypes.data)
    return out, info


def potrf_f32(a: np.ndarray) -> tuple[np.ndarray, np.ndarray]:
    """Same algorithm in FP32 arithmetic."""
    a = _as3(a, np.float32)
    out = np.empty_like(a)
    info = np.zeros(a.shape[0], dtype=np.int32)
    _load().oracle_potrf_f32(a.ctypes.data, out.ctypes.data, a.shape[0], a.shape[1], info.ctypes.data)
    return out, info


def residuals(a: np.ndarray, l: np.ndarray) -> dict[str, np.ndarray]:
    """FP64 per-matrix norms: ||A||_1, ||triu(L,1)||_1, ||LL^T-A||_1, rel. Frobenius."""
    a = _as3(a, np.float32)
    l = _as3(l, np.float32)
    out = np.empty((a.shape[0], 4), dtype=np.float64)
    _load().oracle_residuals(a.ctypes.data, l.ctypes.data, a.shape[0], a.shape[1], out.ctypes.data)
    return {"a_l1": out[:, 0], "upper_l1": out[:, 1], "resid_l1": out[:, 2], "rel_fro": out[:, 3]}


def potrf_backward_f64(l: np.ndarray, lbar: np.ndarray) -> np.ndarray:
    """Abar = 1/2 (S + S^T), S = L^{-T} Phi(L^T Lbar) L^{-1}, in FP64."""
    l = _as3(l, np.float64)
    lbar = _as3(lbar, np.float64)
    out = np.empty_like(l)
    _load().oracle_potrf_backward_f64(l.ctypes.data, lbar.ctypes.data, out.ctypes.data, l.shape[0], l.shape[1])
    return out


def _l1(x: np.ndarray) -> np.ndarray:
    """Matrix 1-norm (max column abs sum) per matrix, like torch.linalg.matrix_norm(ord=1)."""
    return np.abs(x).sum(axis=-2).max(axis=-1)


def check_implementation(data: np.ndarray, output: np.ndarray) -> tuple[bool, str]:
    """Restatement of the reference checker (reference/reference.py:137-188) in numpy FP32."""
    data = np.asarray(data)
    output = np.asarray(output)
    if output.shape != data.shape:
        return False, f"output shape must be {tuple(data.shape)}, got {tuple(output.shape)}"
    if output.dtype != np.float32:
        return False, f"output dtype must be torch.float32, got {output.dtype}"
    if not np.isfinite(output).all():
        return False, "output contains NaN or Inf"
    batch, n, _ = data.shape
    scale = np.maximum(_l1(data.astype(np.float32)), np.float32(_TINY32))
    upper = np.triu(output, k=1)
    tri = _l1(upper)
    if np.any(tri > _TRIANGULAR_RTOL_FACTOR * max(n, 1) * _EPS32 * scale):
        worst = float((tri / scale).max())
        return False, f"output is not lower triangular enough: relative_residual={worst:.3g}"
    diag = np.diagonal(output, axis1=-2, axis2=-1)
    if np.any(diag <= 0):
        return False, "output diagonal must be strictly positive"
    recon = np.matmul(output, np.swapaxes(output, -1, -2))
    resid = _l1(recon - data)
    if np.any(resid > _RECON_RTOL_FACTOR * max(n, 1) * _EPS32 * scale):
        worst = float((resid / scale).max())
        return False, f"L @ L.T does not reconstruct A: relative_residual={worst:.3g}"
    scaled = float((resid / (_EPS32 * max(n, 1) * scale)).max())
    return True, f"scaled_reconstruction_residual={scaled:.3g}; batch={batch}; n={n}"


def scaled_residual(message: str) -> float:
    """Parse the scaled residual out of a passing checker message."""
    head = message.split(";")[0]
    return float(head.split("=")[1])


def ref_kernel_cpu(a):
    """The reference's own CPU route for the path (reference/reference.py:129-130)."""
    import torch

    return torch.linalg.cholesky_ex(a, check_errors=False).L
