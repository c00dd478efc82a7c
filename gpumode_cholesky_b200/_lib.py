"""ctypes binding of ``libb200potrf.so`` (the C ABI in ``include/b200_potrf.h``).

The shared object is built in-tree by :mod:`gpumode_cholesky_b200.build`.
Loading fails loudly when it is missing: there is no CPU or vendor fallback.
"""

from __future__ import annotations

import ctypes
import threading
from pathlib import Path

from .build import LIB_PATH

B2P_OK = 0
B2P_ERR_INVALID_ARG = 1
B2P_ERR_UNSUPPORTED = 2
B2P_ERR_WORKSPACE = 3
B2P_ERR_CUDA = 4
B2P_ERR_TIMEOUT = 5

MODE_FP32 = 0
MODE_TF32 = 1
MODE_BF16X3 = 2
MODE_FP8 = 3
FLAG_FP64_DIAG = 0x100
FLAG_GUARD = 0x200
FLAGS = {"fp64diag": FLAG_FP64_DIAG, "guard": FLAG_GUARD}

MODES = {"fp32": MODE_FP32, "tf32": MODE_TF32, "bf16x3": MODE_BF16X3, "fp8": MODE_FP8}

PATHS = {"auto": 0, "blocked": 1, "fused": 2, "fused_ws": 3, "split": 4}


class RaggedOptions(ctypes.Structure):
    """Mirror of b2p_ragged_options (include/b200_potrf.h); zero = default."""

    _fields_ = [
        ("dense_min_n", ctypes.c_int32),
        ("pad_step", ctypes.c_int32),
        ("pad_step_large", ctypes.c_int32),
        ("large_path", ctypes.c_int32),
        ("streams", ctypes.c_int32),
    ]

# Every symbol the header declares, with (restype, argtypes).
_c_i64 = ctypes.c_int64
_c_sz = ctypes.c_size_t
_c_p = ctypes.c_void_p
SIGNATURES = {
    "b2p_version": (ctypes.c_int, []),
    "b2p_status_string": (ctypes.c_char_p, [ctypes.c_int]),
    "b2p_last_error": (ctypes.c_char_p, []),
    "b2p_potrf_workspace_size": (_c_sz, [_c_i64, _c_i64, ctypes.c_int]),
    "b2p_potrf_batched": (
        ctypes.c_int,
        [_c_p, _c_p, _c_i64, _c_i64, ctypes.c_int, _c_p, _c_sz, _c_p, _c_p],
    ),
    "b2p_potrf_path_workspace_size": (_c_sz, [_c_i64, _c_i64, ctypes.c_int, ctypes.c_int]),
    "b2p_potrf_batched_path": (
        ctypes.c_int,
        [_c_p, _c_p, _c_i64, _c_i64, ctypes.c_int, ctypes.c_int, _c_p, _c_sz, _c_p, _c_p],
    ),
    "b2p_potrf_batched_ex": (
        ctypes.c_int,
        [_c_p, _c_p, _c_i64, _c_i64, ctypes.c_int, ctypes.c_int, _c_p, _c_sz, _c_p, _c_p, _c_p],
    ),
    "b2p_potrf_host_workspace_size": (_c_sz, [_c_i64, _c_i64, ctypes.c_int, _c_i64]),
    "b2p_potrf_batched_host": (
        ctypes.c_int,
        [_c_p, _c_p, _c_i64, _c_i64, ctypes.c_int, _c_i64, _c_p, _c_sz, _c_p, _c_p],
    ),
    "b2p_noalloc_scratch_bytes": (_c_sz, []),
    "b2p_potrf_batched_noalloc": (ctypes.c_int, [_c_p, _c_p, _c_i64, _c_i64, ctypes.c_int, _c_p, _c_p]),
    "b2p_ragged_plan_create": (ctypes.c_int, [_c_p, _c_p, _c_i64, ctypes.c_int, ctypes.c_int, _c_p]),
    "b2p_trsv_batched": (ctypes.c_int, [_c_p, _c_p, _c_p, _c_i64, _c_i64, ctypes.c_int, _c_p]),
    "b2p_gp_nll_forward": (ctypes.c_int, [_c_p, _c_p, _c_p, _c_p, _c_i64, _c_i64, _c_p]),
    "b2p_gp_nll_backward": (ctypes.c_int, [_c_p, _c_p, _c_p, _c_p, _c_p, _c_i64, _c_i64, _c_p]),
    "b2p_ragged_plan_create_ex": (ctypes.c_int, [_c_p, _c_p, _c_i64, ctypes.c_int, _c_p, _c_p]),
    "b2p_ragged_plan_destroy": (None, [_c_p]),
    "b2p_ragged_plan_table_bytes": (_c_sz, [_c_p]),
    "b2p_ragged_plan_workspace_bytes": (_c_sz, [_c_p]),
    "b2p_ragged_plan_upload": (ctypes.c_int, [_c_p, _c_p, _c_p]),
    "b2p_potrf_ragged": (ctypes.c_int, [_c_p, _c_p, _c_p, _c_p, _c_p, _c_sz, _c_p, _c_p]),
    "b2p_potrf_backward_workspace_size": (_c_sz, [_c_i64, _c_i64]),
    "b2p_potrf_backward": (ctypes.c_int, [_c_p, _c_p, _c_p, _c_i64, _c_i64, ctypes.c_int, _c_p, _c_sz, _c_p]),
    "b2p_debug_tc_gemm": (ctypes.c_int, [_c_p, _c_p, _c_p, _c_i64, ctypes.c_int, _c_p, _c_p]),
    "b2p_debug_tc_gemm_stall": (ctypes.c_int, [_c_p, _c_p, _c_p, _c_i64, ctypes.c_int, ctypes.c_uint32, _c_p, _c_p]),
    "b2p_trace_enable": (ctypes.c_int, [ctypes.c_int]),
    "b2p_trace_read": (ctypes.c_int, [_c_p, _c_p, ctypes.c_int]),
    "b2p_trace_read_units": (ctypes.c_int, [_c_p, ctypes.c_int]),
    "b2p_trace_read_starts": (ctypes.c_int, [_c_p, ctypes.c_int]),
    "b2p_kernel_name": (ctypes.c_char_p, [ctypes.c_int]),
}

_lock = threading.Lock()
_lib: ctypes.CDLL | None = None


class PotrfError(RuntimeError):
    """A library call returned a non-zero status."""

    def __init__(self, status: int, where: str, detail: str):
        self.status = status
        super().__init__(f"{where}: {status_string(status)} ({detail})" if detail else f"{where}: {status_string(status)}")


def lib_path() -> Path:
    return LIB_PATH


def load(path: Path | None = None) -> ctypes.CDLL:
    """Load the shared object (once) and declare every exported signature."""
    global _lib
    with _lock:
        if _lib is not None and path is None:
            return _lib
        p = Path(path) if path is not None else LIB_PATH
        if not p.exists():
            raise RuntimeError(
                f"CUDA library {p} is missing; build it with `python -m gpumode_cholesky_b200.build`"
            )
        lib = ctypes.CDLL(str(p))
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        if path is None:
            _lib = lib
        return lib


class LaunchTrace:
    """Context manager recording per-launch device time of every library kernel.

    Use outside CUDA-graph capture.  ``records()`` returns (kernel name, ms)
    pairs in launch order after synchronising the recorded events;
    ``units()`` the algorithmic work the library attached to each launch
    (flops, or bytes for the n <= 32 kernel; 0 where none is defined).
    """

    def __init__(self, capacity: int = 65536):
        self.capacity = capacity
        self._records: list[tuple[str, float]] = []
        self._units: list[float] = []
        self._starts: list[float] = []

    def __enter__(self):
        check(load().b2p_trace_enable(self.capacity), "b2p_trace_enable")
        return self

    def __exit__(self, *exc):
        lib = load()
        ids = (ctypes.c_int32 * self.capacity)()
        ms = (ctypes.c_float * self.capacity)()
        k = lib.b2p_trace_read(ids, ms, self.capacity)
        self._records = [(lib.b2p_kernel_name(ids[i]).decode(), float(ms[i])) for i in range(k)]
        units = (ctypes.c_double * self.capacity)()
        ku = lib.b2p_trace_read_units(units, self.capacity)
        self._units = [float(units[i]) for i in range(min(k, ku))]
        starts = (ctypes.c_float * self.capacity)()
        ks = lib.b2p_trace_read_starts(starts, self.capacity)
        self._starts = [float(starts[i]) for i in range(min(k, ks))]
        lib.b2p_trace_enable(0)
        return False

    def records(self) -> list[tuple[str, float]]:
        return list(self._records)

    def timeline(self) -> list[tuple[str, float, float]]:
        """(kernel name, start ms after the first launch, duration ms) per launch."""
        return [(name, s, t) for (name, t), s in zip(self._records, self._starts)]

    def units(self) -> dict[str, float]:
        """Algorithmic work per kernel name, summed over its launches."""
        out: dict[str, float] = {}
        for (name, _), u in zip(self._records, self._units):
            out[name] = out.get(name, 0.0) + u
        return out

    def totals(self) -> dict[str, tuple[int, float]]:
        out: dict[str, tuple[int, float]] = {}
        for name, t in self._records:
            c, s = out.get(name, (0, 0.0))
            out[name] = (c + 1, s + t)
        return out


def status_string(status: int) -> str:
    return load().b2p_status_string(status).decode()


def check(status: int, where: str) -> None:
    if status != B2P_OK:
        detail = load().b2p_last_error().decode()
        raise PotrfError(status, where, detail)
