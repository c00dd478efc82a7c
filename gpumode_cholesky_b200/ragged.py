"""Ragged batches: many SPD matrices of different orders in one packed buffer.

A :class:`RaggedPlan` is built once per list of orders (host-side schedule
in the library, tables uploaded to the device once); :meth:`RaggedPlan.factor`
then enqueues the whole factorization on the current stream without host
synchronisation, and :meth:`RaggedPlan.capture` records it into a CUDA graph
that replays the entire ragged batch as one graph launch.

Layout: matrix i occupies ``buf[offsets[i] : offsets[i] + n_i * n_i]``
(row-major), offsets multiples of 4 elements (16 bytes).  The reference has
no ragged path (its dispatcher routes exact (batch, n) shapes only,
submission.py:4111-4268).
"""

from __future__ import annotations

import ctypes
from collections.abc import Sequence

import torch

from . import _lib
from .inputs import pack_offsets
from .potrf import _stream_ptr, resolve_mode


def pack(mats: Sequence[torch.Tensor], device=None) -> tuple[torch.Tensor, list[int], list[int]]:
    """Pack square FP32 matrices into one buffer; returns (buffer, orders, offsets)."""
    orders = [int(m.shape[-1]) for m in mats]
    offs = pack_offsets(orders)
    dev = device if device is not None else (mats[0].device if mats else "cpu")
    buf = torch.zeros(offs[-1], dtype=torch.float32, device=dev)
    for m, n, o in zip(mats, orders, offs):
        buf[o : o + n * n] = m.reshape(-1).to(device=dev, dtype=torch.float32)
    return buf, orders, offs[:-1]


def unpack(buf: torch.Tensor, orders: Sequence[int], offsets: Sequence[int]) -> list[torch.Tensor]:
    """Views of the packed matrices."""
    return [buf[o : o + n * n].view(n, n) for n, o in zip(orders, offsets)]


class RaggedPlan:
    """Schedule for one list of orders (and offsets) on one device.

    ``tc_min_n`` (tensor modes): matrices of at least this order (and > 128)
    are factored as identity-padded dense batches, one per padded order
    (multiple of ``pad_step``, or ``pad_step_large`` above 1024: 64, 128 or
    256); smaller ones take the blocked ragged schedule.  ``large_path``
    picks the algorithm of the groups above 1024 ("split" or "fused_ws");
    ``streams`` runs the groups on that many streams at once.  Zero / "auto"
    take the library defaults (every n > 128 padded to a multiple of 128,
    warp-specialized groups above 1024, four streams).
    """

    def __init__(
        self,
        orders: Sequence[int],
        offsets: Sequence[int] | None = None,
        mode: str | int | None = None,
        tc_min_n: int = 0,
        device: torch.device | str | None = None,
        pad_step: int = 0,
        pad_step_large: int = 0,
        large_path: str = "auto",
        streams: int = 0,
    ):
        self.orders = [int(n) for n in orders]
        self.offsets = [int(o) for o in (offsets if offsets is not None else pack_offsets(self.orders)[:-1])]
        if len(self.offsets) != len(self.orders):
            raise ValueError("orders and offsets differ in length")
        self.count = len(self.orders)
        self.total = max((o + n * n for n, o in zip(self.orders, self.offsets)), default=0)
        self.mode = resolve_mode(mode, max(self.orders, default=0))
        self.device = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
        lib = _lib.load()
        offs = (ctypes.c_int64 * max(self.count, 1))(*self.offsets)
        ns = (ctypes.c_int32 * max(self.count, 1))(*self.orders)
        handle = ctypes.c_void_p()
        if large_path not in ("auto", "split", "fused_ws"):
            raise ValueError(f"large_path must be auto, split or fused_ws, not {large_path!r}")
        self.options = _lib.RaggedOptions(
            int(tc_min_n), int(pad_step), int(pad_step_large), _lib.PATHS[large_path], int(streams)
        )
        _lib.check(
            lib.b2p_ragged_plan_create_ex(
                offs, ns, self.count, self.mode, ctypes.byref(self.options), ctypes.byref(handle)
            ),
            "b2p_ragged_plan_create_ex",
        )
        self._handle = handle
        self.table_bytes = lib.b2p_ragged_plan_table_bytes(handle)
        self.workspace_bytes = lib.b2p_ragged_plan_workspace_bytes(handle)
        self.tables = torch.empty(max(self.table_bytes, 16), dtype=torch.uint8, device=self.device)
        self.workspace = torch.empty(max(self.workspace_bytes, 256), dtype=torch.uint8, device=self.device)
        with torch.cuda.device(self.device):
            _lib.check(
                lib.b2p_ragged_plan_upload(handle, self.tables.data_ptr(), _stream_ptr(self.device)),
                "b2p_ragged_plan_upload",
            )

    def close(self) -> None:
        if getattr(self, "_handle", None) is not None and self._handle.value:
            _lib.load().b2p_ragged_plan_destroy(self._handle)
            self._handle = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def factor(self, a: torch.Tensor, out: torch.Tensor | None = None, info: torch.Tensor | None = None):
        """Factor every matrix of the packed buffer ``a`` into ``out`` (same layout)."""
        if not a.is_cuda or a.dtype != torch.float32 or a.dim() != 1:
            raise ValueError("a must be a 1-D float32 CUDA buffer")
        if a.numel() < self.total:
            raise ValueError(f"buffer holds {a.numel()} elements, the plan needs {self.total}")
        if out is None:
            out = torch.empty_like(a)
        if info is not None and (info.dtype != torch.int32 or info.numel() < self.count):
            raise ValueError("info must be int32 with one entry per matrix")
        with torch.cuda.device(a.device):
            st = _lib.load().b2p_potrf_ragged(
                self._handle,
                self.tables.data_ptr(),
                a.data_ptr(),
                out.data_ptr(),
                self.workspace.data_ptr(),
                self.workspace.numel(),
                info.data_ptr() if info is not None else None,
                _stream_ptr(a.device),
            )
        _lib.check(st, "b2p_potrf_ragged")
        return out

    def capture(self, a_static: torch.Tensor, out_static: torch.Tensor) -> torch.cuda.CUDAGraph:
        """Record factor(a_static -> out_static) into a CUDA graph (replay with ``g.replay()``)."""
        self.factor(a_static, out_static)  # warm: sets kernel attributes outside capture
        torch.cuda.synchronize(a_static.device)
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g):
            self.factor(a_static, out_static)
        return g


def split_runs(orders: Sequence[int], offsets: Sequence[int], parts: int) -> list[tuple[int, int]]:
    """Cut a packed list into at most ``parts`` contiguous runs of about equal bytes.

    Returns (first, end) matrix indices of each non-empty run, in order.  A
    run ends at the first matrix whose end reaches its share of the buffer.
    """
    count = len(orders)
    if count == 0:
        return []
    parts = max(1, min(int(parts), count))
    ends = [o + n * n for n, o in zip(orders, offsets)]
    base, total = offsets[0], ends[-1]
    runs, first = [], 0
    for k in range(1, parts + 1):
        target = base + (total - base) * k / parts
        end = first
        while end < count and (end == first or ends[end - 1] < target):
            end += 1
        if k == parts:
            end = count
        if end > first:
            runs.append((first, end))
            first = end
        if first >= count:
            break
    return runs


class RaggedHostPlan:
    """Factor a packed ragged list held in host memory into host memory.

    The list is cut into ``parts`` contiguous runs of about equal bytes
    (:func:`split_runs`; 0 picks runs of about 160 MiB, at most 64), each
    with its own :class:`RaggedPlan` (``plan_options`` are passed on).
    :meth:`factor` copies run i in on a copy stream, factors it on the
    current stream once it has arrived, and copies it out on a second copy
    stream, so the copies of the runs before and after overlap its
    factorization; PCIe is full duplex, so a call costs about one direction's
    transfer plus one run.  The plan keeps full-size device buffers for the
    input and the factors (each run has its own slice, so no buffer is
    reused within a call).  Host buffers should be pinned for the copies to
    overlap.  A run picks its dense groups from its own matrices, so results
    can differ in the last bits from one plan over the whole list.
    """

    def __init__(
        self,
        orders: Sequence[int],
        offsets: Sequence[int] | None = None,
        mode: str | int | None = None,
        parts: int = 0,
        device: torch.device | str | None = None,
        **plan_options,
    ):
        self.orders = [int(n) for n in orders]
        self.offsets = [int(o) for o in (offsets if offsets is not None else pack_offsets(self.orders)[:-1])]
        if len(self.offsets) != len(self.orders):
            raise ValueError("orders and offsets differ in length")
        if parts < 0:
            raise ValueError("parts must be >= 0")
        for i in range(1, len(self.orders)):
            if self.offsets[i] < self.offsets[i - 1] + self.orders[i - 1] ** 2:
                raise ValueError("a host plan needs ascending, non-overlapping offsets")
        self.count = len(self.orders)
        self.mode = resolve_mode(mode, max(self.orders, default=0))
        self.total = max((o + n * n for n, o in zip(self.orders, self.offsets)), default=0)
        self.device = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
        if parts == 0:
            parts = min(64, max(1, -(-self.total * 4 // (160 << 20))))
        self.runs = []  # (first, end, element start, element end, plan)
        for i0, i1 in split_runs(self.orders, self.offsets, parts):
            e0 = self.offsets[i0]
            e1 = self.offsets[i1 - 1] + self.orders[i1 - 1] ** 2
            plan = RaggedPlan(
                self.orders[i0:i1], [o - e0 for o in self.offsets[i0:i1]], self.mode, device=self.device, **plan_options
            )
            self.runs.append((i0, i1, e0, e1, plan))
        self.dev_in = torch.empty(max(self.total, 1), dtype=torch.float32, device=self.device)
        self.dev_out = torch.empty_like(self.dev_in)
        self._s_in = torch.cuda.Stream(self.device)
        self._s_out = torch.cuda.Stream(self.device)

    def factor(
        self,
        a: torch.Tensor,
        out: torch.Tensor | None = None,
        info: torch.Tensor | None = None,
        non_blocking: bool = False,
    ) -> torch.Tensor:
        """Factor every matrix of the host buffer ``a`` into ``out`` (same layout, host).

        With ``non_blocking`` the call only enqueues: ``out`` holds the
        factors once the current stream is synchronised.
        """
        if a.is_cuda or a.dtype != torch.float32 or a.dim() != 1:
            raise ValueError("a must be a 1-D float32 host buffer")
        if a.numel() < self.total:
            raise ValueError(f"buffer holds {a.numel()} elements, the plan needs {self.total}")
        if out is None:
            out = torch.empty(a.shape, dtype=torch.float32, pin_memory=True)
        elif out.is_cuda or out.dtype != torch.float32 or out.shape != a.shape:
            raise ValueError("out must be a float32 host buffer shaped like a")
        if info is not None and (info.dtype != torch.int32 or info.numel() < self.count or not info.is_cuda):
            raise ValueError("info must be an int32 CUDA tensor with one entry per matrix")
        with torch.cuda.device(self.device):
            cur = torch.cuda.current_stream(self.device)
            # Copies start after the work already on the caller's stream
            # (an earlier call may still read the device buffers).
            self._s_in.wait_stream(cur)
            self._s_out.wait_stream(cur)
            for i0, i1, e0, e1, plan in self.runs:
                with torch.cuda.stream(self._s_in):
                    self.dev_in[e0:e1].copy_(a[e0:e1], non_blocking=True)
                cur.wait_stream(self._s_in)
                plan.factor(self.dev_in[e0:e1], self.dev_out[e0:e1], info[i0:i1] if info is not None else None)
                self._s_out.wait_stream(cur)
                with torch.cuda.stream(self._s_out):
                    out[e0:e1].copy_(self.dev_out[e0:e1], non_blocking=True)
            cur.wait_stream(self._s_out)
            if not non_blocking:
                cur.synchronize()
        return out


#: Candidate plan options for :func:`autotune`: padded-order step for orders
#: <= 1024 and above, path of the groups above 1024, and concurrent streams.
AUTOTUNE_GRID: tuple[dict, ...] = tuple(
    {"pad_step": ps, "pad_step_large": pl, "large_path": lp, "streams": st}
    for ps in (64, 128)
    for pl in (128, 256)
    for lp in ("fused_ws", "split")
    for st in (1, 4)
)


def autotune(
    a: torch.Tensor,
    orders: Sequence[int],
    offsets: Sequence[int] | None = None,
    mode: str | int | None = "bf16x3",
    candidates: Sequence[dict] | None = None,
    reps: int = 2,
) -> tuple[RaggedPlan, list[tuple[dict, float]]]:
    """Pick the fastest plan options for this list of orders on this GPU.

    Every candidate (default :data:`AUTOTUNE_GRID`: the padded-order steps per
    size bucket, the path of the large groups, the stream count) is built,
    captured in a CUDA graph over the packed buffer ``a`` and timed with CUDA
    events (one warm-up replay, then ``reps``).  Returns the fastest plan and
    the (options, microseconds) of every candidate.  The candidates differ
    only in grouping and scheduling; all factor every matrix in the same
    precision mode.
    """
    cands = list(candidates if candidates is not None else AUTOTUNE_GRID)
    if not cands:
        raise ValueError("no candidate options")
    out = torch.empty_like(a)
    results: list[tuple[dict, float]] = []
    best_us, best = float("inf"), None
    for opt in cands:
        plan = RaggedPlan(orders, offsets, mode=mode, device=a.device, **opt)
        g = plan.capture(a, out)
        g.replay()
        start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        start.record()
        for _ in range(reps):
            g.replay()
        end.record()
        end.synchronize()
        us = start.elapsed_time(end) * 1000.0 / reps
        results.append((dict(opt), us))
        del g
        if us < best_us:
            if best is not None:
                best.close()
            best_us, best = us, plan
        else:
            plan.close()
        del plan
        torch.cuda.empty_cache()
    assert best is not None
    return best, results


def cholesky_ragged(
    a: torch.Tensor, orders: Sequence[int], offsets: Sequence[int] | None = None, mode: str | int | None = None
) -> torch.Tensor:
    """One-shot ragged factorization (builds a plan each call)."""
    plan = RaggedPlan(orders, offsets, mode=mode, device=a.device)
    try:
        return plan.factor(a)
    finally:
        torch.cuda.current_stream(a.device).synchronize()
        plan.close()
