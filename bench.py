#!/usr/bin/env python
"""Benchmark of the batched Cholesky hot path on B200.

Workload (one "step"): factor the two plain-FP32 mid-size batches of the
benchmark suite, 640 matrices of order 512 and 60 of order 1024, each batch
half well-conditioned (M M^T/n + I) and half prescribed-spectrum
(Q diag(logspace[1, 1e6]) Q^T).  Inputs are synthetic and seeded, resident
in HBM (0.92 GB, larger than the 126 MB L2, so no flush is needed between
steps).  ``value`` is device time per step in microseconds (lower is better).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--mode fp32|bf16x3|tf32|auto]
    python bench.py --impl reference     # the reference's CPU route, timed on host cores

With N > 1 (torchrun) every rank factors its own full step (weak scaling, no
collective on the data path); the reported time is the max over ranks.
"""

from __future__ import annotations

import argparse
import json
import math
import os
import subprocess
import sys
import tempfile
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

import torch  # noqa: E402

SHAPES = [(640, 512), (60, 1024)]
SEEDS = {512: 510512, 1024: 511024}
WORKLOAD = "mid-size batched potrf: 640x512 + 60x1024 FP32, half MM^T/n+I, half spectrum [1,1e6]"
METRIC = "batched potrf us per step (640x512 + 60x1024)"


def _dist():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def _flops(batch: int, n: int) -> float:
    return batch * n**3 / 3.0


def _clock_sampler_start(gpu_index: int):
    path = tempfile.NamedTemporaryFile(prefix="clocks", suffix=".csv", delete=False).name
    q = (
        "timestamp,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
        "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
        "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap"
    )
    try:
        f = open(path, "w")
        p = subprocess.Popen(
            ["nvidia-smi", "-i", str(gpu_index), f"--query-gpu={q}", "--format=csv,noheader,nounits", "-lms", "100"],
            stdout=f,
            stderr=subprocess.DEVNULL,
        )
        return p, f, path
    except Exception:
        return None, None, path


def _clock_sampler_stop(state, t0: float, t1: float) -> dict:
    """Median SM clock and throttle reasons of the samples taken in [t0, t1] (host time)."""
    import datetime as _dt

    p, f, path = state
    if p is None:
        return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
    p.terminate()
    try:
        p.wait(timeout=5)
    except Exception:
        p.kill()
    f.close()
    names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
    rows = []
    for line in Path(path).read_text().splitlines():
        parts = [x.strip() for x in line.split(",")]
        if len(parts) < 9:
            continue
        try:
            ts = _dt.datetime.strptime(parts[0], "%Y/%m/%d %H:%M:%S.%f").timestamp()
            rows.append((ts, float(parts[1]), float(parts[2]), parts[5:9]))
        except ValueError:
            continue
    os.unlink(path)
    window = [r for r in rows if t0 - 0.05 <= r[0] <= t1 + 0.05]
    label = "timed region"
    if not window:
        window, label = rows, "whole run (timed region shorter than the sampling period)"
    sms = sorted(r[1] for r in window)
    reasons = {nm for r in window for nm, v in zip(names, r[3]) if v.lower() == "active"}
    return {
        "sm_mhz": sms[len(sms) // 2] if sms else None,
        "sm_max_mhz": max((r[2] for r in window), default=None),
        "samples": len(sms),
        "window": label,
        "reasons": sorted(reasons),
    }


def _measured_peaks() -> dict:
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return {"hbm_gbs": d["hbm_gbs"], "bf16_tflops": d["bf16_tflops"], "src": "measured"}
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "src": "fallback"}


def _profiled_traffic() -> dict:
    """DRAM bytes per launch of the dominant kernels from the committed ncu summaries."""
    out = {}
    for p in (ROOT / "profiles").glob("*.md"):
        for line in p.read_text().splitlines():
            if line.startswith("traffic_bytes_per_unit:"):
                # traffic_bytes_per_unit: <kernel> <mode> <bytes per algorithmic byte/flop>
                parts = line.split()
                if len(parts) >= 4:
                    out[(parts[1], parts[2])] = float(parts[3])
    return out


# ---------------------------------------------------------------------------
def run_reference(args) -> int:
    """The reference's CPU route (torch.linalg.cholesky_ex FP32, reference/reference.py:129-130)."""
    ws, rank, _ = _dist()
    if rank != 0:
        return 0
    import oracle  # the CPU leg may use the oracle package (reference route restated there)
    from gpumode_cholesky_b200 import inputs

    threads = os.cpu_count() or 1
    torch.set_num_threads(threads)
    frac = args.ref_sample
    sample = [(max(1, int(round(b * frac))), n) for b, n in SHAPES]
    data = [inputs.mixed_batch(b, n, SEEDS[n], device="cpu") for b, n in sample]
    for _ in range(args.warmup):
        for a in data:
            oracle.ref_kernel_cpu(a)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        for a in data:
            oracle.ref_kernel_cpu(a)
    dt = (time.perf_counter() - t0) / args.steps
    scale = sum(_flops(b, n) for b, n in SHAPES) / sum(_flops(b, n) for b, n in sample)
    us = dt * 1e6 * scale
    desc = " + ".join(f"{b}x{n}" for b, n in sample) + f" per step, scaled by flops x{scale:.2f} to the full step"
    line = {
        "impl": "reference",
        "metric": METRIC,
        "value": round(us, 1),
        "unit": "us",
        "n_gpus": ws,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": round(us / 1000.0, 3),
        "higher_is_better": False,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32",
        "data": "synthetic",
        "config": {"workload": WORKLOAD, "l2": "inputs larger than L2"},
        "cpu_baseline": {
            "value": round(us, 1),
            "unit": "us",
            "cores": threads,
            "kind": "reference",
            "sample": "torch.linalg.cholesky_ex FP32 on CPU (reference ref_kernel); " + desc,
        },
        "e2e": {"value": round(us, 1), "unit": "us", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))
    return 0


# ---------------------------------------------------------------------------
def run_ours(args) -> int:
    ws, rank, local = _dist()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if ws > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=dev)
    from gpumode_cholesky_b200 import _lib, build, inputs
    from gpumode_cholesky_b200.potrf import cholesky

    if not build.LIB_PATH.exists():
        build.build()
    _lib.load()
    mode = args.mode
    data = [inputs.mixed_batch(b, n, SEEDS[n] + 7919 * rank, device=dev) for b, n in SHAPES]
    outs = [torch.empty_like(a) for a in data]
    torch.cuda.synchronize()

    def step(m):
        for a, o in zip(data, outs):
            cholesky(a, mode=m, out=o)

    def timed(fn, k):
        s = torch.cuda.current_stream()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(s)
        for _ in range(k):
            fn()
        e1.record(s)
        e1.synchronize()
        return e0.elapsed_time(e1) / k

    def barrier():
        if ws > 1:
            import torch.distributed as dist

            dist.barrier()

    clk = _clock_sampler_start(local)
    time.sleep(0.3)  # let nvidia-smi start sampling
    for _ in range(args.warmup):
        step(mode)
    barrier()
    torch.cuda.synchronize()
    t_start = time.time()
    ms = timed(lambda: step(mode), args.steps)
    torch.cuda.synchronize()
    t_end = time.time()
    barrier()
    clocks = _clock_sampler_stop(clk, t_start, t_end)
    if ws > 1:
        import torch.distributed as dist

        t = torch.tensor([ms], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())

    # Per-shape times, plain FP32 vs the chosen mode, and cuSOLVER on the same GPU.
    per_shape = {}
    for (b, n), a, o in zip(SHAPES, data, outs):
        per_shape[f"{b}x{n}"] = round(1000 * timed(lambda: cholesky(a, mode=mode, out=o), args.steps), 1)
    plain = None
    if mode not in (None, "fp32"):
        plain = round(1000 * timed(lambda: step("fp32"), args.steps), 1)
    cusolver = round(
        1000 * timed(lambda: [torch.linalg.cholesky_ex(a, check_errors=False) for a in data], max(2, args.steps // 2)),
        1,
    )

    # Accuracy at full size (FP64 on the device).
    step(mode)
    resid = {}
    for (b, n), a, o in zip(SHAPES, data, outs):
        ld = o.double()
        ad = a.double()
        r = torch.linalg.matrix_norm(ld @ ld.transpose(-1, -2) - ad) / torch.linalg.matrix_norm(ad)
        resid[f"{b}x{n}"] = float(r.max())

    # Per-kernel device time of one step (CUDA events on the launch stream).
    with _lib.LaunchTrace() as tr:
        step(mode)
    totals = tr.totals()
    launches_per_step = sum(c for c, _ in totals.values())
    dom = max(totals.items(), key=lambda kv: kv[1][1])
    dom_name, (dom_count, dom_ms) = dom
    peaks = _measured_peaks()
    roof = _roofline(dom_name, dom_ms, dom_count, mode, peaks)

    # End to end through the public API: pinned host in, host out, every step.
    host_in = [a.cpu().pin_memory() for a in data]
    host_out = [torch.empty_like(h).pin_memory() for h in host_in]
    dev_in = [torch.empty_like(a) for a in data]

    def e2e_step():
        for hi, di, do, ho in zip(host_in, dev_in, outs, host_out):
            di.copy_(hi, non_blocking=True)
            cholesky(di, mode=mode, out=do)
            ho.copy_(do, non_blocking=True)

    e2e_step()
    torch.cuda.synchronize()
    e2e_ms = timed(e2e_step, max(2, args.steps // 2))
    h2d = sum(h.numel() * 4 for h in host_in)

    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu:
        cpu = _cpu_baseline(args)

    if rank == 0:
        line = {
            "metric": METRIC,
            "value": round(ms * 1000, 1),
            "unit": "us",
            "n_gpus": ws,
            "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": round(ms, 4),
            "higher_is_better": False,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "f32" if mode in (None, "fp32") else f"f32 ({mode} trailing updates)",
            "data": "synthetic",
            "config": {
                "workload": WORKLOAD,
                "shapes": [f"{b}x{n}" for b, n in SHAPES],
                "mode": mode or "fp32",
                "l2": "inputs (0.92 GB) larger than L2; no flush",
                "parallelism": f"weak scaling, {ws} rank(s) each a full step",
            },
            "per_shape_us": per_shape,
            "plain_fp32_us": plain,
            "cusolver_same_gpu_us": cusolver,
            "rel_residual_fro": resid,
            "matrices_per_s": round(ws * sum(b for b, _ in SHAPES) / (ms / 1000.0), 1),
            "gflops_per_s": round(ws * sum(_flops(b, n) for b, n in SHAPES) / (ms / 1000.0) / 1e9, 1),
            "roofline": roof,
            "kernels_one_step": {k: {"launches": c, "ms": round(t, 4)} for k, (c, t) in sorted(totals.items())},
            "cpu_baseline": cpu,
            "e2e": {
                "value": round(e2e_ms * 1000, 1),
                "unit": "us",
                "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": h2d,
            },
            "gpu_launches": launches_per_step * args.steps,
            "clocks": clocks,
        }
        print(json.dumps(line))
    if ws > 1:
        import torch.distributed as dist

        dist.barrier()
        dist.destroy_process_group()
    return 0


def _roofline(name: str, ms: float, count: int, mode, peaks: dict) -> dict:
    """Roofline of the dominant kernel over one step.

    Algorithmic units: the trailing SYRK kernels count the flops of the lower
    triangle they update, R(R+1)*nb per matrix and step (R = rows below the
    block column, nb = 64); other kernels count FP32 bytes read + written.
    """
    nb = 64
    flops = 0.0
    if name.startswith("trail"):
        for b, n in SHAPES:
            for k0 in range(0, n, nb):
                r = n - k0 - nb
                if r > 0:
                    flops += b * r * (r + 1) * nb
        achieved = flops / (ms / 1000.0) / 1e12
        peak = peaks["bf16_tflops"]
        tr = _profiled_traffic().get((name, str(mode or "fp32")))
        return {
            "kernel": name,
            "bound": "tensor",
            "achieved": round(achieved, 2),
            "peak": peak,
            "unit": "TFLOP/s",
            "frac": round(achieved / peak, 4),
            "peak_src": f"bf16 dense, {peaks['src']}",
            "traffic": None if tr is None else round(tr * flops / max(count, 1)),
            "launches": count,
            "ms": round(ms, 4),
        }
    byts = sum(8.0 * b * n * n for b, n in SHAPES)
    achieved = byts / (ms / 1000.0) / 1e9
    return {
        "kernel": name,
        "bound": "hbm",
        "achieved": round(achieved, 1),
        "peak": peaks["hbm_gbs"],
        "unit": "GB/s",
        "frac": round(achieved / peaks["hbm_gbs"], 4),
        "peak_src": peaks["src"],
        "traffic": None,
        "launches": count,
        "ms": round(ms, 4),
    }


def _cpu_baseline(args) -> dict:
    """The reference's CPU route on a bounded sample, on all host cores."""
    import oracle
    from gpumode_cholesky_b200 import inputs

    threads = os.cpu_count() or 1
    torch.set_num_threads(threads)
    sample = [(max(1, int(round(b * args.ref_sample))), n) for b, n in SHAPES]
    data = [inputs.mixed_batch(b, n, SEEDS[n], device="cpu") for b, n in sample]
    for a in data:
        oracle.ref_kernel_cpu(a)
    reps = 2
    t0 = time.perf_counter()
    for _ in range(reps):
        for a in data:
            oracle.ref_kernel_cpu(a)
    dt = (time.perf_counter() - t0) / reps
    scale = sum(_flops(b, n) for b, n in SHAPES) / sum(_flops(b, n) for b, n in sample)
    return {
        "value": round(dt * 1e6 * scale, 1),
        "unit": "us",
        "cores": threads,
        "kind": "reference",
        "sample": "torch.linalg.cholesky_ex FP32 on CPU (reference ref_kernel) on "
        + " + ".join(f"{b}x{n}" for b, n in sample)
        + f", scaled by flops x{scale:.2f}",
    }


def main() -> int:
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--mode", default="fp32")
    ap.add_argument("--ref-sample", type=float, default=0.05, help="fraction of the step the CPU legs factor")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
