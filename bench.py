#!/usr/bin/env python
"""Benchmark of the batched Cholesky hot path on B200.

Default workload ("mid", one "step"): factor the two plain-FP32 mid-size
batches of the benchmark suite, 640 matrices of order 512 and 60 of order
1024, each batch half well-conditioned (M M^T/n + I) and half
prescribed-spectrum (Q diag(logspace[1, 1e6]) Q^T).  Inputs are synthetic,
seeded and resident in HBM (0.92 GB, larger than the 126 MB L2, so no flush
is needed between steps).  ``value`` is device time per step in microseconds
(lower is better) in the chosen precision mode ("auto" = BF16x3 trailing
updates for n > 128, the mixed form that meets the 1e-5 relative residual);
the plain FP32 form and cuSOLVER on the same GPU are reported beside it.

Other workloads (profiling and extra lines, not the headline):
  small   4096 x 32 (HBM-bound; 8 rotating input sets, 256 MiB > L2)
  large   1 x 8192 (GG^T/n + 0.1 I); large12k, large16k, large32k: 1 x 12288,
          1 x 16384, 1 x 32768
  ragged  3000 matrices, n log-uniform in [16, 2048], packed (one ragged plan
          replayed from a CUDA graph; --autotune picks the plan options)
  gp      Gaussian-process loss, forward and backward through autograd
          (eager calls), 256 x 128 + 8 x 2048 RBF kernels

    python bench.py [--gpus N] [--steps K] [--warmup W] [--mode auto|fp32|bf16x3|tf32]
    python bench.py --impl reference     # the reference's CPU route, timed on host cores

With N > 1 (torchrun) every rank factors its own full step (weak scaling, no
collective on the data path); the reported time is the max over ranks.
Steps are replayed from a CUDA graph captured once (launch overhead is not
part of the device time); ``e2e`` instead calls the public entry point per
step with host<->device copies.
"""

from __future__ import annotations

import argparse
import json
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

WORKLOADS = {
    "mid": {
        "shapes": [(640, 512), (60, 1024)],
        "seeds": [510512, 511024],
        "gen": "mixed",
        "sets": 1,
        "desc": "mid-size batched potrf: 640x512 + 60x1024 FP32, half MM^T/n+I, half spectrum [1,1e6]",
        "metric": "batched potrf us per step (640x512 + 60x1024)",
    },
    "small": {
        "shapes": [(4096, 32)],
        "seeds": [41032],
        "gen": "well",
        "sets": 8,
        "desc": "small batched potrf: 4096x32 FP32, MM^T/n+I",
        "metric": "batched potrf us per step (4096x32)",
        # the reference's published device time of its shipped kernel for this exact shape
        "baseline_us": 14.0,
    },
    "ragged": {
        "ragged": True,
        "count": 3000,
        "orders_seed": 4,
        "seeds": [5],
        "shapes": [],
        "gen": "well",
        "sets": 1,
        "desc": "ragged potrf: 3000 FP32 SPD matrices, n = round(exp(U[ln16, ln2048])) (seed 4), MM^T/n+I, "
        "packed with offsets",
        "metric": "ragged potrf us per step (3000 matrices, n log-uniform in [16, 2048])",
    },
    "gp": {
        "gp": True,
        "shapes": [(256, 128), (8, 2048)],
        "seeds": [5128, 52048],
        "gen": "rbf",
        "sets": 1,
        "desc": "GP log-likelihood forward+backward: 256x128 + 8x2048 FP32 RBF kernels over U[0,1]^3 points, "
        "lengthscale U[0.2,0.5], variance 1, jitter 1e-4 I, y ~ N(0,1)",
        "metric": "gp nll fwd+bwd us per step (256x128 + 8x2048)",
    },
    "large": {
        "shapes": [(1, 8192)],
        "seeds": [48192],
        "gen": "gram",
        "sets": 1,
        "desc": "large potrf: 1x8192 FP32, GG^T/n+0.1I",
        "metric": "potrf us per step (1x8192)",
        "baseline_us": 5773.79,
    },
    "large12k": {
        "shapes": [(1, 12288)],
        "seeds": [412288],
        "gen": "gram",
        "sets": 1,
        "desc": "large potrf: 1x12288 FP32, GG^T/n+0.1I (the first order with the outer-block update; profiling)",
        "metric": "potrf us per step (1x12288)",
    },
    "large16k": {
        "shapes": [(1, 16384)],
        "seeds": [416384],
        "gen": "gram",
        "sets": 1,
        "desc": "large potrf: 1x16384 FP32, GG^T/n+0.1I",
        "metric": "potrf us per step (1x16384)",
        "baseline_us": 8365.65,
    },
    "large32k": {
        "shapes": [(1, 32768)],
        "seeds": [432768],
        "gen": "gram",
        "sets": 1,
        "desc": "large potrf: 1x32768 FP32, GG^T/n+0.1I",
        "metric": "potrf us per step (1x32768)",
        "baseline_us": 22980.53,
        "cpu_sample": [(1, 16384)],
    },
}


def _dist():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def _flops(batch: int, n: int) -> float:
    return batch * n**3 / 3.0


def _make(gen: str, b: int, n: int, seed: int, device):
    from gpumode_cholesky_b200 import inputs

    if gen == "mixed":
        return inputs.mixed_batch(b, n, seed, device=device)
    if gen == "gram":
        return inputs.large_gram(n, seed, device=device).expand(b, n, n).contiguous()
    return inputs.well_conditioned(b, n, seed, device=device)


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
        return {"hbm_gbs": d["hbm_gbs"], "bf16_tflops": d["bf16_tflops"], "src": "of measured"}
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "src": "of fallback"}


def _profiled_traffic() -> dict:
    """DRAM bytes per algorithmic byte (or flop) of a kernel, from the committed ncu summaries.

    A summary line reads ``traffic_per_unit: <kernel> <workload> <mode> <value>``.
    """
    out = {}
    for p in (ROOT / "profiles").glob("*.md"):
        for line in p.read_text().splitlines():
            if line.startswith("traffic_per_unit:"):
                parts = line.split()
                if len(parts) >= 5:
                    out[(parts[1], parts[2], parts[3])] = float(parts[4])
    return out


def _resolve_mode(mode: str, n: int):
    """The mode name a shape runs in ("auto": what custom_kernel picks)."""
    if mode != "auto":
        return mode
    return "bf16x3+guard" if n > 128 and n % 64 == 0 else "fp32"


def _shapes(wl: dict, args) -> list[tuple[int, int]]:
    return [(max(1, int(round(b * args.scale))), n) for b, n in wl["shapes"]]


def _dense_config(wl: dict, args, ws: int, shapes) -> dict:
    """The workload's config, identical in both arms of the bench."""
    return {
        "workload": wl["desc"] + ("" if args.scale == 1.0 else f" (batch scaled x{args.scale})"),
        "shapes": [f"{b}x{n}" for b, n in shapes],
        "mode": args.mode,
        "modes": {f"{b}x{n}": _resolve_mode(args.mode, n) for b, n in shapes},
        "entry": "custom_kernel(A)" if args.mode == "auto" else f"cholesky(A, mode={args.mode!r})",
        "l2": "inputs larger than L2 (rotating sets where one set is smaller); no flush",
        "timing": "CUDA-graph replay of one step, CUDA events, max over ranks",
        "parallelism": f"weak scaling, {ws} rank(s) each a full step",
    }


def _ragged_config(wl: dict, args, ws: int) -> dict:
    return {
        "workload": wl["desc"],
        "mode": args.mode,
        "l2": "inputs larger than L2 (5.2 GB packed); no flush",
        "timing": "CUDA-graph replay of the whole ragged plan, CUDA events, max over ranks",
        "parallelism": f"weak scaling, {ws} rank(s) each a full draw",
    }


def _cpu_sample(wl: dict, shapes, args) -> tuple[list[tuple[int, int]], float]:
    """The shapes the CPU legs factor per step and the flops scale to the full step.

    The whole step, unless ``--ref-sample`` asks for a fraction of each batch
    or the workload names a smaller stand-in (1 x 32768 takes minutes per
    factorization on the host, so its CPU legs factor 1 x 16384 and scale by
    flops).
    """
    if args.ref_sample is not None:
        sample = [(max(1, int(round(b * args.ref_sample))), n) for b, n in shapes]
    else:
        sample = list(wl.get("cpu_sample", shapes))
    scale = sum(_flops(b, n) for b, n in shapes) / sum(_flops(b, n) for b, n in sample)
    return sample, scale


# ---------------------------------------------------------------------------
def run_reference(args) -> int:
    """The reference's CPU route (torch.linalg.cholesky_ex FP32, reference/reference.py:129-130)."""
    ws, rank, _ = _dist()
    if rank != 0:
        return 0
    import oracle  # the CPU leg may use the oracle package (reference route restated there)

    wl = WORKLOADS[args.workload]
    threads = os.cpu_count() or 1
    torch.set_num_threads(threads)
    if wl.get("ragged"):
        return _run_reference_ragged(args, wl, ws, threads)
    if wl.get("gp"):
        print(json.dumps({"impl": "reference", "unavailable": "the reference has no Gaussian-process or backward path (forward factorization only)"}))
        return 0
    shapes = _shapes(wl, args)
    sample, scale = _cpu_sample(wl, shapes, args)
    data = [_make(wl["gen"], b, n, s, "cpu") for (b, n), s in zip(sample, wl["seeds"])]
    for _ in range(args.warmup):
        for a in data:
            oracle.ref_kernel_cpu(a)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        for a in data:
            oracle.ref_kernel_cpu(a)
    dt = (time.perf_counter() - t0) / args.steps
    # With N GPUs every rank of the library's arm factors a full step, so the
    # whole job is N steps' work; the host cores do that work in turn.
    us = dt * 1e6 * scale * ws
    if scale == 1.0:
        desc = "the whole step (" + " + ".join(f"{b}x{n}" for b, n in sample) + ") every step"
    else:
        desc = " + ".join(f"{b}x{n}" for b, n in sample) + f" per step, scaled by flops x{scale:.2f} to the full step"
    if ws > 1:
        desc += f", x{ws} for the {ws} replicas of the whole job"
    line = {
        "impl": "reference",
        "metric": wl["metric"],
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
        "config": _dense_config(wl, args, ws, shapes),
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


def _ragged_cpu_sample(orders, offsets, host_buf=None, every: int = 50):
    """Every ``every``-th matrix of the draw (from the packed host buffer when
    given, else freshly generated with the same distribution)."""
    from gpumode_cholesky_b200 import inputs

    idx = list(range(0, len(orders), every))
    if host_buf is not None:
        mats = [host_buf[offsets[i] : offsets[i] + orders[i] ** 2].view(1, orders[i], orders[i]) for i in idx]
    else:
        mats = [inputs.well_conditioned(1, orders[i], seed=1000 + i, device="cpu") for i in idx]
    scale = sum(n**3 for n in orders) / sum(orders[i] ** 3 for i in idx)
    return mats, scale


def _run_reference_ragged(args, wl, ws: int, threads: int) -> int:
    """Reference CPU route per matrix over the whole draw, every step."""
    import oracle
    from gpumode_cholesky_b200 import inputs

    orders = inputs.ragged_orders(wl["count"], seed=wl["orders_seed"])
    mats, scale = _ragged_cpu_sample(orders, None, every=1)
    for _ in range(args.warmup):
        for m in mats:
            oracle.ref_kernel_cpu(m)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        for m in mats:
            oracle.ref_kernel_cpu(m)
    dt = (time.perf_counter() - t0) / args.steps
    us = dt * 1e6 * scale * ws  # the whole job: one draw per replica
    line = {
        "impl": "reference",
        "metric": wl["metric"],
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
        "config": _ragged_config(wl, args, ws),
        "cpu_baseline": {
            "value": round(us, 1),
            "unit": "us",
            "cores": threads,
            "kind": "reference",
            "sample": f"torch.linalg.cholesky_ex FP32 on CPU (reference ref_kernel) per matrix over the whole draw "
            f"({len(mats)} matrices) every step"
            + (f", x{ws} for the {ws} replicas of the whole job" if ws > 1 else ""),
        },
        "e2e": {"value": round(us, 1), "unit": "us", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))
    return 0


# ---------------------------------------------------------------------------
def _timed(fn, k: int) -> float:
    """Mean ms per call of k calls, CUDA events on the current stream."""
    s = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(s)
    for _ in range(k):
        fn()
    e1.record(s)
    e1.synchronize()
    return e0.elapsed_time(e1) / k


def _copy_floor_ms(host_in, dev_in, dev_out, host_out) -> float:
    """Mean ms of the same copies in both directions at once, on two streams.

    The least any host-to-host call over this link can take for these bytes.
    """
    s_in, s_out = torch.cuda.Stream(), torch.cuda.Stream()

    def copies():
        cur = torch.cuda.current_stream()
        s_in.wait_stream(cur)
        s_out.wait_stream(cur)
        with torch.cuda.stream(s_in):
            for h, d in zip(host_in, dev_in):
                d.copy_(h, non_blocking=True)
        with torch.cuda.stream(s_out):
            for d, h in zip(dev_out, host_out):
                h.copy_(d, non_blocking=True)
        cur.wait_stream(s_in)
        cur.wait_stream(s_out)

    copies()
    torch.cuda.synchronize()
    return _timed(copies, 3)


def run_ours_ragged(args, wl) -> int:
    """The ragged workload: one plan over the whole packed draw, graph-replayed."""
    ws, rank, local = _dist()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if ws > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=dev)
    from gpumode_cholesky_b200 import _lib, build, inputs
    from gpumode_cholesky_b200.potrf import resolve_mode
    from gpumode_cholesky_b200.ragged import RaggedHostPlan, RaggedPlan, autotune

    if not build.LIB_PATH.exists():
        build.build()
    _lib.load()
    orders = inputs.ragged_orders(wl["count"], seed=wl["orders_seed"])
    buf, offs = inputs.ragged_batch(orders, seed=wl["seeds"][0] + 7919 * rank, device=dev)
    offsets = offs[:-1]
    code = resolve_mode(args.mode, max(orders))
    tuned = None
    if args.autotune:
        plan, res = autotune(buf, orders, offsets, mode=code)
        tuned = sorted(({"options": o, "us": round(t, 1)} for o, t in res), key=lambda r: r["us"])
    else:
        plan = RaggedPlan(orders, offsets, mode=code, device=dev)
    out = torch.empty_like(buf)
    graph = plan.capture(buf, out)

    def barrier():
        if ws > 1:
            import torch.distributed as dist

            dist.barrier()

    clk = _clock_sampler_start(local)
    time.sleep(0.3)
    for _ in range(args.warmup):
        graph.replay()
    barrier()
    torch.cuda.synchronize()
    t_start = time.time()
    ms = _timed(graph.replay, args.steps)
    torch.cuda.synchronize()
    t_end = time.time()
    barrier()
    clocks = _clock_sampler_stop(clk, t_start, t_end)
    if ws > 1:
        import torch.distributed as dist

        t = torch.tensor([ms], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())

    with _lib.LaunchTrace() as tr:
        plan.factor(buf, out)
    totals = tr.totals()
    launches_per_step = sum(c for c, _ in totals.values())
    # Roofline of the tensor-core kernels of the padded dense groups (the
    # fused, warp-specialized and split kernels together factor every matrix
    # with n > 128): algorithmic n^3/3 flops of those matrices over their
    # time.  The groups run on several streams, so the traced (serialised)
    # per-kernel sums overstate that time; the dense kernels' time is the
    # timed step minus the other launches, which run alone on the stream.
    dense_names = [k for k in totals if k.startswith(("potrf_fused", "split_"))]
    other_ms = sum(t for k, (_, t) in totals.items() if k not in dense_names)
    big_flops = sum(n**3 / 3.0 for n in orders if n > 128)
    peaks = _measured_peaks()
    roof = None
    if dense_names:
        t_dense = max(ms - other_ms, 1e-6)
        achieved = big_flops / (t_dense / 1000.0) / 1e12
        roof = {
            "kernel": "+".join(sorted(dense_names)),
            "bound": "tensor",
            "achieved": round(achieved, 3),
            "peak": peaks["bf16_tflops"],
            "unit": "TFLOP/s",
            "frac": round(achieved / peaks["bf16_tflops"], 5),
            "peak_src": "dense BF16 cuBLAS " + peaks["src"] + " (algorithmic n^3/3 flops of the n > 128 matrices)",
            "algorithmic_flops": big_flops,
            "traffic": None,
            "share_of_step": round(t_dense / ms, 4),
            "ms": round(t_dense, 4),
        }

    extra = {}
    e2e = None
    cpu = None
    if not args.quick:
        worst = 0.0
        for n, o in zip(orders, offsets):
            if n > 1000 or n % 97 == 0:
                ld = out[o : o + n * n].view(n, n).double()
                ad = buf[o : o + n * n].view(n, n).double()
                worst = max(worst, (torch.linalg.norm(ld @ ld.T - ad) / torch.linalg.norm(ad)).item())
        extra["rel_residual_fro_max"] = worst
        extra["sum_n3_over_3"] = sum(n**3 / 3.0 for n in orders)
        # End to end: RaggedHostPlan streams runs of the list through the
        # device, copies in and out overlapping the factorization.
        host_in = buf.cpu().pin_memory()
        host_out = torch.empty_like(host_in).pin_memory()
        hplan = RaggedHostPlan(orders, offsets, mode=code, device=dev, **(dict(tuned[0]["options"]) if tuned else {}))

        def e2e_step():
            hplan.factor(host_in, host_out, non_blocking=True)

        e2e_step()
        torch.cuda.synchronize()
        e2e_ms = _timed(e2e_step, 2)
        nbytes = host_in.numel() * 4
        e2e = {
            "value": round(e2e_ms * 1000, 1),
            "unit": "us",
            "h2d_bytes_per_step": nbytes,
            "d2h_bytes_per_step": nbytes,
            "api": f"ragged.RaggedHostPlan, {len(hplan.runs)} runs",
        }
        worst_e2e = 0.0
        for n, o in zip(orders, offsets):
            if n > 1000 or n % 97 == 0:
                ld = host_out[o : o + n * n].view(n, n).to(buf.device).double()
                ad = buf[o : o + n * n].view(n, n).double()
                worst_e2e = max(worst_e2e, (torch.linalg.norm(ld @ ld.T - ad) / torch.linalg.norm(ad)).item())
        e2e["rel_residual_fro_max"] = worst_e2e
        del hplan
        dev_in = torch.empty_like(buf)
        floor_ms = _copy_floor_ms([host_in], [dev_in], [out], [host_out])
        e2e["copy_floor_us"] = round(floor_ms * 1000, 1)
        e2e["frac_of_copy_floor"] = round(floor_ms / e2e_ms, 4)
        del dev_in
        if rank == 0 and ws == 1 and not args.no_cpu:
            import oracle

            threads = os.cpu_count() or 1
            torch.set_num_threads(threads)
            mats, scale = _ragged_cpu_sample(orders, offsets, host_in, every=1)
            for m in mats:
                oracle.ref_kernel_cpu(m)
            t0 = time.perf_counter()
            for m in mats:
                oracle.ref_kernel_cpu(m)
            dt = time.perf_counter() - t0
            cpu = {
                "value": round(dt * 1e6 * scale, 1),
                "unit": "us",
                "cores": threads,
                "kind": "reference",
                "sample": f"torch.linalg.cholesky_ex FP32 on CPU (reference ref_kernel) per matrix over the whole "
                f"draw ({len(mats)} matrices)",
            }

    if rank == 0:
        line = {
            "metric": wl["metric"],
            "value": round(ms * 1000, 1),
            "unit": "us",
            "n_gpus": ws,
            "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": round(ms, 4),
            "higher_is_better": False,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "f32",
            "data": "synthetic",
            "config": _ragged_config(wl, args, ws),
            "plan_options": {k: getattr(plan.options, k) for k, _ in plan.options._fields_},
            **extra,
            "autotune": tuned,
            "matrices_per_s": round(ws * len(orders) / (ms / 1000.0), 1),
            "gflops_per_s": round(ws * sum(n**3 / 3.0 for n in orders) / (ms / 1000.0) / 1e9, 1),
            "roofline": roof,
            "kernels_one_step": {k: {"launches": c, "ms": round(t, 4)} for k, (c, t) in sorted(totals.items())},
            "cpu_baseline": cpu,
            "e2e": e2e,
            "gpu_launches": launches_per_step * args.steps,
            "clocks": clocks,
        }
        print(json.dumps(line))
    del graph
    if ws > 1:
        import torch.distributed as dist

        dist.barrier()
        dist.destroy_process_group()
    return 0


def _gp_step(pairs, gp_nll):
    grads = []
    for a, y in pairs:
        aa = a.detach().requires_grad_(True)
        loss = gp_nll(aa, y).sum()
        loss.backward()
        grads.append(aa.grad)
    return grads


def run_ours_gp(args, wl) -> int:
    """The GP workload: loss and dLoss/dA per step, eager autograd calls."""
    ws, rank, local = _dist()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if ws > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=dev)
    from gpumode_cholesky_b200 import _lib, build, gp_nll, inputs

    if not build.LIB_PATH.exists():
        build.build()
    _lib.load()
    pairs = [inputs.rbf_kernel_batch(b, n, seed=s + 7919 * rank, device=dev) for (b, n), s in zip(wl["shapes"], wl["seeds"])]
    clk = _clock_sampler_start(local)
    time.sleep(0.3)
    for _ in range(args.warmup):
        _gp_step(pairs, gp_nll)
    if ws > 1:
        import torch.distributed as dist

        dist.barrier()
    torch.cuda.synchronize()
    t_start = time.time()
    ms = _timed(lambda: _gp_step(pairs, gp_nll), args.steps)
    t_end = time.time()
    clocks = _clock_sampler_stop(clk, t_start, t_end)
    if ws > 1:
        import torch.distributed as dist

        t = torch.tensor([ms], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    with _lib.LaunchTrace() as tr:
        _gp_step(pairs, gp_nll)
        torch.cuda.synchronize()
    totals = tr.totals()
    launches = sum(c for c, _ in totals.values())
    all_ms = max(sum(t for _, t in totals.values()), 1e-12)
    dom_name, (dom_count, dom_ms) = max(totals.items(), key=lambda kv: kv[1][1])
    peaks = _measured_peaks()
    # Algorithmic flops per step: forward n^3/3, adjoint n^3 (P = Phi(L^T Lbar),
    # U = L^{-1}, Z = P U, S = U^T Z), both per matrix.
    fwd_flops = sum(b * n**3 / 3.0 for b, n in wl["shapes"])
    bwd_flops = sum(b * n**3 for b, n in wl["shapes"])
    dom_flops = bwd_flops if dom_name.startswith("bwd") else fwd_flops
    t_dom = ms * dom_ms / all_ms
    achieved = dom_flops / (t_dom / 1000.0) / 1e12
    roof = {
        "kernel": dom_name,
        "bound": "tensor" if dom_name.startswith("bwd_gemm") else "fp32",
        "achieved": round(achieved, 3),
        "peak": peaks["bf16_tflops"],
        "unit": "TFLOP/s",
        "frac": round(achieved / peaks["bf16_tflops"], 5),
        "peak_src": "dense BF16 cuBLAS " + peaks["src"] + " (algorithmic flops of the part this kernel belongs to)",
        "algorithmic_flops": dom_flops,
        "traffic": None,
        "share_of_step": round(dom_ms / all_ms, 4),
        "launches": dom_count,
        "ms": round(t_dom, 4),
    }
    extra, e2e, cpu = {}, None, None
    if not args.quick:
        grads = _gp_step(pairs, gp_nll)
        errs = {}
        for (b, n), (a, y), g in zip(wl["shapes"], pairs, grads):
            from gpumode_cholesky_b200.gp import gp_nll_grad_closed_form

            want = gp_nll_grad_closed_form(a, y)
            errs[f"{b}x{n}"] = float(torch.linalg.norm((g.double() - want).flatten()) / torch.linalg.norm(want.flatten()))
        extra["grad_rel_err_vs_fp64"] = errs
        host = [(a.cpu().pin_memory(), y.cpu().pin_memory()) for a, y in pairs]
        dev_in = [(torch.empty_like(a), torch.empty_like(y)) for a, y in pairs]
        outs = [torch.empty(a.shape, dtype=torch.float32).pin_memory() for a, _ in host]

        def e2e_step():
            for (ha, hy), (da, dy), ho in zip(host, dev_in, outs):
                da.copy_(ha, non_blocking=True)
                dy.copy_(hy, non_blocking=True)
                aa = da.detach().requires_grad_(True)
                gp_nll(aa, dy).sum().backward()
                ho.copy_(aa.grad, non_blocking=True)

        e2e_step()
        torch.cuda.synchronize()
        e2e_ms = _timed(e2e_step, max(2, args.steps // 2))
        h2d = sum(a.numel() * 4 + y.numel() * 4 for a, y in host)
        d2h = sum(o.numel() * 4 for o in outs)
        e2e = {"value": round(e2e_ms * 1000, 1), "unit": "us", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h}
        if rank == 0 and ws == 1 and not args.no_cpu:
            threads = os.cpu_count() or 1
            torch.set_num_threads(threads)
            sample, _ = _cpu_sample(wl, wl["shapes"], args)
            cpairs = [inputs.rbf_kernel_batch(b, n, seed=s, device="cpu") for (b, n), s in zip(sample, wl["seeds"])]

            def cpu_step():
                for a, y in cpairs:
                    aa = a.detach().requires_grad_(True)
                    lc = torch.linalg.cholesky(aa)
                    al = torch.linalg.solve_triangular(lc, y.unsqueeze(-1), upper=False).squeeze(-1)
                    (0.5 * (al * al).sum(-1) + torch.log(torch.diagonal(lc, dim1=-2, dim2=-1)).sum(-1)).sum().backward()

            cpu_step()
            t0 = time.perf_counter()
            cpu_step()
            dt = time.perf_counter() - t0
            scale = sum(b * n**3 for b, n in wl["shapes"]) / sum(b * n**3 for b, n in sample)
            cpu = {
                "value": round(dt * 1e6 * scale, 1),
                "unit": "us",
                "cores": threads,
                "kind": "port",
                "sample": "torch CPU FP32 autograd of the same loss (cholesky, solve_triangular, log-diagonal) on "
                + " + ".join(f"{b}x{n}" for b, n in sample)
                + f", scaled by sum b n^3 x{scale:.2f}",
            }
    if rank == 0:
        line = {
            "metric": wl["metric"],
            "value": round(ms * 1000, 1),
            "unit": "us",
            "n_gpus": ws,
            "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": round(ms, 4),
            "higher_is_better": False,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "f32",
            "data": "synthetic",
            "config": {
                "workload": wl["desc"],
                "shapes": [f"{b}x{n}" for b, n in wl["shapes"]],
                "mode": "forward fp32, adjoint bf16x3 (gp_nll defaults)",
                "l2": "inputs larger than L2 (8x2048 is 128 MB); no flush",
                "timing": "eager autograd calls (forward and backward), CUDA events, max over ranks",
                "parallelism": f"weak scaling, {ws} rank(s) each a full step",
            },
            **extra,
            "roofline": roof,
            "kernels_one_step": {k: {"launches": c, "ms": round(t, 4)} for k, (c, t) in sorted(totals.items())},
            "cpu_baseline": cpu,
            "e2e": e2e,
            "gpu_launches": launches * args.steps,
            "clocks": clocks,
        }
        print(json.dumps(line))
    if ws > 1:
        import torch.distributed as dist

        dist.barrier()
        dist.destroy_process_group()
    return 0


def run_ours(args) -> int:
    wl0 = WORKLOADS[args.workload]
    if wl0.get("ragged"):
        return run_ours_ragged(args, wl0)
    if wl0.get("gp"):
        return run_ours_gp(args, wl0)
    ws, rank, local = _dist()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if ws > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=dev)
    from gpumode_cholesky_b200 import _lib, build
    from gpumode_cholesky_b200 import checker
    from gpumode_cholesky_b200.potrf import cholesky, cholesky_host, custom_kernel

    if not build.LIB_PATH.exists():
        build.build()
    _lib.load()
    wl = WORKLOADS[args.workload]
    shapes = [(max(1, int(round(b * args.scale))), n) for b, n in wl["shapes"]]
    modes = [_resolve_mode(args.mode, n) for _, n in shapes]
    sets = [
        [_make(wl["gen"], b, n, s + 7919 * rank + 104729 * k, dev) for (b, n), s in zip(shapes, wl["seeds"])]
        for k in range(wl["sets"])
    ]
    outs = [[torch.empty_like(a) for a in st] for st in sets]
    torch.cuda.synchronize()

    drop_in = args.mode == "auto"

    def eager_step(i: int, mode_list=None):
        # The headline step is the reference-facing entry itself: one
        # custom_kernel(A) call per shape, each returning a fresh output (a
        # graph-pool tensor under capture, kept in outs).
        if mode_list is None and drop_in:
            st = sets[i % len(sets)]
            for j, a in enumerate(st):
                outs[i % len(sets)][j] = custom_kernel(a)
            return
        ml = mode_list or modes
        for a, o, m in zip(sets[i % len(sets)], outs[i % len(sets)], ml):
            cholesky(a, mode=m, out=o)

    # One CUDA graph per input set (warm-up first: kernel attributes are set outside capture).
    for i in range(len(sets)):
        eager_step(i)
    torch.cuda.synchronize()
    graphs = []
    for i in range(len(sets)):
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g):
            eager_step(i)
        graphs.append(g)
    counter = [0]

    def step():
        graphs[counter[0] % len(graphs)].replay()
        counter[0] += 1

    def barrier():
        if ws > 1:
            import torch.distributed as dist

            dist.barrier()

    clk = _clock_sampler_start(local)
    time.sleep(0.3)  # let nvidia-smi start sampling
    for _ in range(args.warmup):
        step()
    barrier()
    torch.cuda.synchronize()
    t_start = time.time()
    ms = _timed(step, args.steps)
    torch.cuda.synchronize()
    t_end = time.time()
    barrier()
    clocks = _clock_sampler_stop(clk, t_start, t_end)
    if ws > 1:
        import torch.distributed as dist

        t = torch.tensor([ms], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())

    extra = {}
    if not args.quick:
        # Per-shape times, the plain FP32 form, and cuSOLVER on the same GPU.
        per_shape = {}
        for j, ((b, n), m) in enumerate(zip(shapes, modes)):
            a, o = sets[0][j], outs[0][j]
            call = (lambda: custom_kernel(a)) if drop_in else (lambda: cholesky(a, mode=m, out=o))
            per_shape[f"{b}x{n}"] = round(1000 * _timed(call, args.steps), 1)
        plain = None
        if any(m != "fp32" for m in modes):
            plain = round(1000 * _timed(lambda: eager_step(0, ["fp32"] * len(shapes)), args.steps), 1)
        cus = round(
            1000
            * _timed(lambda: [torch.linalg.cholesky_ex(a, check_errors=False) for a in sets[0]], max(2, args.steps // 2)),
            1,
        )
        # Accuracy at full size on the device: the relative Frobenius residual
        # in FP64, and the reference checker's verdict (FP32 reconstruction).
        eager_step(0)
        resid, verdicts = {}, {}
        for (b, n), a, o in zip(shapes, sets[0], outs[0]):
            resid[f"{b}x{n}"] = float(checker.residual_norms(a, o, precision="fp64")["rel_fro"].max())
            verdicts[f"{b}x{n}"] = checker.check(a, o)[1]
        extra = {
            "per_shape_us": per_shape,
            "plain_fp32_us": plain,
            "cusolver_same_gpu_us": cus,
            "rel_residual_fro": resid,
            "reference_checker": verdicts,
        }

    # Per-kernel device time of one eager step (CUDA events on the launch stream).
    torch.cuda.synchronize()
    with _lib.LaunchTrace() as tr:
        eager_step(0)
    totals = tr.totals()
    launches_per_step = sum(c for c, _ in totals.values())
    dom_name, (dom_count, dom_ms) = max(totals.items(), key=lambda kv: kv[1][1])
    # The dominant kernel's share of one traced step, applied to the timed
    # (graph-replayed) step time: its device time inside the timed region.
    share = dom_ms / max(sum(t for _, t in totals.values()), 1e-12)
    roof = _roofline(
        args.workload, shapes, dom_name, ms * share, dom_count, tr.units().get(dom_name, 0.0), modes, _measured_peaks()
    )
    roof["share_of_step"] = round(share, 4)

    # End to end through the public API: pinned host in, host out, every step.
    # cholesky_host (b2p_potrf_batched_host) streams each shape through the
    # device in chunks, its copies in and out overlapping the factorization.
    e2e = None
    if not args.quick:
        host_in = [a.cpu().pin_memory() for a in sets[0]]
        host_out = [torch.empty_like(h).pin_memory() for h in host_in]

        def e2e_step():
            for hi, ho, m in zip(host_in, host_out, modes):
                cholesky_host(hi, mode=m, out=ho, chunk=args.e2e_chunk, non_blocking=True)

        e2e_step()
        torch.cuda.synchronize()
        e2e_ms = _timed(e2e_step, max(2, args.steps // 2))
        h2d = sum(h.numel() * 4 for h in host_in)
        e2e = {
            "value": round(e2e_ms * 1000, 1),
            "unit": "us",
            "h2d_bytes_per_step": h2d,
            "d2h_bytes_per_step": h2d,
            "api": "cholesky_host (b2p_potrf_batched_host), chunk %s" % (args.e2e_chunk or "default"),
            # Chunks pick their algorithm for their own batch size, so the
            # host result may differ from the device call's in the last bits.
            "max_abs_diff_vs_device": max(float((ho.to(o.device) - o).abs().max()) for ho, o in zip(host_out, outs[0])),
        }
        dev_in = [torch.empty_like(a) for a in sets[0]]
        floor_ms = _copy_floor_ms(host_in, dev_in, outs[0], host_out)
        e2e["copy_floor_us"] = round(floor_ms * 1000, 1)
        e2e["frac_of_copy_floor"] = round(floor_ms / e2e_ms, 4)
        del dev_in

    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu and not args.quick:
        cpu = _cpu_baseline(args, wl)

    if rank == 0:
        line = {
            "metric": wl["metric"],
            "value": round(ms * 1000, 1),
            "unit": "us",
            "n_gpus": ws,
            "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": round(ms, 4),
            "higher_is_better": False,
            "scaling": "weak",
            "vs_baseline": (
                round(ms * 1000 / wl["baseline_us"], 4) if wl.get("baseline_us") and args.scale == 1.0 and ws == 1 else None
            ),
            "dtype": "f32",
            "data": "synthetic",
            "config": _dense_config(wl, args, ws, shapes),
            **extra,
            "matrices_per_s": round(ws * sum(b for b, _ in shapes) / (ms / 1000.0), 1),
            "gflops_per_s": round(ws * sum(_flops(b, n) for b, n in shapes) / (ms / 1000.0) / 1e9, 1),
            "roofline": roof,
            "kernels_one_step": {k: {"launches": c, "ms": round(t, 4)} for k, (c, t) in sorted(totals.items())},
            "cpu_baseline": cpu,
            "e2e": e2e,
            "gpu_launches": launches_per_step * args.steps,
            "clocks": clocks,
        }
        print(json.dumps(line))
    del graphs
    if ws > 1:
        import torch.distributed as dist

        dist.barrier()
        dist.destroy_process_group()
    return 0


def _roofline(workload: str, shapes, name: str, ms: float, count: int, units: float, modes, peaks: dict) -> dict:
    """Roofline of the dominant kernel over one step.

    ``units`` is the algorithmic work the library attached to that kernel's
    launches in one traced step (the launch trace): 8*n^2 bytes per matrix
    for the HBM-bound n <= 32 warp kernel (read A, write L once), and for the
    factorization kernels the flops B*n^3/3 of the matrices those launches
    factor -- only theirs: a batch the dispatcher splits between two kernels
    credits each with its own matrices.  Update kernels carry the flops of
    their product.  Where a kernel carries none (the blocked FP32 path), its
    trailing update counts the lower triangle it updates, R(R+1)*64 per
    matrix and step.
    """
    traffic_tab = _profiled_traffic()
    if name == "potrf_warp32_kernel":
        byts = units if units > 0 else sum(8.0 * b * n * n for b, n in shapes)
        achieved = byts / (ms / count / 1000.0) / 1e9
        tpu = traffic_tab.get((name, workload, "fp32"))
        return {
            "kernel": name,
            "bound": "hbm",
            "achieved": round(achieved, 1),
            "peak": peaks["hbm_gbs"],
            "unit": "GB/s",
            "frac": round(achieved / peaks["hbm_gbs"], 4),
            "peak_src": "HBM copy " + peaks["src"],
            "algorithmic_bytes_per_launch": byts,
            "traffic": None if tpu is None else round(tpu * byts),
            "launches": count,
            "ms": round(ms, 4),
        }
    if units > 0:
        flops = units
    elif name.startswith("trail"):
        flops = 0.0
        for b, n in shapes:
            for k0 in range(0, n, 64):
                r = n - k0 - 64
                if r > 0:
                    flops += b * r * (r + 1) * 64
    else:
        flops = sum(_flops(b, n) for b, n in shapes)
    per_launch = flops / max(count, 1)
    achieved = flops / (ms / 1000.0) / 1e12
    # The guard adds a separate launch and leaves the factorization kernels
    # as they are, so their profiled traffic is that of the bare mode.
    mode = modes[-1].split("+")[0]
    tpu = traffic_tab.get((name, workload, mode))
    return {
        "kernel": name,
        "bound": "tensor",
        "achieved": round(achieved, 3),
        "peak": peaks["bf16_tflops"],
        "unit": "TFLOP/s",
        "frac": round(achieved / peaks["bf16_tflops"], 5),
        "peak_src": "dense BF16 cuBLAS " + peaks["src"] + " (algorithmic n^3/3 flops; BF16x3 issues 3 MMAs each)",
        "algorithmic_flops_per_launch": per_launch,
        "traffic": None if tpu is None else round(tpu * per_launch),
        "launches": count,
        "ms": round(ms, 4),
    }


def _cpu_baseline(args, wl) -> dict:
    """The reference's CPU route on a bounded sample, on all host cores."""
    import oracle

    threads = os.cpu_count() or 1
    torch.set_num_threads(threads)
    shapes = _shapes(wl, args)
    sample, scale = _cpu_sample(wl, shapes, args)
    data = [_make(wl["gen"], b, n, s, "cpu") for (b, n), s in zip(sample, wl["seeds"])]
    for a in data:
        oracle.ref_kernel_cpu(a)
    reps = 3
    t0 = time.perf_counter()
    for _ in range(reps):
        for a in data:
            oracle.ref_kernel_cpu(a)
    dt = (time.perf_counter() - t0) / reps
    what = " + ".join(f"{b}x{n}" for b, n in sample)
    return {
        "value": round(dt * 1e6 * scale, 1),
        "unit": "us",
        "cores": threads,
        "kind": "reference",
        "sample": "torch.linalg.cholesky_ex FP32 on CPU (reference ref_kernel) on "
        + (f"the whole step ({what}), mean of {reps}" if scale == 1.0 else f"{what}, scaled by flops x{scale:.2f}"),
    }


def main() -> int:
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=sorted(WORKLOADS), default="mid")
    ap.add_argument("--mode", default="auto")
    ap.add_argument(
        "--ref-sample", type=float, default=None, help="fraction of each batch the CPU legs factor (default: all)"
    )
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--quick", action="store_true", help="timed region and roofline only (for profiling)")
    ap.add_argument("--scale", type=float, default=1.0, help="batch scale (small profiling cases); 1 = the workload")
    ap.add_argument("--e2e-chunk", type=int, default=0, help="matrices per chunk of the e2e leg (0: library default)")
    ap.add_argument("--autotune", action="store_true", help="ragged workload: time the plan options first")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
