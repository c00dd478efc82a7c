"""CPU: the bench's reference arm keeps the JSON-line contract.

`bench.py --impl reference` times the reference's CPU route on the host
cores and prints one line; under a 2-rank launch rank 0 alone prints, and
the whole job's time covers both replicas' work.
"""

from __future__ import annotations

import json
import os
import subprocess
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parent.parent


def _lines(cmd: list[str], timeout: int = 240) -> list[dict]:
    env = dict(os.environ, PYTHONPATH=str(ROOT))
    res = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=timeout, env=env)
    assert res.returncode == 0, res.stderr[-2000:]
    return [json.loads(x) for x in res.stdout.splitlines() if x.startswith("{")]


def test_reference_arm_line_single_rank():
    out = _lines([sys.executable, "bench.py", "--impl", "reference", "--workload", "small", "--steps", "1", "--warmup", "3"])
    assert len(out) == 1
    d = out[0]
    assert d["impl"] == "reference" and d["unit"] == "us" and d["higher_is_better"] is False
    assert d["n_gpus"] == 1 and d["steps"] == 1 and d["warmup"] >= 3 and d["value"] > 0
    assert d["metric"] == "batched potrf us per step (4096x32)"
    cb = d["cpu_baseline"]
    assert cb["kind"] == "reference" and cb["cores"] >= 1 and cb["value"] == d["value"] and cb["sample"]
    assert d["e2e"] == {"value": d["value"], "unit": "us", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}


def test_reference_arm_gp_is_unavailable():
    out = _lines([sys.executable, "bench.py", "--impl", "reference", "--workload", "gp", "--steps", "1"])
    assert len(out) == 1 and out[0]["impl"] == "reference" and out[0]["unavailable"]


def test_reference_arm_two_ranks_prints_once():
    cmd = [
        sys.executable, "-m", "torch.distributed.run", "--standalone", "--local-addr", "127.0.0.1",
        "--nnodes=1", "--nproc-per-node", "2",
        "bench.py", "--impl", "reference", "--gpus", "2", "--workload", "small", "--steps", "1", "--warmup", "3",
    ]
    out = _lines(cmd, timeout=300)
    assert len(out) == 1
    d = out[0]
    assert d["n_gpus"] == 2 and d["impl"] == "reference"
    assert "x2 for the 2 replicas" in d["cpu_baseline"]["sample"]
