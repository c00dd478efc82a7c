"""GPU: the sharded entry points over NCCL, one process per GPU under torchrun.

The pool gives one GPU per run, so this runs world size 1 (every collective
on the NCCL path, the shard arithmetic trivial); the world-size-2 sharding
logic is covered on CPU with gloo (tests/test_distributed.py).
"""

from __future__ import annotations

import os
import socket
import subprocess
import sys

import pytest
import torch

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_nccl_sharded_factorization(tmp_path):
    assert torch.cuda.is_available()
    out = tmp_path / "result.txt"
    cmd = [
        sys.executable,
        "-m",
        "torch.distributed.run",
        "--nnodes=1",
        "--nproc-per-node=1",
        "--master-addr=127.0.0.1",
        "--master-port=%d" % _free_port(),
        os.path.join(HERE, "_dist_gpu_worker.py"),
        str(out),
    ]
    env = dict(os.environ, NCCL_NVLS_ENABLE="0")
    res = subprocess.run(cmd, capture_output=True, text=True, timeout=300, env=env)
    assert res.returncode == 0, res.stdout[-2000:] + res.stderr[-2000:]
    assert out.read_text() == "ok"
