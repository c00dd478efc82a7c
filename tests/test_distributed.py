"""CPU: sharding logic on world-size-2 gloo process groups (no GPU).

The factor function is the FP32 oracle (tests may use it as the checker);
the GPU path plugs the library's cholesky in its place.
"""

from __future__ import annotations

import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from gpumode_cholesky_b200 import inputs
from gpumode_cholesky_b200.distributed import factor_ragged_sharded, factor_sharded, partition_by_cost, shard_range


def _oracle_factor(a: torch.Tensor) -> torch.Tensor:
    import oracle

    l, _ = oracle.potrf_f32(a.numpy())
    return torch.from_numpy(l)


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank: int, world: int, port: int, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=__import__("datetime").timedelta(seconds=60))
    try:
        a = inputs.generate_input(5, 12, 2, 31, "dense", device="cpu")
        full = factor_sharded(a, factor_fn=_oracle_factor)
        want = _oracle_factor(a)
        ok_dense = bool(torch.equal(full, want))
        mats = [inputs.generate_input(1, n, 2, 40 + n, "dense", device="cpu")[0] for n in (3, 40, 9, 17, 25)]
        got = factor_ragged_sharded(mats, factor_fn=_oracle_factor)
        ok_ragged = all(torch.equal(g, _oracle_factor(m.unsqueeze(0))[0]) for g, m in zip(got, mats))
        q.put((rank, ok_dense, ok_ragged))
    finally:
        dist.destroy_process_group()


def test_shard_range_covers_batch():
    for batch in (0, 1, 7, 640):
        for world in (1, 2, 3, 8):
            spans = [shard_range(batch, world, r) for r in range(world)]
            assert spans[0][0] == 0 and spans[-1][1] == batch
            assert all(spans[i][1] == spans[i + 1][0] for i in range(world - 1))
            sizes = [e - s for s, e in spans]
            assert max(sizes) - min(sizes) <= 1


def test_partition_by_cost_balances():
    orders = inputs.ragged_orders(3000, seed=4)
    parts = partition_by_cost(orders, 8)
    assert sorted(i for p in parts for i in p) == list(range(3000))
    loads = [sum(orders[i] ** 3 for i in p) for p in parts]
    assert max(loads) / min(loads) < 1.05


def test_gloo_world2_sharded_factorization():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(2)]
    for p in procs:
        p.join(timeout=60)
    assert all(p.exitcode == 0 for p in procs)
    assert sorted(r for r, _, _ in res) == [0, 1]
    assert all(d and g for _, d, g in res), res
