"""torchrun worker for tests/test_distributed_gpu.py (not collected by pytest).

One process per GPU over NCCL.  Every rank factors its shard of a dense batch
and of a ragged list through the library's CUDA path, gathers the factors, and
checks them bitwise against the same library call on the whole input.  Rank 0
writes "ok" (or the failure) to the file named by argv[1].
"""

from __future__ import annotations

import datetime
import os
import sys

import torch
import torch.distributed as dist

sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), ".."))

from gpumode_cholesky_b200 import cholesky, inputs  # noqa: E402
from gpumode_cholesky_b200.distributed import factor_ragged_sharded, factor_sharded  # noqa: E402


def main() -> int:
    out_path = sys.argv[1]
    local = int(os.environ["LOCAL_RANK"])
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=60), device_id=dev)
    rank = dist.get_rank()
    msg = "ok"
    try:
        factor = lambda x: cholesky(x, mode="auto")  # noqa: E731
        a = inputs.well_conditioned(37, 256, seed=5, device=dev)
        got = factor_sharded(a, factor_fn=factor)
        want = factor(a)
        if not torch.equal(got, want):
            msg = "dense shards differ: max %g" % float((got - want).abs().max())
        mats = [inputs.well_conditioned(1, n, seed=n, device=dev)[0] for n in (32, 100, 192, 320, 512)]
        rg = factor_ragged_sharded(mats, factor_fn=factor)
        for m, g in zip(mats, rg):
            w = factor(m.unsqueeze(0))[0].cpu()
            if not torch.equal(g, w):
                msg = "ragged shard of order %d differs" % m.shape[-1]
        torch.cuda.synchronize()
        dist.barrier()
    except Exception as e:  # reported to the test through the file
        msg = "error: %r" % (e,)
    finally:
        dist.destroy_process_group()
    if rank == 0:
        with open(out_path, "w") as f:
            f.write(msg)
    return 0 if msg == "ok" else 1


if __name__ == "__main__":
    sys.exit(main())
