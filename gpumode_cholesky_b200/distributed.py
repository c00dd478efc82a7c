"""Sharding independent matrices across ranks (one process per GPU).

The factorizations of different matrices are independent, so a batch shards
with no collective on the data path: each rank factors its own slice and, if
the caller wants the whole result on every rank, one all-gather moves the
factors (NCCL over NVLink between GPUs, gloo on CPU).  A ragged list is split
by cost (sum of n^3) with the longest-processing-time rule so that ranks
finish together.  A single large matrix is not split (replicas only).
"""

from __future__ import annotations

from collections.abc import Callable, Sequence

import torch
import torch.distributed as dist


def shard_range(batch: int, world: int, rank: int) -> tuple[int, int]:
    """Contiguous slice [start, stop) of a batch for `rank` of `world` (sizes differ by at most 1)."""
    if world <= 0 or not 0 <= rank < world:
        raise ValueError("bad world/rank")
    q, r = divmod(batch, world)
    start = rank * q + min(rank, r)
    return start, start + q + (1 if rank < r else 0)


def partition_by_cost(orders: Sequence[int], world: int) -> list[list[int]]:
    """Assign matrix indices to ranks, balancing sum(n^3): largest first onto the lightest rank."""
    loads = [0.0] * world
    parts: list[list[int]] = [[] for _ in range(world)]
    for i in sorted(range(len(orders)), key=lambda j: -orders[j]):
        r = min(range(world), key=lambda k: loads[k])
        parts[r].append(i)
        loads[r] += float(orders[i]) ** 3
    for p in parts:
        p.sort()
    return parts


def _default_factor(a: torch.Tensor) -> torch.Tensor:
    from .potrf import cholesky

    return cholesky(a)


def factor_sharded(
    a: torch.Tensor,
    group=None,
    factor_fn: Callable[[torch.Tensor], torch.Tensor] | None = None,
    gather: bool = True,
) -> torch.Tensor:
    """Factor a (batch, n, n) batch split across the ranks of `group`.

    Every rank passes the same full `a` (or at least its own slice).  With
    gather=True every rank returns the full L (all-gather); otherwise each
    returns only its slice.
    """
    fn = factor_fn or _default_factor
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    batch = a.shape[0]
    lo, hi = shard_range(batch, world, rank)
    mine = fn(a[lo:hi].contiguous()) if hi > lo else a[lo:hi].clone()
    if not gather:
        return mine
    # all_gather needs equal sizes: pad every shard to the largest one.
    width = shard_range(batch, world, 0)[1]
    buf = torch.zeros((width,) + tuple(a.shape[1:]), dtype=mine.dtype, device=mine.device)
    buf[: hi - lo] = mine
    outs = [torch.empty_like(buf) for _ in range(world)]
    dist.all_gather(outs, buf, group=group)
    pieces = []
    for r in range(world):
        s, e = shard_range(batch, world, r)
        pieces.append(outs[r][: e - s])
    return torch.cat(pieces, dim=0)


def factor_ragged_sharded(
    mats: Sequence[torch.Tensor],
    group=None,
    factor_fn: Callable[[torch.Tensor], torch.Tensor] | None = None,
) -> list[torch.Tensor]:
    """Factor a list of square matrices split by cost; every rank gets all factors back.

    `factor_fn` takes a (batch, n, n) tensor.  Each rank factors its share one
    matrix at a time and the factors are exchanged with all_gather_object
    (host objects; intended for the ragged tail, the bulk should use the
    ragged plan on each rank).
    """
    fn = factor_fn or _default_factor
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    parts = partition_by_cost([int(m.shape[-1]) for m in mats], world)
    mine = {i: fn(mats[i].unsqueeze(0))[0].cpu() for i in parts[rank]}
    gathered: list[dict] = [None] * world  # type: ignore[list-item]
    dist.all_gather_object(gathered, mine, group=group)
    out: dict[int, torch.Tensor] = {}
    for d in gathered:
        out.update(d)
    return [out[i] for i in range(len(mats))]
