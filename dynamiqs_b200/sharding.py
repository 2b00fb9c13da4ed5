"""Sharding independent mesolve instances over the ranks of a process group.

Instances are independent ODEs, so a batch splits across GPUs with no exchange on the
data path: each rank solves a contiguous block of the flattened batch
(:func:`shard_range`), timings are combined as the maximum over ranks
(:func:`max_over_ranks`), and results can be collected on one rank afterwards
(:func:`gather_to`).  One process per GPU; ``torch.distributed`` (NCCL on GPUs, gloo on
CPU) is the plumbing.
"""

from __future__ import annotations

import numpy as np

__all__ = ['shard_range', 'max_over_ranks', 'gather_to', 'sharded_solve']


def shard_range(batch: int, rank: int, world: int) -> tuple[int, int]:
    """[start, stop) of the instances owned by ``rank``: contiguous blocks whose sizes
    differ by at most one."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f'bad rank {rank} for world size {world}')
    base, extra = divmod(batch, world)
    start = rank * base + min(rank, extra)
    return start, start + base + (1 if rank < extra else 0)


def max_over_ranks(value: float, group=None, device=None) -> float:
    """Maximum of a per-rank scalar (e.g. a CUDA-event time) over the group."""
    import torch
    import torch.distributed as dist

    if not dist.is_initialized() or dist.get_world_size(group) == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    return float(t.item())


def gather_to(local, dst: int = 0, group=None):
    """Concatenate every rank's leading-axis block on rank ``dst`` (others get None).
    Blocks may differ in length by one (see :func:`shard_range`)."""
    import torch
    import torch.distributed as dist

    if not dist.is_initialized() or dist.get_world_size(group) == 1:
        return local
    world = dist.get_world_size(group)
    n = torch.tensor([local.shape[0]], dtype=torch.int64, device=local.device)
    sizes = [torch.zeros_like(n) for _ in range(world)]
    dist.all_gather(sizes, n, group=group)
    m = int(max(int(s) for s in sizes))
    pad = torch.zeros((m, *local.shape[1:]), dtype=local.dtype, device=local.device)
    pad[: local.shape[0]] = local
    parts = [torch.zeros_like(pad) for _ in range(world)]
    dist.all_gather(parts, pad, group=group)
    if dist.get_rank(group) != dst:
        return None
    return torch.cat([p[: int(s)] for p, s in zip(parts, sizes)])


def sharded_solve(solve, batch_items, rank: int, world: int):
    """Run ``solve`` on this rank's block of ``batch_items`` (any sliceable batch) and
    return (start, stop, result)."""
    start, stop = shard_range(len(batch_items), rank, world)
    return start, stop, solve(batch_items[start:stop])


def flat_shard(x: np.ndarray, rank: int, world: int) -> np.ndarray:
    start, stop = shard_range(x.shape[0], rank, world)
    return x[start:stop]
