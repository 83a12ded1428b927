"""Sharding a compression job over several GPUs (one process per GPU).

Members are independent and the path has no exchange step, so a job shards
by partitioning its inputs: each rank compresses a contiguous range of the
input list on its own device (its own context, pool and queue) and the
results are put back in input order on the host.  Nothing crosses NVLink on
the data path; the only collective is the final gather of the finished
gzip streams to the rank that writes them, which is host-side plumbing
(`torch.distributed` object gather, gloo or NCCL).

The reference drives one GPU per process and has no multi-GPU mode; this is
the weak-scaling replacement for running several gpzip processes side by
side.
"""
from __future__ import annotations

from typing import Callable, List, Optional, Sequence, Tuple


def partition(sizes: Sequence[int], world: int) -> List[Tuple[int, int]]:
    """Contiguous [lo, hi) index ranges, one per rank, balanced by bytes.

    A boundary is placed after the last item whose midpoint lies at or below
    r / world of the total, so every rank gets within one item of an equal
    byte share.  Ranges are contiguous and in order, so concatenating the
    ranks' outputs rank by rank gives the input order back.  Ranks may get
    empty ranges when there are fewer items than ranks.
    """
    if world < 1:
        raise ValueError("world must be >= 1")
    total = sum(int(s) for s in sizes)
    k = len(sizes)
    bounds = [0]
    acc = 0
    i = 0
    for r in range(1, world):
        target = total * r / world
        while i < k and acc + sizes[i] / 2 <= target:
            acc += sizes[i]
            i += 1
        bounds.append(max(i, bounds[-1]))
    bounds.append(k)
    return [(bounds[r], bounds[r + 1]) for r in range(world)]


def compress_shard(items: Sequence[bytes], rank: int, world: int,
                   compress: Callable[[Sequence[bytes]], List[bytes]]) -> Tuple[int, List[bytes]]:
    """Compresses this rank's range of ``items`` with ``compress`` (for
    example ``Context.compress_batch`` of this rank's device context).
    Returns (first index, gzip streams of the range)."""
    lo, hi = partition([len(x) for x in items], world)[rank]
    return lo, [bytes(x) for x in compress(items[lo:hi])] if hi > lo else []


def assemble(parts: Sequence[Tuple[int, List[bytes]]], count: int) -> List[bytes]:
    """Puts the ranks' (first index, streams) parts back in input order and
    checks that every item is present exactly once."""
    out: List[Optional[bytes]] = [None] * count
    for lo, streams in parts:
        for j, s in enumerate(streams):
            if out[lo + j] is not None:
                raise ValueError(f"item {lo + j} returned twice")
            out[lo + j] = s
    missing = [i for i, s in enumerate(out) if s is None]
    if missing:
        raise ValueError(f"items missing from the gathered parts: {missing[:8]}")
    return out  # type: ignore[return-value]


def compress_distributed(items: Sequence[bytes], compress: Callable[[Sequence[bytes]], List[bytes]],
                         group=None, dst: int = 0) -> Optional[List[bytes]]:
    """Every rank calls this with the same ``items``; rank ``dst`` returns the
    gzip streams of all of them in input order, the other ranks None."""
    import torch.distributed as dist

    rank, world = dist.get_rank(group), dist.get_world_size(group)
    part = compress_shard(items, rank, world, compress)
    gathered = [None] * world if rank == dst else None
    dist.gather_object(part, gathered, dst=dst, group=group)
    if rank != dst:
        return None
    return assemble(gathered, len(items))
