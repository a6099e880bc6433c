"""Frames across GPUs: one process per GPU, each coding its own share of a
batch, no collective on the data path (frames are independent). Shares are
balanced by macroblock count; timings are reduced to the slowest rank."""

from __future__ import annotations

from typing import List, Sequence, Tuple


def macroblocks(width: int, height: int) -> int:
    return ((width + 15) // 16) * ((height + 15) // 16)


def shard_by_macroblocks(sizes: Sequence[Tuple[int, int]], world: int) -> List[List[int]]:
    """Frame indices for each rank: the largest frames first, each to the rank
    with the fewest macroblocks so far (ties to the lower rank). The same
    split as the library's prores_shard_frames, which its multi-device batch
    calls use."""
    order = sorted(range(len(sizes)), key=lambda i: (-macroblocks(*sizes[i]), i))
    load = [0] * world
    shards: List[List[int]] = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        shards[r].append(i)
        load[r] += macroblocks(*sizes[i])
    return [sorted(s) for s in shards]


def max_over_ranks(values: Sequence[float], dist=None, device=None) -> List[float]:
    """Element-wise maximum of `values` over all ranks (identity alone)."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return list(values)
    import torch

    t = torch.tensor(list(values), dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(x) for x in t.tolist()]
