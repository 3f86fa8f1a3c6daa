"""Rows across GPUs: one process per GPU, rows split into contiguous ranges.

Rows are independent, so a batch shards with no collective on the data path:
rank r selects the rows of its range on its own GPU and writes its own slice of
the outputs.  ``gather_rows`` is only for callers that want every row's
results on one rank (an ``all_gather`` of the per-rank slices).
"""
from __future__ import annotations

import bisect
from typing import List, Sequence, Tuple


def shard_rows(lengths: Sequence[int], world: int, rank: int) -> Tuple[int, int]:
    """[first, last) row range of ``rank``: contiguous ranges with about equal
    sums of n (the keys each GPU reads); with at least ``world`` rows every
    range is non-empty."""
    if world <= 0 or not 0 <= rank < world:
        raise ValueError("bad world / rank")
    B = len(lengths)
    prefix = [0]
    for n in lengths:
        prefix.append(prefix[-1] + int(n))
    total = prefix[-1]
    cuts = [0]
    for r in range(1, world):
        target = r * total / world
        i = bisect.bisect_left(prefix, target)
        lo = cuts[-1] + (1 if B >= world else 0)
        hi = B - (world - r) if B >= world else B
        cuts.append(min(max(i, lo), hi))
    cuts.append(B)
    return cuts[rank], cuts[rank + 1]


def shard_bounds(lengths: Sequence[int], world: int) -> List[Tuple[int, int]]:
    return [shard_rows(lengths, world, r) for r in range(world)]


def gather_rows(vals, idx, k: int, lengths: Sequence[int], group=None):
    """All-gathers per-rank (vals [b_r, k], idx [b_r, k]) slices, in rank
    order, into full (vals [B, k], idx [B, k]) on every rank."""
    import torch
    import torch.distributed as dist

    world = dist.get_world_size(group)
    bounds = shard_bounds(lengths, world)
    Bmax = max(b - a for a, b in bounds)
    pv = torch.zeros((Bmax, k), dtype=vals.dtype, device=vals.device)
    pi = torch.zeros((Bmax, k), dtype=idx.dtype, device=idx.device)
    pv[: vals.shape[0]] = vals
    pi[: idx.shape[0]] = idx
    gv = [torch.empty_like(pv) for _ in range(world)]
    gi = [torch.empty_like(pi) for _ in range(world)]
    dist.all_gather(gv, pv, group=group)
    dist.all_gather(gi, pi, group=group)
    out_v = torch.cat([g[: b - a] for g, (a, b) in zip(gv, bounds)])
    out_i = torch.cat([g[: b - a] for g, (a, b) in zip(gi, bounds)])
    return out_v, out_i
