"""Splitting independent references across GPUs (one process per GPU).

A single reference does not shard: every doubling round needs the whole rank
array.  A collection of references does: each GPU builds its own share with
no data-path collective, and only the timings are reduced.  Shares are
assigned by longest-processing-time bin packing on each reference's device
footprint (``sufgpu_device_bytes``, which grows linearly with its length), so
every GPU gets about the same HBM and work; every rank computes the same
assignment from the same sizes.
"""
from __future__ import annotations

import heapq
from typing import Sequence

import numpy as np


def assign(sizes: Sequence[int], ranks: int) -> list[list[int]]:
    """Indices of `sizes` per rank: largest first, each to the least loaded
    rank (ties by rank number; deterministic).  Indices inside a share are in
    ascending order."""
    if ranks < 1:
        raise ValueError("ranks must be at least 1")
    heap = [(0, r) for r in range(ranks)]
    shares: list[list[int]] = [[] for _ in range(ranks)]
    for i in sorted(range(len(sizes)), key=lambda j: (-int(sizes[j]), j)):
        load, r = heapq.heappop(heap)
        shares[r].append(i)
        heapq.heappush(heap, (load + int(sizes[i]), r))
    return [sorted(s) for s in shares]


def _reduce(value: float, dist, device, op: str) -> float:
    if dist is None:
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=getattr(dist.ReduceOp, op))
    return float(t.item())


def max_over_ranks(value: float, dist=None, device=None) -> float:
    """The largest `value` over all ranks of the default process group (the
    slowest GPU's time); the value itself without one."""
    return _reduce(value, dist, device, "MAX")


def sum_over_ranks(value: float, dist=None, device=None) -> float:
    """The sum of `value` over all ranks (the symbols all shares hold)."""
    return _reduce(value, dist, device, "SUM")


def collection_share(count: int, world: int, rank: int, scale: float = 1.0):
    """This rank's share of a bacterial collection of `count` references:
    (indices, logical texts).  Only the share's sequences are generated; each
    reference has its own random stream, so the shares of all ranks together
    are the collection built on one GPU from the same indices."""
    from . import synth
    sizes = synth.uneven_sizes(count, scale)
    mine = assign([s + 1 for s in sizes], world)[rank]
    texts: list[np.ndarray] = [synth.uneven_reference(i, sizes[i]).logical_text()
                               for i in mine]
    return mine, texts
