"""Multi-GPU sharding of the alignment path (one process per GPU).

Pairs and reads are independent units, so the path shards with no exchange
on the data path: every rank takes a longest-processing-time share of the
units (cost = in-band DP cells for extension pairs, anchors for chaining
reads), aligns it on its own GPU, and only timings (max over ranks) or, if a
caller wants them, results cross ranks.  No collective and no load from
another GPU's memory touches the alignment data.
"""

from __future__ import annotations

import heapq
from typing import Optional

import numpy as np


def lpt_partition(costs: np.ndarray, n_ranks: int) -> list:
    """Units in decreasing cost order, each to the least-loaded rank so far
    (ties: lowest rank).  Returns each rank's unit indices, ascending.  The
    largest load is at most the mean load plus the largest unit cost."""
    costs = np.asarray(costs, dtype=np.float64)
    if n_ranks < 1:
        raise ValueError("n_ranks must be >= 1")
    order = np.argsort(-costs, kind="stable")
    heap = [(0.0, r) for r in range(n_ranks)]
    parts: list = [[] for _ in range(n_ranks)]
    for u in order:
        load, r = heapq.heappop(heap)
        parts[r].append(int(u))
        heapq.heappush(heap, (load + float(costs[u]), r))
    return [np.sort(np.array(p, dtype=np.int64)) for p in parts]


def pair_costs(pairs) -> np.ndarray:
    from .synth import band_cells

    return band_cells(pairs.query_len, pairs.target_len, pairs.half_band, pairs.band_offset).astype(np.float64)


def read_costs(anchors) -> np.ndarray:
    return np.diff(np.asarray(anchors.read_off, np.int64)).astype(np.float64)


def shard_pairs(pairs, rank: int, world: int):
    """This rank's share of an extension batch: (PairSet, original indices)."""
    idx = lpt_partition(pair_costs(pairs), world)[rank]
    return pairs.subset(idx), idx


def shard_reads(anchors, rank: int, world: int) -> np.ndarray:
    """Indices of this rank's reads of a chaining batch."""
    return lpt_partition(read_costs(anchors), world)[rank]


def max_over_ranks(x: float, group=None, device: Optional[str] = None) -> float:
    """The largest value of ``x`` over the ranks (e.g. a step time measured
    on each rank's device); ``x`` itself without an initialised process
    group."""
    import torch
    import torch.distributed as dist

    if not dist.is_available() or not dist.is_initialized():
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=device or "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    return float(t.item())
