"""Sharding a batch of independent circuits over GPUs (one process per GPU).

Monte Carlo instances share nothing, so a batch splits into one shard per
rank with no exchange during the solve: each rank builds the NewtonBatch of
its own instances in its own HBM, and the only collective is the gather of
per-instance status (and, when a caller wants them, the solutions) at the
end.  Instances are assigned longest-processing-time first: in decreasing
order of weight (the circuit's component count, a proxy for its nonzeros
and Krylov work known before compiling), each to the least-loaded shard, so
that the slowest rank, which sets the batch time, carries at most the mean
load plus one instance.  Every rank computes the same partition from the
same weights; nothing is communicated to agree on it.
"""
from __future__ import annotations

import heapq

import numpy as np


def lpt_partition(weights, n_shards: int) -> list[np.ndarray]:
    """Instance indices of each shard (increasing order within a shard).
    Ties in weight go to the lower index first; ties in load to the lower
    shard, so the result is deterministic."""
    if n_shards < 1:
        raise ValueError("n_shards must be >= 1")
    w = np.asarray(weights, dtype=np.float64)
    order = np.lexsort((np.arange(w.size), -w))        # weight descending, then index
    heap = [(0.0, s) for s in range(n_shards)]
    members: list[list[int]] = [[] for _ in range(n_shards)]
    for i in order:
        load, s = heapq.heappop(heap)
        members[s].append(int(i))
        heapq.heappush(heap, (load + float(w[i]), s))
    return [np.array(sorted(m), dtype=np.int64) for m in members]


def shard_loads(weights, shards) -> np.ndarray:
    w = np.asarray(weights, dtype=np.float64)
    return np.array([float(w[s].sum()) for s in shards])


def gather_status(local_status, local_index, n_total: int, group=None) -> np.ndarray:
    """Per-instance status codes of the whole batch on every rank: the one
    collective of a sharded batch solve (an all-gather of each rank's
    (instance, status) pairs over the default process group)."""
    import torch.distributed as dist

    pairs = list(zip([int(i) for i in local_index], [int(s) for s in local_status]))
    if not dist.is_initialized() or dist.get_world_size(group) == 1:
        parts = [pairs]
    else:
        parts = [None] * dist.get_world_size(group)
        dist.all_gather_object(parts, pairs, group=group)
    out = np.full(n_total, -1, dtype=np.int64)
    for part in parts:
        for i, s in part:
            out[i] = s
    return out
