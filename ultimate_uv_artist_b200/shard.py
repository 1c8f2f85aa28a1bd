"""Islands across ranks (one process per GPU).

Islands are independent and every solve is block-diagonal, so a batch shards
by islands with no exchange on the data path: each rank builds its own
DeviceBatch and runs its own persistent launches. The only collectives are
the final gather of per-island results and the reduction of step timings.

* ``lpt_partition``: greedy longest-processing-time assignment of islands to
  ranks by a cost (triangle count by default), deterministic, so every rank
  computes the same partition without communication.
* ``gather_chart_uvs``: per-island UV arrays of all ranks back in the
  original island order (on every rank, or on rank 0 only).
* ``reduce_step``: max over ranks of a step time and sum of the units done.
"""
from __future__ import annotations

import heapq

import numpy as np


def lpt_partition(costs, world):
    """List of ``world`` int64 index arrays (ascending): island i goes to the
    rank with the least assigned cost, islands taken by decreasing cost
    (ties: lower island index first, lower rank first)."""
    costs = np.asarray(costs, np.float64)
    world = int(world)
    if world < 1:
        raise ValueError("world must be >= 1")
    order = np.lexsort((np.arange(len(costs)), -costs))
    heap = [(0.0, r) for r in range(world)]
    parts = [[] for _ in range(world)]
    for i in order:
        load, r = heapq.heappop(heap)
        parts[r].append(int(i))
        heapq.heappush(heap, (load + float(costs[i]), r))
    return [np.array(sorted(p), np.int64) for p in parts]


def shard_charts(charts, rank, world, costs=None):
    """(indices, charts) of this rank's share; ``charts`` items are
    (P, T[, U]) as for gpu.Batch."""
    if costs is None:
        costs = [len(ch[1]) for ch in charts]
    idx = lpt_partition(costs, world)[int(rank)]
    return idx, [charts[i] for i in idx]


def gather_chart_uvs(local_uvs, indices, n_total, group=None, dst=None):
    """Per-island UV arrays of every rank in the original island order.
    ``dst=None``: every rank gets the list; else only rank ``dst`` (others get
    None). Uses torch.distributed object collectives (any backend)."""
    import torch.distributed as dist
    payload = (np.asarray(indices, np.int64), [np.asarray(u) for u in local_uvs])
    world = dist.get_world_size(group)
    if dst is None:
        parts = [None] * world
        dist.all_gather_object(parts, payload, group=group)
    else:
        parts = [None] * world if dist.get_rank(group) == dst else None
        dist.gather_object(payload, parts, dst=dst, group=group)
        if parts is None:
            return None
    out = [None] * int(n_total)
    for idx, uvs in parts:
        for i, u in zip(idx.tolist(), uvs):
            out[i] = u
    if any(u is None for u in out):
        raise RuntimeError("gather_chart_uvs: some islands were not produced by any rank")
    return out


def reduce_step(ms, units, device=None, group=None):
    """(max over ranks of ``ms``, sum over ranks of ``units``)."""
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(ms), float(units)], dtype=torch.float64, device=device)
    mx = t.clone()
    dist.all_reduce(mx, op=dist.ReduceOp.MAX, group=group)
    sm = t.clone()
    dist.all_reduce(sm, op=dist.ReduceOp.SUM, group=group)
    return float(mx[0]), float(sm[1])
