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

Validation shards with one exchange step: every rank holds the whole mesh
and tests the candidate overlap pairs whose first shared grid cell lies in
its band of cell rows (``band_rows``); the per-triangle overlap bits are
combined by an all-reduce MAX (``allreduce_max``) and the pair counts by a
SUM (``allreduce_sum``), after which every rank holds the whole report
(``engine.validate.validate_uvs(..., group=...)``).
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


def rank_world(group=None):
    """(rank, world) of an explicit process group; (0, 1) without one (a
    validation without a group is a whole, local one)."""
    if group is None:
        return 0, 1
    import torch.distributed as dist
    return dist.get_rank(group), dist.get_world_size(group)


def band_rows(G, rank, world):
    """Cell rows [lo, hi) of a rank's band of a G x G validation grid (the
    rows uva_validate's pair kernels keep for shard rank of world)."""
    return (G * rank) // world, (G * (rank + 1)) // world


def _allreduce(t, op, group):
    import torch.distributed as dist
    if t.is_cuda and dist.get_backend(group) == "gloo":   # gloo reduces host tensors
        h = t.cpu()
        dist.all_reduce(h, op=op, group=group)
        return h.to(t.device)
    dist.all_reduce(t, op=op, group=group)
    return t


def allreduce_max(t, group=None):
    """Element-wise maximum over the ranks of `group` (in place when the
    backend reduces the tensor where it lives); returns the result."""
    import torch.distributed as dist
    return _allreduce(t, dist.ReduceOp.MAX, group)


def allreduce_sum(t, group=None):
    """Element-wise sum over the ranks of `group`; returns the result."""
    import torch.distributed as dist
    return _allreduce(t, dist.ReduceOp.SUM, group)
