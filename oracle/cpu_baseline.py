"""Timed CPU baseline of the batched LSCM + ARAP workload (test / bench
infrastructure only): the oracle's restatement of the reference's per-chart
CPU path, param.lscm + param.refine (engine/param.py:136-169, 379-414), run
chart by chart over a process pool of the host's cores, the way the reference
pipeline fans charts out over a thread pool (engine/pipeline.py:608-610).
"""
from __future__ import annotations

import multiprocessing as mp
import os
import time

import numpy as np


def _solve_one(args):
    P, T, iters = args
    from oracle import arap as O
    P = np.asarray(P, np.float64)
    U = O.lscm(P, T)
    U = O.refine_arap(P, T, U, iters=iters, line_search=True, tol=0.0)
    return len(T)


def sample_islands(islands, budget_tris):
    """Every k-th island of the size-sorted list, so the sample keeps the size
    distribution; stops at about ``budget_tris`` triangles."""
    order = np.argsort([len(t) for _, t in islands])
    total = sum(len(t) for _, t in islands)
    k = max(1, int(round(total / max(budget_tris, 1))))
    pick = order[::k]
    return [islands[i] for i in pick]


def time_cpu(islands, iters, workers=None, repeats=1):
    """Returns (tris*iters per second, seconds, workers, triangles)."""
    workers = workers or os.cpu_count() or 1
    ctx = mp.get_context("spawn")
    jobs = [(p, t, iters) for p, t in sorted(islands, key=lambda x: -len(x[1]))]
    tris = sum(len(t) for _, t in islands)
    best = None
    with ctx.Pool(workers) as pool:
        pool.map(_solve_one, jobs[:min(len(jobs), workers)])   # warm the workers' imports
        for _ in range(repeats):
            t0 = time.perf_counter()
            pool.map(_solve_one, jobs, chunksize=1)
            dt = time.perf_counter() - t0
            best = dt if best is None else min(best, dt)
    return tris * iters / best, best, workers, tris
