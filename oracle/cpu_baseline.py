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
    return U


def sample_indices(islands, budget_tris):
    """Every k-th island of the size-sorted list, so the sample keeps the size
    distribution; stops at about ``budget_tris`` triangles."""
    order = np.argsort([len(t) for _, t in islands])
    total = sum(len(t) for _, t in islands)
    k = max(1, int(round(total / max(budget_tris, 1))))
    return order[::k]


def sample_islands(islands, budget_tris):
    return [islands[i] for i in sample_indices(islands, budget_tris)]


def time_cpu(islands, iters, workers=None, repeats=1, return_uv=False):
    """Returns (tris*iters per second, seconds, workers, triangles), plus the
    FP64 UVs of every island (input order) when ``return_uv``."""
    workers = workers or os.cpu_count() or 1
    ctx = mp.get_context("spawn")
    order = sorted(range(len(islands)), key=lambda i: -len(islands[i][1]))   # largest first
    jobs = [(islands[i][0], islands[i][1], iters) for i in order]
    tris = sum(len(t) for _, t in islands)
    best = None
    uvs = None
    with ctx.Pool(workers) as pool:
        pool.map(_solve_one, jobs[:min(len(jobs), workers)])   # warm the workers' imports
        for _ in range(repeats):
            t0 = time.perf_counter()
            out = pool.map(_solve_one, jobs, chunksize=1)
            dt = time.perf_counter() - t0
            best = dt if best is None else min(best, dt)
            uvs = [None] * len(islands)
            for i, u in zip(order, out):
                uvs[i] = u
    if return_uv:
        return tris * iters / best, best, workers, tris, uvs
    return tris * iters / best, best, workers, tris


def uv_error_batch(islands, uvs, iters, count=12):
    """Checker of the GPU bench result: the FP64 oracle of the batched path
    (LSCM with far-pair pins, engine/param.py:136-179, then gpu.Batch.arap
    semantics, engine/gpu.py:230-249, with exact global solves) on ``count``
    size-stratified islands; returns (max relative UV error, islands,
    triangles). ``uvs`` holds the GPU UVs of the same islands. The soft-pin
    weight is the one of the whole batch (max |w| over every island,
    engine/gpu.py:138-140), as in the GPU run."""
    from oracle import arap as O
    offs = np.cumsum([0] + [len(p) for p, _ in islands])
    Pall = np.concatenate([np.asarray(p, np.float64) for p, _ in islands])
    Tall = np.concatenate([np.asarray(t, np.int64) + o for (_, t), o in zip(islands, offs[:-1])])
    wpin = max(float(np.abs(O.batch_frames(Pall, Tall)["w"]).max()), 1e-12)
    del Pall, Tall
    order = np.argsort([len(t) for _, t in islands])
    pick = order[np.linspace(0, len(order) - 1, min(count, len(order))).astype(int)]
    charts = []
    for i in pick:
        P, T = islands[i]
        P = np.asarray(P, np.float64)
        charts.append((P, T, O.lscm(P, T)))
    ref = O.BatchRef(charts, wpin=wpin)
    ref.arap(iters, line_search=True)
    Uref = np.concatenate(ref.chart_uvs())
    U = np.concatenate([uvs[i] for i in pick])
    off = np.cumsum([0] + [len(c[0]) for c in charts])
    return O.uv_rel_error(U, Uref, off), len(pick), int(sum(len(c[1]) for c in charts))


def time_boundary(islands, uvs, budget_tris):
    """Seconds of the oracle's boundary_intersections (max_report 1000, one
    thread) over a size-stratified sample of the charts at the given UVs;
    returns (seconds, sampled chart indices, their counts)."""
    from oracle import segments as OS
    pick = sample_indices(islands, budget_tris)
    t0 = time.perf_counter()
    want = [OS.boundary_intersections(uvs[i], islands[i][1], 1000) for i in pick]
    return time.perf_counter() - t0, [int(i) for i in pick], want


def time_hier_relax():
    """Seconds of the oracle's hier.Solver.relax (6 iterations, exact sparse
    LU) on the bench's mesh_charts workload (one thread)."""
    from oracle import hier as OH
    from ultimate_uv_artist_b200 import synth
    V, F, FF, faces, loc, chart, CV, nv, nchart, U0 = synth.mesh_charts()
    t0 = time.perf_counter()
    OH.relax(V, F, faces, CV, nv, chart, nchart, U0, iters=6)
    return time.perf_counter() - t0


def time_validation(V, F, UV, atlas=4096, padding=4, repeats=3):
    """Best-of-``repeats`` seconds of the oracle's validate_uvs on an atlas
    (numpy + scipy, and the C restatement of the reference's overlap scan on
    OpenMP threads over cells, as the reference's numba prange), and its
    report. The threads are OMP_NUM_THREADS, else every host core."""
    from oracle import validate as OV
    best, rep = None, None
    for _ in range(max(repeats, 1)):
        t0 = time.perf_counter()
        rep, _, _ = OV.validate_uvs(V, F, UV, atlas=atlas, padding=padding, count_pairs=False)
        dt = time.perf_counter() - t0
        best = dt if best is None else min(best, dt)
    return best, rep


def omp_threads():
    """Threads of the C oracle's parallel loops."""
    v = os.environ.get("OMP_NUM_THREADS", "")
    return int(v) if v.isdigit() and int(v) > 0 else (os.cpu_count() or 1)


def cpu_model():
    """The host CPU model name (lscpu's 'Model name')."""
    try:
        with open("/proc/cpuinfo") as fh:
            for line in fh:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"
