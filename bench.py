"""Benchmark of the batched LSCM + ARAP hot path (one JSON line on rank 0).

Workload (one step): 2,000 disk grid islands displaced by 8 Gaussian bumps,
square-grid triangle counts log-uniform in [20, 20,000] (about 4.3M triangles
after the disk cut), float32 positions, seed 2000 + rank. A step rebuilds the
device-side frames and Laplacian from the positions, runs batched LSCM
(hard far-pair pins) and 20 ARAP local/global iterations with the flip-safe
line search; every global step is solved per island to ||b - Lx|| <= 2e-7
||b|| per column (FP32 CG, FP64 residual refinement), checked in FP64: below
the metric's 1e-6, so that the UVs stay within 1e-5 of exact solves.

Metric: ARAP triangles x outer iterations per second (higher is better).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

With N > 1 (torchrun, one rank per GPU) every rank solves its own batch
(islands are independent: weak scaling, no collective on the data path);
the step time is the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "ARAP tris/sec @1e-6 resid, batched-FP32+FP64-refine"
UNIT = "tri-iters/s"
ITERS = 20
ISLANDS = 2000
TRAFFIC_ARAP = 32.78e9   # bytes per ARAP launch of the default workload (ncu dram__bytes_read + write)


def _args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--islands", type=int, default=ISLANDS)
    ap.add_argument("--iters", type=int, default=ITERS)
    ap.add_argument("--e2e-steps", type=int, default=4)
    ap.add_argument("--cpu-budget-tris", type=int, default=2_000_000)
    ap.add_argument("--cpu-repeats", type=int, default=3)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-validate", action="store_true")
    ap.add_argument("--no-plain", action="store_true")
    ap.add_argument("--plain-budget-tris", type=int, default=60_000)
    ap.add_argument("--no-graph", action="store_true")
    ap.add_argument("--no-tune", action="store_true")
    ap.add_argument("--no-config5", action="store_true")
    ap.add_argument("--no-config1", action="store_true")
    ap.add_argument("--no-config4", action="store_true")
    ap.add_argument("--no-pack", action="store_true")
    ap.add_argument("--no-giant", action="store_true")
    ap.add_argument("--pack-charts", type=int, default=3000)
    ap.add_argument("--pack-only", action="store_true",
                    help="only the packing leg, as one JSON line (for launch lists of the packer)")
    ap.add_argument("--hier-only", action="store_true",
                    help="only the hier.Solver leg, as one JSON line (for launch lists of its kernels)")
    ap.add_argument("--validate-only", action="store_true",
                    help="only the validation leg, as one JSON line (for launch lists of its kernels)")
    return ap.parse_args()


def _dist():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


class Clocks:
    """nvidia-smi sampling of SM clocks and throttle reasons during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = os.path.join(tempfile.gettempdir(), f"uva_bench_clocks_{os.getpid()}_{index}.csv")

    def start(self):
        try:
            os.makedirs(os.path.dirname(self.path), exist_ok=True)
            self.fh = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                                          "-lms", "50", "-i", str(self.index)], stdout=self.fh,
                                         stderr=subprocess.DEVNULL)
        except Exception:  # noqa: BLE001 - clocks are best effort
            self.proc = None
            return
        # the timed region starts only once the sampler is running (its start
        # takes a few hundred ms; a short region would otherwise get no sample)
        t_end = time.time() + 5.0
        while time.time() < t_end and os.path.getsize(self.path) == 0 and self.proc.poll() is None:
            time.sleep(0.02)
        self.fh.flush()
        with open(self.path) as fh:   # samples before this point are not the timed region's
            self.skip = sum(1 for _ in fh)

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:  # noqa: BLE001
            self.proc.kill()
        self.fh.close()
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        with open(self.path) as fh:
            for k, line in enumerate(fh):
                if k < getattr(self, "skip", 0):
                    continue
                parts = [p.strip() for p in line.split(",")]
                if len(parts) < 9:
                    continue
                try:
                    sm.append(float(parts[1])); mx.append(float(parts[2]))
                except ValueError:
                    continue
                for nm, val in zip(names, parts[5:9]):
                    if val.lower().startswith("active"):
                        reasons.add(nm)
        try:
            os.remove(self.path)
        except OSError:
            pass
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def _island_stats(batch):
    """Per island: vertices, triangles and nnz = n + 2E of the Laplacian."""
    p = batch.db.plan
    n = np.diff(p.vofs.astype(np.int64))
    t = np.diff(p.tofs.astype(np.int64))
    valid = (p.slot_edge >= 0).astype(np.int64)
    slot_isl = np.zeros(p.nslots, np.int64)
    slice_isl = np.repeat(np.arange(p.nc), np.diff(p.sofs.astype(np.int64)))
    widths = np.diff(p.slice_ptr.astype(np.int64))
    slot_isl = np.repeat(slice_isl, widths)
    off = np.bincount(slot_isl, weights=valid, minlength=p.nc).astype(np.int64)
    return n, t, n + off


def arap_bytes(n, t, nnz, st):
    """Algorithmic bytes of one ARAP launch (fp32 data, int32 indices):
    per outer iteration 48 t + 40 n (local step, RHS, line search), per CG
    iteration 8 nnz + 56 n, per FP64 residual 8 nnz + 52 n; K and R as
    executed. Also the compulsory bytes (K = R = 1 per outer iteration)."""
    it = st["outer_iters"].astype(np.float64)
    K = st["cg_iters"].astype(np.float64)
    R = st["refinements"].astype(np.float64)
    per_outer = 48.0 * t + 40.0 * n
    cg = 8.0 * nnz + 56.0 * n
    rf = 8.0 * nnz + 52.0 * n
    full = float((it * per_outer + K * cg + R * rf).sum())
    comp = float((it * (per_outer + cg + rf)).sum())
    return full, comp


def lscm_bytes(n, nnz, nbnd, st):
    """Algorithmic bytes of one LSCM launch: the PCG formula on the 2n
    unknowns (u, v) of each island, whose matrix holds the Laplacian twice
    plus the boundary coupling (nnz_H = 2 nnz + 4 boundary vertices): per CG
    iteration 8 nnz_H + 56 n, per FP64 residual 8 nnz_H + 52 n, with K and R
    as executed; the compulsory bytes count one of each."""
    K = st["cg_iters"].astype(np.float64)
    R = st["refinements"].astype(np.float64)
    nnz_h = 2.0 * nnz + 4.0 * nbnd
    cg = 8.0 * nnz_h + 56.0 * n
    rf = 8.0 * nnz_h + 52.0 * n
    return float((K * cg + R * rf).sum()), float((cg + rf).sum())


class PlainBatch:
    """The plain GPU solve the batched path is measured against: the
    reference's gpu.Batch algorithm (engine/gpu.py:66-249) restated with torch
    CUDA ops. Frames in FP64 on the host (gpu.py:88-121), the block-diagonal
    cotangent Laplacian with a soft pin on each chart's first vertex as a torch
    CSR matrix (gpu.py:126-142, cuSPARSE SpMV, one per UV column), Jacobi-PCG
    with the reference's stop test on the whole batch and a host sync per
    iteration (gpu.py:184-202), the atan2 rotation RHS (gpu.py:165-182) and
    the flip-safe line search (gpu.py:204-249); FP32 on the device. Used by
    the bench only, to time the plain method; ``cg_iters`` is raised so that
    every solve reaches the 1e-6 residual."""

    def __init__(self, charts, dev):
        import torch
        self.torch, self.dev = torch, dev
        f = torch.float32
        offs = np.cumsum([0] + [len(c[0]) for c in charts])
        P = np.concatenate([np.asarray(c[0], np.float64) for c in charts])
        T = np.concatenate([np.asarray(c[1], np.int64) + o for c, o in zip(charts, offs[:-1])])
        U = np.concatenate([np.asarray(c[2], np.float64) for c in charts])
        self.n, self.nc = len(P), len(charts)
        cv = np.repeat(np.arange(self.nc), np.diff(offs))
        ct = np.repeat(np.arange(self.nc), [len(c[1]) for c in charts])
        e1 = P[T[:, 1]] - P[T[:, 0]]
        e2 = P[T[:, 2]] - P[T[:, 0]]
        l1 = np.maximum(np.linalg.norm(e1, axis=1), 1e-30)
        nrm = np.cross(e1, e2)
        dbl = np.linalg.norm(nrm, axis=1)
        ex = e1 / l1[:, None]
        ey = np.cross(nrm / np.maximum(dbl, 1e-30)[:, None], ex)
        X = np.zeros((len(T), 3, 2))
        X[:, 1, 0] = l1
        X[:, 2, 0] = (e2 * ex).sum(1)
        X[:, 2, 1] = (e2 * ey).sum(1)
        ok = (dbl > 1e-14 * np.maximum(l1 * l1, 1e-300)) & np.isfinite(dbl)
        X[~ok] = 0.0
        w = np.zeros((len(T), 3))
        for k in range(3):
            a = X[:, (k + 1) % 3] - X[:, k]
            b = X[:, (k + 2) % 3] - X[:, k]
            cr = np.maximum(np.abs(a[:, 0] * b[:, 1] - a[:, 1] * b[:, 0]), 1e-30)
            w[:, k] = 0.5 * np.clip((a * b).sum(1) / cr, -1e4, 1e4)
        w[~ok] = 0.0
        t_ = lambda a, dt=f: torch.from_numpy(np.ascontiguousarray(a)).to(dev, dt)
        self.T = t_(T, torch.int64)
        self.U = t_(U)
        self.cv, self.ct = t_(cv, torch.int64), t_(ct, torch.int64)
        self.ok = t_(ok, torch.bool)
        self.X, self.w = t_(X), t_(w)
        self.x1 = t_(np.maximum(X[:, 1, 0], 1e-30))
        self.x2 = t_(X[:, 2, 0])
        self.y2 = t_(np.where(np.abs(X[:, 2, 1]) > 1e-30, X[:, 2, 1], 1e-30))
        # Laplacian
        a = torch.cat([self.T[:, 1], self.T[:, 2], self.T[:, 0]])
        b = torch.cat([self.T[:, 2], self.T[:, 0], self.T[:, 1]])
        key = torch.minimum(a, b) * self.n + torch.maximum(a, b)
        uk, inv = torch.unique(key, return_inverse=True)
        ea, eb = uk // self.n, uk % self.n
        W = torch.cat([self.w[:, 0], self.w[:, 1], self.w[:, 2]])
        wsum = torch.zeros(len(uk), device=dev, dtype=f).index_add_(0, inv, W)
        diag = torch.zeros(self.n, device=dev, dtype=f)
        diag.index_add_(0, ea, wsum)
        diag.index_add_(0, eb, wsum)
        self.pins = t_(offs[:-1], torch.int64)
        self.wpin = W.abs().max().clamp_min(1e-12)
        diag[self.pins] += self.wpin
        rows = torch.cat([ea, eb, torch.arange(self.n, device=dev)])
        cols = torch.cat([eb, ea, torch.arange(self.n, device=dev)])
        vals = torch.cat([-wsum, -wsum, diag])
        o = torch.argsort(rows * self.n + cols)
        crow = torch.zeros(self.n + 1, dtype=torch.int64, device=dev)
        crow[1:] = torch.cumsum(torch.bincount(rows, minlength=self.n), 0)
        self.L = torch.sparse_csr_tensor(crow.to(torch.int32), cols[o].to(torch.int32), vals[o], (self.n, self.n))
        self.dinv = 1.0 / diag.clamp_min(1e-30)
        self.cg_total = 0

    def _mv(self, x):
        return self.torch.stack([self.L @ x[:, k].contiguous() for k in range(x.shape[1])], 1)

    def _rhs(self, U):
        torch = self.torch
        T = self.T
        a0, a1, a2 = U[T[:, 0]], U[T[:, 1]], U[T[:, 2]]
        j00 = (a1[:, 0] - a0[:, 0]) / self.x1
        j10 = (a1[:, 1] - a0[:, 1]) / self.x1
        j01 = ((a2[:, 0] - a0[:, 0]) - j00 * self.x2) / self.y2
        j11 = ((a2[:, 1] - a0[:, 1]) - j10 * self.x2) / self.y2
        th = torch.atan2(j10 - j01, j00 + j11)
        th = torch.where(self.ok & torch.isfinite(th), th, torch.zeros_like(th))
        c, s = torch.cos(th), torch.sin(th)
        b = torch.zeros(self.n, 2, device=self.dev, dtype=U.dtype)
        for k in range(3):
            i, j = (k + 1) % 3, (k + 2) % 3
            dx = self.X[:, i] - self.X[:, j]
            r = torch.stack([c * dx[:, 0] - s * dx[:, 1], s * dx[:, 0] + c * dx[:, 1]], 1) * self.w[:, k:k + 1]
            b.index_add_(0, T[:, i], r)
            b.index_add_(0, T[:, j], -r)
        b[self.pins] += self.wpin * U[self.pins]
        return b

    def _cg(self, b, x, iters, tol):
        Minv = self.dinv[:, None]
        r = b - self._mv(x)
        z = r * Minv
        p = z.clone()
        rz = (r * z).sum(0)
        b2 = (b * b).sum(0).clamp_min(1e-30)
        for _ in range(iters):
            Ap = self._mv(p)
            alpha = rz / (p * Ap).sum(0).clamp_min(1e-30)
            x = x + p * alpha
            r = r - Ap * alpha
            self.cg_total += 1
            if bool(((r * r).sum(0) <= (tol * tol) * b2).all()):
                break
            z = r * Minv
            rz2 = (r * z).sum(0)
            p = z + p * (rz2 / rz.clamp_min(1e-30))
            rz = rz2
        return x

    def _max_step(self, U, D):
        torch = self.torch
        T = self.T
        u0, u1, u2 = U[T[:, 0]], U[T[:, 1]], U[T[:, 2]]
        d0, d1, d2 = D[T[:, 0]], D[T[:, 1]], D[T[:, 2]]
        ux1, uy1, ux2, uy2 = u1[:, 0] - u0[:, 0], u1[:, 1] - u0[:, 1], u2[:, 0] - u0[:, 0], u2[:, 1] - u0[:, 1]
        dx1, dy1, dx2, dy2 = d1[:, 0] - d0[:, 0], d1[:, 1] - d0[:, 1], d2[:, 0] - d0[:, 0], d2[:, 1] - d0[:, 1]
        C_ = ux1 * uy2 - ux2 * uy1
        B_ = ux1 * dy2 + dx1 * uy2 - ux2 * dy1 - dx2 * uy1
        A_ = dx1 * dy2 - dx2 * dy1
        big = torch.full_like(C_, 1e30)
        lin = torch.where((A_.abs() < 1e-30) & (B_ < 0), -C_ / B_.where(B_ != 0, torch.ones_like(B_)), big)
        disc = B_ * B_ - 4 * A_ * C_
        sq = disc.clamp_min(0).sqrt()
        A2 = torch.where(A_.abs() < 1e-30, torch.ones_like(A_), 2 * A_)
        r1, r2 = (-B_ - sq) / A2, (-B_ + sq) / A2
        quad = torch.minimum(torch.where(r1 > 0, r1, big), torch.where(r2 > 0, r2, big))
        quad = torch.where((disc >= 0) & (A_.abs() >= 1e-30), quad, big)
        t = torch.where(C_ > 0, torch.minimum(lin, quad), big)
        out = torch.full((self.nc,), 1e30, device=self.dev, dtype=U.dtype)
        return out.scatter_reduce_(0, self.ct, t, reduce="amin")

    def arap(self, iters, cg_iters=1_000_000, tol=1e-6):
        torch = self.torch
        U = self.U
        for _ in range(iters):
            Un = self._cg(self._rhs(U), U.clone(), cg_iters, tol)
            badv = ~torch.isfinite(Un).all(1)
            if bool(badv.any()):
                badc = torch.zeros(self.nc, dtype=torch.bool, device=self.dev)
                badc[self.cv[badv]] = True
                Un = torch.where(badc[self.cv][:, None], U, Un)
            D = Un - U
            step = torch.clamp(0.9 * self._max_step(U, D), max=1.0)
            U = U + D * step[self.cv][:, None]
        self.U = U
        return U


def _stratified(islands, budget_tris):
    """Every k-th island of the size-sorted list (keeps the size distribution),
    about ``budget_tris`` triangles in all."""
    order = np.argsort([len(t) for _, t in islands])
    total = sum(len(t) for _, t in islands)
    return order[::max(1, int(round(total / max(budget_tris, 1))))]


def bench_plain(islands, uvs, iters, dev, budget_tris):
    """Plain GPU solve (PlainBatch) of the same islands from the same LSCM
    start: one batch per island on a size-stratified sample (per-island 1e-6
    stop), and one batch of all islands (the reference's global stop, run to
    1e-6). Seconds count the ARAP iterations only, not the batch build."""
    import torch
    pick = _stratified(islands, budget_tris)
    PlainBatch([(islands[pick[0]][0], islands[pick[0]][1], uvs[pick[0]])], dev).arap(1)   # warm-up
    secs, cg = 0.0, 0
    for i in pick:
        pb = PlainBatch([(islands[i][0], islands[i][1], uvs[i])], dev)
        torch.cuda.synchronize()
        s0 = time.perf_counter()
        pb.arap(iters)
        torch.cuda.synchronize()
        secs += time.perf_counter() - s0
        cg += pb.cg_total
    sample_tris = int(sum(len(islands[i][1]) for i in pick))
    out = {"per_island": {"value": sample_tris * iters / secs, "unit": UNIT, "islands": len(pick),
                          "triangles": sample_tris, "seconds": secs, "cg_iters": cg,
                          "sample": "size-stratified island sample, one batch per island, 1e-6 stop per island"}}
    allb = PlainBatch([(p, t, u) for (p, t), u in zip(islands, uvs)], dev)
    torch.cuda.synchronize()
    s0 = time.perf_counter()
    allb.arap(iters)
    torch.cuda.synchronize()
    dt = time.perf_counter() - s0
    tris = int(sum(len(t) for _, t in islands))
    out["one_batch"] = {"value": tris * iters / dt, "unit": UNIT, "seconds": dt, "cg_iters": allb.cg_total,
                        "stop": "global ||r|| <= 1e-6 ||b|| per column over the whole batch"}
    return out


def bench_validation(dev, steps=3):
    """Exact validation of the 1M-triangle, 5,000-island atlas (4096, padding
    4, injected faults): device time per pass and candidate pairs per second
    (unordered non-skipped pairs with intersecting FP64 boxes, counted by the
    kernel; the oracle counts the same set)."""
    import torch
    from ultimate_uv_artist_b200 import synth
    from ultimate_uv_artist_b200.engine import metrics
    from ultimate_uv_artist_b200.engine import validate as GV
    V, F, UV, _ = synth.validation_atlas(seed=3000)
    dv = GV.DeviceValidation(V.astype(np.float64), F.astype(np.int32), UV.astype(np.float32), device=dev)
    UV64 = dv.UV.double()
    for _ in range(2):
        dv.run()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True); e1 = torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(steps):
        dv.run()
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / steps
    c = dv.host_counts()
    metrics.min_gutter_device(UV64, dv.F, dv.labels, int(c[6]), 4096)   # warm-up (first-call allocations)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    e2 = torch.cuda.Event(enable_timing=True); e3 = torch.cuda.Event(enable_timing=True)
    e2.record()
    g = metrics.min_gutter_device(UV64, dv.F, dv.labels, int(c[6]), 4096)
    e3.record()
    torch.cuda.synchronize()
    g_ms = (time.perf_counter() - t0) * 1e3
    pairs = int(c[10])
    res = 4096
    return {"workload": "validation_atlas_1M_5000_islands_4096", "triangles": int(len(F)), "uv_vertices": int(len(UV)),
            "pairs_aabb": pairs, "ms_per_pass": ms, "pairs_per_s": pairs / (ms / 1e3), "gutter_ms_wall": g_ms,
            "gutter_span_ms": e2.elapsed_time(e3),
            # the validation byte model: 8 n (UV) + 20 m (faces, per-triangle outputs) per pass;
            # 20 res^2 (label raster, two distance passes) for the gutter
            "bytes_pass": 8 * int(len(UV)) + 20 * int(len(F)), "bytes_gutter": 20 * res * res,
            "overlapping_triangles": int(c[7]), "flipped": int(c[4]), "mirrored": int(c[5]),
            "min_gutter_texels": float(g)}


def bench_boundary(b, reps=5):
    """Boundary self-intersection counts (charts.boundary_intersections,
    max_report 1000) of every chart of the batch at its current UVs, on the
    device (uva_boundary_hits; the boundary half-edges are found once per
    batch and kept)."""
    import torch
    from ultimate_uv_artist_b200 import _lib
    db = b.db
    seg, _, sofs = db.boundary_segments()
    hits = db.boundary_hits(_lib.SEG_COUNT, 1000)
    torch.cuda.synchronize()
    stream = torch.cuda.current_stream(db.dev)
    out = {}
    for name, mode in (("count", _lib.SEG_COUNT), ("any", _lib.SEG_ANY)):
        e0 = torch.cuda.Event(enable_timing=True); e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(reps):
            db.boundary_hits(mode, 1000)
        e1.record(stream)
        torch.cuda.synchronize()
        out[f"{name}_ms"] = e0.elapsed_time(e1) / reps
    m = np.diff(sofs)
    pairs = int((m * (m - 1) // 2).sum())
    h = hits.cpu().numpy()
    out.update({"charts": int(len(m)), "segments": int(m.sum()), "pairs": pairs,
                "pairs_per_s": pairs / (out["count_ms"] / 1e3), "charts_with_crossings": int((h > 0).sum()),
                "hits": h})
    return out


def bench_hier(dev, reps=3):
    """hier.Solver.relax (6 iterations), Solver.lscm and hier.chart_checks on a
    256 x 256 bumpy grid mesh (131,072 faces) cut into 64 charts
    (synth.mesh_charts): wall time of the API calls (host layout, device
    work, download), best of ``reps`` after a warm-up call."""
    import time
    from types import SimpleNamespace
    import torch
    from ultimate_uv_artist_b200 import synth
    from ultimate_uv_artist_b200.engine import hier
    V, F, FF, faces, loc, chart, CV, nv, nchart, U0 = synth.mesh_charts()
    S = hier.Solver(SimpleNamespace(V=V, F=F), dev=dev)
    ba, bb = hier.boundary_directed(F, FF, faces, loc, chart, CV)

    def best(fn):
        fn()
        torch.cuda.synchronize()
        ts = []
        for _ in range(reps):
            t0 = time.perf_counter()
            out = fn()
            torch.cuda.synchronize()
            ts.append(time.perf_counter() - t0)
        return min(ts), out

    t_relax, (U, flips, _) = best(lambda: S.relax(faces, CV, nv, chart, nchart, U0, iters=6))
    t_lscm, _ = best(lambda: S.lscm(faces, CV, nv, chart, nchart, U0, ba, bb))
    t_chk, (col, _, _) = best(lambda: hier.chart_checks(F, FF, faces, loc, chart, CV, U, nchart, nv))
    return {"workload": "mesh_charts_256x256_64_charts", "faces": int(len(F)), "charts": int(nchart),
            "uv_vertices": int(nv), "relax_iters": 6, "relax_ms": 1e3 * t_relax,
            "relax_face_iters_per_s": len(F) * 6 / t_relax, "lscm_ms": 1e3 * t_lscm,
            "chart_checks_ms": 1e3 * t_chk, "flipped_after_relax": int(flips.sum()),
            "charts_colliding": int(col.sum())}


def bench_overlap(islands, uvs, count=16):
    """overlapfix.overlapping_triangles and collision, chart by chart (the
    reference's per-chart API), on the ``count`` largest charts of the batch
    at their final UVs: wall time per chart."""
    import time
    import torch
    from ultimate_uv_artist_b200.engine import overlapfix
    pick = np.argsort([-len(t) for _, t in islands])[:count]
    for i in pick[:2]:   # warm-up
        overlapfix.overlapping_triangles(uvs[i], islands[i][1])
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    bad = sum(int(overlapfix.overlapping_triangles(uvs[i], islands[i][1]).sum()) for i in pick)
    t1 = time.perf_counter()
    coll = sum(overlapfix.collision(uvs[i], islands[i][1]) is not None for i in pick)
    t2 = time.perf_counter()
    tris = int(sum(len(islands[i][1]) for i in pick))
    return {"charts": int(len(pick)), "triangles": tris, "overlapping_triangles_ms_per_chart": 1e3 * (t1 - t0) / len(pick),
            "collision_ms_per_chart": 1e3 * (t2 - t1) / len(pick), "overlapping": bad, "colliding_charts": int(coll)}


def _events(dev):
    import torch
    return torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)


def bench_config5(dev, iters=ITERS, steps=2, cpu=True):
    """Config 5 end to end at its stated size: a 5M-triangle noisy sphere cut
    into 3,000 k-means charts (disk components kept), batched LSCM + ARAP,
    per-chart p95 metrics, packing and exact validation of the packed atlas.
    Device times by CUDA events (solve, metrics, validation), the public-API
    wall time of every stage, validation pairs per second; packing by
    engine.pack with the reference's default schedule (wall time, attempts)
    and one full-grid attempt beside the oracle's on one host core."""
    import torch
    from ultimate_uv_artist_b200 import _lib, synth
    from ultimate_uv_artist_b200.device import DeviceBatch
    from ultimate_uv_artist_b200.engine import gpu, metrics
    from ultimate_uv_artist_b200.engine import param as Pm
    from ultimate_uv_artist_b200.engine import validate as GV
    g0 = time.perf_counter()
    V, F = synth.noisy_sphere(seed=5000, tris=5_000_000)
    charts = synth.disk_charts(V, F, synth.kmeans_charts(V, F, k=3000, seed=5001, device=dev), min_tris=20)
    gen_s = time.perf_counter() - g0
    items = [(p, t, None) for p, t in charts]
    tris = int(sum(len(t) for _, t in charts))
    stream = torch.cuda.current_stream(dev)
    # public API, wall: batch build (host plan + uploads), LSCM + ARAP, download
    w0 = time.perf_counter()
    b = gpu.Batch(items, dev=dev)
    torch.cuda.synchronize(); w1 = time.perf_counter()
    b.db.lscm(); b.db.arap(iters=iters, line_search=True)
    U = b.chart_uvs()
    torch.cuda.synchronize(); w2 = time.perf_counter()
    # device: setup + LSCM + ARAP, inputs resident
    db = b.db
    ev = []
    for _ in range(steps):
        a, c, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True), \
            torch.cuda.Event(enable_timing=True)
        a.record(stream)
        db.setup(); db.lscm()
        c.record(stream)
        db.arap(iters=iters, line_search=True)
        e.record(stream)
        ev.append((a, c, e))
    torch.cuda.synchronize()
    lscm_ms = float(np.mean([a.elapsed_time(c) for a, c, _ in ev]))
    arap_ms = float(np.mean([c.elapsed_time(e) for _, c, e in ev]))
    st = db.island_status()
    # per-chart p95 metrics (param.chart_quality) on a PARAM batch over the same plan
    w3 = time.perf_counter()
    dq = DeviceBatch(db.P, None, b.offsets, b._tofs, U=np.concatenate(U), semantics=_lib.SEM_PARAM, device=dev,
                     plan=db.plan)
    q = Pm.chart_quality_batch(dq)
    torch.cuda.synchronize(); w4 = time.perf_counter()
    p95 = np.array([x["aniso_p95"] for x in q])
    del dq, b, db
    torch.cuda.empty_cache()
    # packing (engine.pack: the reference's schedule, attempts on the device)
    from ultimate_uv_artist_b200.engine import pack as EPK
    uv_charts = [(U[i].astype(np.float64), charts[i][1]) for i in range(len(charts))]
    torch.cuda.synchronize(); w5 = time.perf_counter()
    packed, pinfo = EPK.pack(uv_charts, atlas=4096, padding=4)
    torch.cuda.synchronize(); pack_s = time.perf_counter() - w5
    # one full-grid attempt at 0.97 of the found scale: device (CUDA events) and the oracle (one core)
    Us = [EPK.orient(u) for u, _ in uv_charts]
    Ts = [t for _, t in uv_charts]
    P = EPK.Packer(Us, Ts, np.ones(len(Us)))
    s_att = 0.97 * pinfo["texel_scale_grid"]
    P.attempt(2048, 2, [0, 1, 2, 3], s_att, "area")
    a0, a1 = _events(dev)
    a0.record(stream)
    att = P.attempt(2048, 2, [0, 1, 2, 3], s_att, "area")
    a1.record(stream)
    torch.cuda.synchronize()
    attempt_ms = a0.elapsed_time(a1)
    pack_cpu = None
    if cpu:
        from oracle import pack as OPK
        t0 = time.perf_counter()
        ref_att = OPK.attempt(Us, Ts, np.ones(len(Us)), 2048, 2, [0, 1, 2, 3], s_att, "area")
        pack_cpu = {"attempt_s": time.perf_counter() - t0, "cores": 1, "kind": "port",
                    "same_placement": bool(att is not None and ref_att is not None
                                           and att.placement == ref_att[1][0])}
    offs = np.cumsum([0] + [len(p) for p, _ in charts])
    Vall = np.concatenate([p for p, _ in charts]).astype(np.float32)
    Fall = np.concatenate([t + o for (_, t), o in zip(charts, offs[:-1])])
    UVall = np.concatenate(packed).astype(np.float32)
    w6 = time.perf_counter()
    rep, _ = GV.validate_uvs(Vall, Fall, UVall, atlas=4096, padding=4)
    val_api_s = time.perf_counter() - w6
    dv = GV.DeviceValidation(Vall.astype(np.float64), Fall.astype(np.int32), UVall, device=dev)
    dv.run(); dv.run()
    e0, e1 = _events(dev)
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(3):
        dv.run()
    e1.record(stream)
    torch.cuda.synchronize()
    val_ms = e0.elapsed_time(e1) / 3
    c = dv.host_counts()
    t0 = time.perf_counter()
    g = metrics.min_gutter_device(dv.UV.double(), dv.F, dv.labels, int(c[6]), 4096)
    torch.cuda.synchronize()
    gutter_ms = (time.perf_counter() - t0) * 1e3
    pairs = int(c[10])
    return {"workload": "noisy_sphere_5M_kmeans3000_disk_charts", "mesh_triangles": int(len(F)),
            "charts": len(charts), "triangles": tris, "vertices": int(offs[-1]), "generate_s": gen_s,
            "lscm_setup_ms": lscm_ms, "arap_ms": arap_ms, "arap_iters": iters,
            "tri_iters_per_s": tris * iters / ((lscm_ms + arap_ms) / 1e3),
            "max_resid": float(st["resid"].max()),
            "api_batch_build_s": w1 - w0, "api_solve_download_s": w2 - w1, "api_chart_quality_s": w4 - w3,
            "aniso_p95_median": float(np.median(p95)), "aniso_p95_max": float(p95.max()),
            "pack": {"api_s": pack_s, "attempts": pinfo["attempts"], "attempt_s_total": pinfo["attempt_seconds"],
                     "texel_scale_grid": pinfo["texel_scale_grid"], "plan_occupancy": pinfo["plan_occupancy"],
                     "grid": pinfo["grid"], "attempt_ms_2048": attempt_ms, "cpu_oracle": pack_cpu},
            "validate_api_s": val_api_s,
            "validate_ms_per_pass": val_ms, "pairs_aabb": pairs, "pairs_per_s": pairs / (val_ms / 1e3),
            "gutter_ms_wall": gutter_ms, "min_gutter_texels": float(g), "valid": bool(rep["valid"]),
            "overlapping_triangles": int(rep["overlapping_triangles_exact"]),
            "flipped": int(rep["flipped_triangles"]), "islands": int(rep["islands"])}


def bench_giant(dev, iters=ITERS, big_tris=200_000):
    """Islands up to 200k triangles: the 2,000-island batch plus one disk
    island of about 200k triangles (solved by the whole-GPU class-W team
    before the persistent launch). Setup + LSCM and 20 ARAP iterations
    (CUDA events), the batch's tri-iters/s, and the large island's own
    launch time, CG iterations and team."""
    import torch
    from ultimate_uv_artist_b200 import synth
    from ultimate_uv_artist_b200.engine import gpu
    isl = list(synth.uneven_islands(seed=2000, count=2000))
    isl.append(synth.disk_patch(np.random.default_rng(5), big_tris))
    b = gpu.Batch([(p, t, None) for p, t in isl], dev=dev)
    db = b.db
    stream = torch.cuda.current_stream(dev)
    e0, e1, e2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
    for _ in range(2):
        e0.record(stream); db.setup(); db.lscm(); e1.record(stream)
        db.arap(iters=iters, line_search=True); e2.record(stream)
        torch.cuda.synchronize()
    st = db.island_status()
    tris = int(sum(len(t) for _, t in isl))
    last = len(isl) - 1
    lscm_ms, arap_ms = e0.elapsed_time(e1), e1.elapsed_time(e2)
    return {"workload": f"uneven_islands_2000_plus_one_{len(isl[-1][1])}_tri_island", "triangles": tris,
            "large_island_vertices": int(len(isl[-1][0])), "lscm_setup_ms": lscm_ms, "arap_ms": arap_ms,
            "tri_iters_per_s": tris * iters / ((lscm_ms + arap_ms) / 1e3),
            "large_island_arap_ms": float((st["t_end"][last] - st["t_begin"][last]) / 1e6),
            "large_island_cg_iters": int(st["cg_iters"][last]), "large_island_team": int(st["team"][last]),
            "max_resid": float(st["resid"].max())}


def bench_pack(dev, nch=3000, cpu=True):
    """engine.pack on synthetic disk charts (log-uniform 100 to 6,000
    triangles, stretched up to 6.7x, random in-plane turns) with the
    reference's default schedule (atlas 4096, padding 4, grid 2048, four
    turns, three orderings, no time budget): wall time, attempts, and the
    device time of one full-grid attempt and of one four-probe round (CUDA
    events) beside the oracle's serial first fit of the same attempt on one
    host core."""
    import torch
    from ultimate_uv_artist_b200 import synth
    from ultimate_uv_artist_b200.engine import pack as EPK
    rng = np.random.default_rng(3)
    charts = []
    for _ in range(nch):
        P, T = synth.disk_patch(rng, int(np.exp(rng.uniform(np.log(100), np.log(6000)))))
        charts.append((P[:, :2].astype(np.float64) * rng.uniform(0.3, 2.0, 2), np.asarray(T, np.int64)))
    stream = torch.cuda.current_stream(dev)
    torch.cuda.synchronize(); w0 = time.perf_counter()
    uvs, info = EPK.pack(charts, atlas=4096, padding=4)
    torch.cuda.synchronize(); pack_s = time.perf_counter() - w0
    Us = [EPK.orient(u) for u, _ in charts]
    Ts = [t for _, t in charts]
    P = EPK.Packer(Us, Ts, np.ones(nch))
    s_att = 0.97 * info["texel_scale_grid"]
    P.attempt(2048, 2, [0, 1, 2, 3], s_att, "area")
    a0, a1 = _events(dev)
    a0.record(stream)
    att = P.attempt(2048, 2, [0, 1, 2, 3], s_att, "area")
    a1.record(stream)
    torch.cuda.synchronize()
    attempt_ms = a0.elapsed_time(a1)
    s_half = s_att * 1024 / 2048
    probes = [s_half * f for f in (0.88, 0.92, 0.96, 1.0)]
    P.attempts_at(1024, 1, [0, 1, 2, 3], probes, "area")
    a0.record(stream)
    P.attempts_at(1024, 1, [0, 1, 2, 3], probes, "area")
    a1.record(stream)
    torch.cuda.synchronize()
    round_ms = a0.elapsed_time(a1)
    out = {"workload": f"disk_charts_{nch}", "charts": nch, "triangles": int(sum(len(t) for t in Ts)),
           "api_s": pack_s, "attempts": info["attempts"], "attempt_s_total": info["attempt_seconds"],
           "texel_scale_grid": info["texel_scale_grid"], "plan_occupancy": info["plan_occupancy"],
           "attempt_ms_2048": attempt_ms, "us_per_chart_2048": attempt_ms * 1e3 / nch,
           "probe_round_ms_1024": round_ms}
    if cpu:
        from oracle import pack as OPK
        t0 = time.perf_counter()
        ref_att = OPK.attempt(Us, Ts, np.ones(nch), 2048, 2, [0, 1, 2, 3], s_att, "area")
        cs = time.perf_counter() - t0
        out["cpu_oracle"] = {"attempt_s": cs, "cores": 1, "kind": "port", "speedup_attempt": cs / (attempt_ms / 1e3),
                             "same_placement": bool(att is not None and ref_att is not None
                                                    and att.placement == ref_att[1][0])}
    return out


def bench_energy(dev, hbm, reps=5):
    """Config 4: the ARAP / symmetric-Dirichlet forward and backward kernels
    on 512 islands of 500 to 50,000 triangles (5.8M, 5 % near-degenerate),
    and 50 steps of p95-stretch refinement. Roofline per launch with FP64
    UVs and positions: forward reads T (12 t) and P, U (24 n + 16 n);
    backward reads the same and writes dU, dP (16 n + 24 n)."""
    import torch
    from ultimate_uv_artist_b200 import _lib, synth
    from ultimate_uv_artist_b200.device import DeviceBatch, concat_charts
    from ultimate_uv_artist_b200.energy import DistortionEnergy, sd_refine
    from ultimate_uv_artist_b200.engine import param as Pm
    isl = synth.energy_islands(seed=4000, count=512, tmin=500, tmax=50000)
    P, T, _, vofs, tofs = concat_charts([(p, t) for p, t in isl], with_uv=False)
    db = DeviceBatch(P, T, vofs, tofs, U=P[:, :2].copy(), semantics=_lib.SEM_PARAM, device=dev)
    stream = torch.cuda.current_stream(dev)
    U = db.U[:db.n].clone().requires_grad_(True)
    Pt = db.P[:db.n].clone().requires_grad_(True)
    out = {"workload": "energy_islands_512_500_50000", "islands": db.nc, "triangles": db.t, "vertices": db.n}
    for kind, name in ((0, "arap"), (1, "symmetric_dirichlet")):
        for _ in range(2):
            e = DistortionEnergy.apply(U, Pt, db, kind)
            torch.autograd.grad(e.sum(), (U, Pt))
        fw, bw = [], []
        for _ in range(reps):
            a, b_, c = (torch.cuda.Event(enable_timing=True) for _ in range(3))
            a.record(stream)
            e = DistortionEnergy.apply(U, Pt, db, kind)
            b_.record(stream)
            torch.autograd.grad(e.sum(), (U, Pt))
            c.record(stream)
            torch.cuda.synchronize()
            fw.append(a.elapsed_time(b_)); bw.append(b_.elapsed_time(c))
        fwd_b = 12.0 * db.t + 40.0 * db.n
        bwd_b = 12.0 * db.t + 80.0 * db.n
        f_ms, b_ms = min(fw), min(bw)
        out[name] = {"fwd_ms": f_ms, "bwd_ms": b_ms, "fwd_bytes": fwd_b, "bwd_bytes": bwd_b,
                     "fwd_gbs": fwd_b / (f_ms / 1e3) / 1e9, "bwd_gbs": bwd_b / (b_ms / 1e3) / 1e9,
                     "fwd_frac": fwd_b / (f_ms / 1e3) / 1e9 / hbm, "bwd_frac": bwd_b / (b_ms / 1e3) / 1e9 / hbm}
    q0 = np.array([q["aniso_p95"] for q in Pm.chart_quality_batch(db)])
    a, c = _events(dev)
    torch.cuda.synchronize()
    a.record(stream)
    sd_refine(db, steps=50)
    c.record(stream)
    torch.cuda.synchronize()
    q1 = np.array([q["aniso_p95"] for q in Pm.chart_quality_batch(db)])
    out["sd_refine_50_ms"] = a.elapsed_time(c)
    out["aniso_p95_median_start"] = float(np.median(q0))
    out["aniso_p95_median_after"] = float(np.median(q1))
    return out


def bench_config1(dev, reps=5):
    """Config 1 per call through the drop-in API: param.lscm, then
    param.refine(iters=10) on the 4,802-triangle hemisphere patch (wall time
    of each call, host arrays in and out), beside the oracle's restatement of
    the reference's per-chart CPU calls (one thread, exact LU)."""
    import torch
    from oracle import arap as O
    from ultimate_uv_artist_b200 import synth
    from ultimate_uv_artist_b200.engine import param as Pm
    V, F = synth.hemisphere_patch(seed=1000, n=50, jitter=0.01)
    P = V.astype(np.float64)

    def best(fn):
        out, ts = None, []
        for _ in range(reps):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            out = fn()
            ts.append(time.perf_counter() - t0)
        return out, min(ts)

    Pm.lscm(P, F); Pm.refine(P, F, Pm.lscm(P, F), iters=10, tol=0.0)      # warm
    U0, lscm_s = best(lambda: Pm.lscm(P, F))
    U1, ref_s = best(lambda: Pm.refine(P, F, U0, iters=10, tol=0.0)[0])
    R0, o_lscm = best(lambda: O.lscm(P, F))
    R1, o_ref = best(lambda: O.refine_arap(P, F, R0, iters=10, line_search=True, tol=0.0))
    ext = float(np.ptp(R1, 0).max())
    return {"workload": "hemisphere_50x50_4802_tris", "triangles": int(len(F)),
            "lscm_ms": lscm_s * 1e3, "refine10_ms": ref_s * 1e3,
            "oracle_cpu_lscm_ms": o_lscm * 1e3, "oracle_cpu_refine10_ms": o_ref * 1e3,
            "speedup_per_call": (o_lscm + o_ref) / (lscm_s + ref_s),
            "max_rel_uv_error": float(np.abs(U1 - R1).max() / ext)}


def run_reference(args):
    """CPU reference arm: the oracle port of param.lscm + param.refine per
    island over all host cores, on a bounded sample of the same workload."""
    from oracle import cpu_baseline
    from ultimate_uv_artist_b200 import synth
    islands = synth.uneven_islands(seed=2000, count=args.islands)
    sample = cpu_baseline.sample_islands(islands, args.cpu_budget_tris)
    vals = []
    for _ in range(max(args.warmup, 0)):
        cpu_baseline.time_cpu(sample[:8], args.iters)
        break
    for _ in range(args.steps):
        v, dt, workers, tris = cpu_baseline.time_cpu(sample, args.iters)
        vals.append(v)
    value = float(np.median(vals))
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": 0, "steps": args.steps,
            "warmup": args.warmup, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic",
            "config": {"workload": "uneven_islands_2000_lscm_arap20", "islands": len(sample),
                       "triangles": int(tris), "iters": args.iters, "sample": "size-stratified island sample"},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": workers, "kind": "port",
                             "sample": f"{len(sample)} of {len(islands)} islands, {tris} triangles"},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    args = _args()
    ws, rank, local = _dist()
    if args.impl == "reference":
        if rank == 0:
            run_reference(args)
        return
    import torch
    import torch.distributed as dist
    if ws > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if args.validate_only:
        if rank == 0:
            print(json.dumps({"validate": bench_validation(dev)}))
        if ws > 1:
            dist.destroy_process_group()
        return
    if args.hier_only:
        if rank == 0:
            print(json.dumps({"hier_solver": bench_hier(dev)}))
        if ws > 1:
            dist.destroy_process_group()
        return
    if args.pack_only:
        if rank == 0:
            print(json.dumps({"pack": bench_pack(dev, args.pack_charts, cpu=not args.no_cpu_baseline)}))
        if ws > 1:
            dist.destroy_process_group()
        return
    from ultimate_uv_artist_b200 import synth
    from ultimate_uv_artist_b200.engine import gpu

    islands = synth.uneven_islands(seed=2000 + rank, count=args.islands)
    charts = [(p, t, None) for p, t in islands]
    b = gpu.Batch(charts, dev=dev)
    db = b.db
    tris = int(sum(len(t) for _, t in islands))
    stream = torch.cuda.current_stream(dev)

    ev = []
    tuned = None
    if not args.no_tune:   # schedule autotuner (warm-up; the timed steps use its choice)
        from ultimate_uv_artist_b200 import autotune
        db.setup(); db.lscm()
        tuned, _ = autotune.tune(db)
    graphs = None
    if not args.no_graph:
        # the warm-up pass sets the kernels' attributes; then setup + LSCM and
        # the ARAP iterations are captured as two graphs (events between them
        # time the ARAP launch alone)
        db.setup(); db.lscm(); db.arap(iters=1)
        torch.cuda.synchronize()
        graphs = (db.step_graph(setup=True, lscm=False, arap_iters=0),
                  db.step_graph(setup=False, lscm=True, arap_iters=0),
                  db.step_graph(setup=False, lscm=False, arap_iters=args.iters, line_search=True))

    def step(record):
        if record:
            e = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
        if graphs:
            graphs[0].launch()
        else:
            db.setup()
        if record:
            e[0].record(stream)
        if graphs:
            graphs[1].launch()
        else:
            db.lscm()
        if record:
            e[1].record(stream)
        if graphs:
            graphs[2].launch()
        else:
            db.arap(iters=args.iters, line_search=True)
        if record:
            e[2].record(stream)
            ev.append(e)

    for _ in range(args.warmup):
        step(False)
    torch.cuda.synchronize()
    if ws > 1:
        dist.barrier()
    clocks = Clocks(local)
    clocks.start()
    t0 = torch.cuda.Event(enable_timing=True); t1 = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    t0.record(stream)
    for _ in range(args.steps):
        step(True)
    t1.record(stream)
    torch.cuda.synchronize()
    ck = clocks.stop()
    if ws > 1:
        dist.barrier()
    ms = t0.elapsed_time(t1) / args.steps
    arap_ms = float(np.mean([e[1].elapsed_time(e[2]) for e in ev]))
    lscm_ms = float(np.mean([e[0].elapsed_time(e[1]) for e in ev]))
    st = db.island_status()
    our_uvs = b.chart_uvs()
    db.setup(); db.lscm()                 # the LSCM solve's own counters
    st_lscm = db.island_status()
    n, t, nnz = _island_stats(b)
    full, comp = arap_bytes(n, t, nnz, st)
    units = float(tris * args.iters)
    if ws > 1:
        from ultimate_uv_artist_b200 import shard
        ms_max, units_all = shard.reduce_step(ms, units, device=dev)
    else:
        ms_max, units_all = ms, units
    value = units_all / (ms_max / 1e3)

    # ---- end to end through the public API: host charts in, host UVs out
    e2e_val = None
    h2d = d2h = 0
    if args.e2e_steps > 0:
        def e2e_step():
            bb = gpu.Batch(charts, dev=dev)
            bb.db.lscm()
            bb.db.arap(iters=args.iters, line_search=True)
            return bb, bb.chart_uvs()

        for _ in range(2):   # untimed warm-up, same pattern as the timed loop (the previous
            bb, Us = e2e_step()   # batch is alive while the next is built): page-locked host caches
        torch.cuda.synchronize()
        w0 = time.perf_counter()
        for _ in range(args.e2e_steps):
            bb, Us = e2e_step()
        torch.cuda.synchronize()
        e2e_s = (time.perf_counter() - w0) / args.e2e_steps
        e2e_val = units / e2e_s
        dbb = bb.db
        h2d = int(dbb.h2d_bytes)   # every host -> device copy of the batch constructor
        d2h = int(sum(u.nbytes for u in Us))
        del bb
        if ws > 1:
            x = torch.tensor([e2e_s], dtype=torch.float64, device=dev)
            dist.all_reduce(x, op=dist.ReduceOp.MAX)
            e2e_val = units_all / float(x[0])

    # our kernels per step: setup (k_frames, k_wpin, k_vert_isl, k_rows,
    # k_far_pair, then k_coarse for the whole-CTA classes and for the rest),
    # then k_islands for LSCM and for ARAP, each with k_wide before it when
    # the batch has islands of the whole-GPU class
    co = [int(db.desc.class_ofs[c]) for c in range(5)]
    big = min(max(co[2], 0), db.nc)
    n_coarse = int(big > 0) + int(db.nc - big > 0)
    n_wide = 2 if co[1] > co[0] else 0
    launches_per_step = 5 + n_coarse + 2 + n_wide
    peaks = {}
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fh:
            peaks = json.load(fh)
        hbm = float(peaks["hbm_gbs"]); peak_src = "measured"
    except Exception:  # noqa: BLE001
        hbm = 6650.0; peak_src = "fallback"
    achieved = full / (arap_ms / 1e3) / 1e9
    achieved_c = comp / (arap_ms / 1e3) / 1e9
    nbnd = np.diff(db.plan.bofs.astype(np.int64))
    lfull, lcomp = lscm_bytes(n, nnz, nbnd, st_lscm)

    # the single-GPU legs (diagnostics beside the headline step) run only
    # without torchrun: a scaling run holds every GPU while rank 0 works
    solo = rank == 0 and ws == 1
    val = None
    if solo and not args.no_validate:
        val = bench_validation(dev)
        gbs = val["bytes_pass"] / (val["ms_per_pass"] / 1e3) / 1e9
        val["roofline"] = {"kernel": "uva_validate (one pass)", "bound": "compute",
                           "note": "the exact pair predicates bound the pass; its modelled bytes are a small "
                                   "fraction of HBM", "achieved": gbs, "peak": hbm, "unit": "GB/s",
                           "frac": gbs / hbm, "peak_source": peak_src, "algorithmic_bytes": val["bytes_pass"]}
        ggs = val["bytes_gutter"] / (val["gutter_span_ms"] / 1e3) / 1e9
        val["roofline_gutter"] = {"kernel": "min_gutter_device (raster + distance passes)", "bound": "hbm",
                                  "note": "device span of the call, its host readbacks included",
                                  "achieved": ggs, "peak": hbm, "unit": "GB/s", "frac": ggs / hbm,
                                  "peak_source": peak_src, "algorithmic_bytes": val["bytes_gutter"]}

    plain = None
    if rank == 0 and ws == 1 and not args.no_plain:
        db.setup(); db.lscm()            # the common LSCM start
        lscm_uvs = b.chart_uvs()
        plain = bench_plain(islands, lscm_uvs, args.iters, dev, args.plain_budget_tris)
        plain["speedup_vs_per_island"] = value / plain["per_island"]["value"]
        plain["speedup_vs_one_batch"] = value / plain["one_batch"]["value"]

    bnd = hier_b = ovl = None
    if solo and not args.no_validate:
        bnd = bench_boundary(b)
        hier_b = bench_hier(dev)
        ovl = bench_overlap(islands, our_uvs)
    c5 = c1 = c4 = pk = gi = None
    if solo and not args.no_giant:
        gi = bench_giant(dev, args.iters)
    if solo and not args.no_pack:
        pk = bench_pack(dev, args.pack_charts, cpu=not args.no_cpu_baseline)
    if solo and not args.no_config5:
        c5 = bench_config5(dev, cpu=not args.no_cpu_baseline)
    if solo and not args.no_config4:
        c4 = bench_energy(dev, hbm)
    if solo and not args.no_config1:
        c1 = bench_config1(dev)

    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        from oracle import cpu_baseline
        sample = cpu_baseline.sample_islands(islands, args.cpu_budget_tris)
        v, dt, workers, stris = cpu_baseline.time_cpu(sample, args.iters, repeats=args.cpu_repeats)
        small = cpu_baseline.sample_islands(islands, args.cpu_budget_tris // 16)
        v1, dt1, _, stris1 = cpu_baseline.time_cpu(small, args.iters, workers=1)
        cpu = {"value": v, "unit": UNIT, "cores": workers, "kind": "port", "cpu_model": cpu_baseline.cpu_model(),
               "sample": f"{len(sample)} size-stratified islands of {len(islands)} ({stris} triangles), "
                         f"LSCM + {args.iters} ARAP iterations per island (param.lscm + param.refine, "
                         f"exact LU), best of {args.cpu_repeats}: {dt:.1f} s",
               "one_thread": {"value": v1, "unit": UNIT, "seconds": dt1, "triangles": stris1,
                              "sample": f"{len(small)} size-stratified islands"}}
        if val is not None:   # the validation workload's CPU time (oracle port; overlap scan on all cores)
            from ultimate_uv_artist_b200 import synth as _synth
            Vv, Fv, UVv, _ = _synth.validation_atlas(seed=3000)
            vs, vrep = cpu_baseline.time_validation(Vv, Fv, UVv)
            cpu["validation"] = {"seconds": vs, "cores": cpu_baseline.omp_threads(), "kind": "port",
                                 "best_of": 3,
                                 "pairs_per_s": val["pairs_aabb"] / vs,
                                 "same_report": all(float(vrep[k]) == float(val[k2]) for k, k2 in
                                                    (("overlapping_triangles_exact", "overlapping_triangles"),
                                                     ("flipped_triangles", "flipped"),
                                                     ("mirrored_islands", "mirrored")))}
        if bnd is not None:   # the boundary checks' CPU time on a sample (oracle port, one thread)
            bs, bsel, bwant = cpu_baseline.time_boundary(islands, our_uvs, args.cpu_budget_tris)
            cpu["boundary_checks"] = {"seconds": bs, "cores": 1, "kind": "port", "charts": len(bsel),
                                      "same_counts": bool(all(int(bnd["hits"][i]) == w for i, w in zip(bsel, bwant)))}
        if hier_b is not None:   # hier.Solver.relax on the same mesh (oracle port, exact solves, one thread)
            hs = cpu_baseline.time_hier_relax()
            cpu["hier_relax"] = {"seconds": hs, "cores": 1, "kind": "port",
                                 "face_iters_per_s": hier_b["faces"] * 6 / hs}
        err, ni, nt_ = cpu_baseline.uv_error_batch(islands, our_uvs, args.iters)
        cpu["uv_error_check"] = {"max_rel_uv_error": err, "islands": ni, "triangles": nt_,
                                 "against": "FP64 oracle of LSCM + gpu.Batch.arap with exact solves"}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms_max, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32+f64", "data": "synthetic",
            "config": {"workload": "uneven_islands_2000_lscm_arap20", "islands": args.islands,
                       "triangles_per_gpu": tris, "vertices_per_gpu": int(n.sum()), "arap_iters": args.iters,
                       "resid_tol": 2e-7, "parallelism": f"islands sharded, {ws} rank(s)",
                       "l2": "inputs larger than L2 (about 1 GB resident per GPU)",
                       "step": "device frames+Laplacian, batched LSCM, 20 ARAP iterations",
                       "schedule": tuned},
            "roofline": {"kernel": "k_islands<OP_ARAP>", "bound": "hbm", "achieved": achieved, "peak": hbm,
                         "unit": "GB/s", "frac": achieved / hbm, "peak_source": peak_src,
                         # DRAM read + write of one full-size ARAP launch, measured by
                         # an ncu capture of this workload (summary under profiles/)
                         "traffic": TRAFFIC_ARAP if args.islands == ISLANDS else None, "kernel_ms": arap_ms, "algorithmic_bytes": full,
                         "compulsory_bytes": comp, "compulsory_frac": achieved_c / hbm,
                         "cg_iters_total": int(st["cg_iters"].sum()),
                         "refinements_total": int(st["refinements"].sum()),
                         "max_resid": float(st["resid"].max())},
            "roofline_lscm": {"kernel": "k_islands<OP_LSCM>", "bound": "hbm",
                              "note": "streaming PCG model; the islands' vectors stay in shared memory and the "
                                      "matrices in L2, so the model's bytes can exceed what HBM delivers",
                              "achieved": lfull / (lscm_ms / 1e3) / 1e9, "peak": hbm, "unit": "GB/s",
                              "frac": lfull / (lscm_ms / 1e3) / 1e9 / hbm, "peak_source": peak_src,
                              "traffic": None, "kernel_ms": lscm_ms, "algorithmic_bytes": lfull,
                              "compulsory_bytes": lcomp,
                              "compulsory_frac": lcomp / (lscm_ms / 1e3) / 1e9 / hbm,
                              "cg_iters_total": int(st_lscm["cg_iters"].sum()),
                              "refinements_total": int(st_lscm["refinements"].sum()),
                              "max_resid": float(st_lscm["resid"].max())},
            "cpu_baseline": cpu,
            "e2e": {"value": e2e_val, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
            "gpu_launches": launches_per_step * args.steps,
            "lscm_ms": lscm_ms, "arap_ms": arap_ms,
            "graph": graphs is not None,
            "plain_gpu": plain,
            "clocks": ck,
            "validate": val,
            "boundary_checks": None if bnd is None else {k: v for k, v in bnd.items() if k != "hits"},
            "hier_solver": hier_b,
            "overlap_checks": ovl,
            "config5": c5,
            "pack": pk,
            "giant_island": gi,
            "config4_energy": c4,
            "config1": c1,
        }
        print(json.dumps(line), flush=True)
    if graphs:
        for g in graphs:
            g.close()
    if ws > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
