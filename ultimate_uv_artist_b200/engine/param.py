"""Drop-in replacement of the reference's ``engine/param.py`` (per-chart
LSCM initialisation and ARAP local/global refinement).

Same functions and signatures (engine/param.py:15-551). The numerical work
runs in the uva_b200 CUDA kernels:

* ``lscm``: conformal energy with the far-pair hard pins, solved by FP32 PCG
  with FP64 residual refinement to 1e-9 relative residual;
* ``refine(method="arap")``: the persistent island kernel with param
  semantics (per-chart pin weight, flip-safe step only from a flip-free
  start, relative-energy stop); each global step is solved to 1e-10 relative
  residual, standing in for the reference's exact LU;
* ``repair_flips``: the reference's in-order Gauss-Seidel repair, one thread
  per chart, bit-exact;
* ``chart_quality``, frames, cotangents, signed areas, rotations, right-hand
  side, flip-safe step and energies: device kernels.

``cot_laplacian`` returns a scipy matrix and ``boundary_edges_oriented`` /
``boundary_loops`` / ``_far_pair`` return host index arrays, as the reference
does; the twin test behind the boundary half-edges is a device hash kernel
(``uva_boundary_mask``). ``refine(method="slim")`` (symmetric
Dirichlet SLIM, used by the "artist" profile) runs ``uva_slim``: the SLIM
normal equations applied without forming them, FP64 CG, the reference's
flip-safe step and energy backtracking.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import scipy.sparse as sp
import torch

from .. import _lib, meshops
from ..device import DeviceBatch, Plan, require_cuda

DIRECT_LIMIT = 220_000
# the per-chart LSCM stands in for the reference's exact LU solve: its FP64
# residual bar is tighter than the batched default
LSCM_TOL = 1e-9
PARALLEL_MIN_TRIS = 20000
(OP_FRAMES, OP_COTS, OP_SIGNED_AREA, OP_ROTATIONS, OP_RHS, OP_MAX_STEP, OP_ENERGY) = range(7)
vp = C.c_void_p


def _sig():
    L = _lib.lib()
    if not getattr(L, "_uva_param_sig", False):
        L.uva_chart_op.argtypes = [C.c_int32, C.c_int32] + [vp] * 8 + [C.c_int32, C.c_int32, vp, vp, vp]
        L.uva_chart_op.restype = C.c_int32
        L.uva_csr_pcg.argtypes = [C.c_int32, vp, vp, vp, vp, vp, C.c_int32, C.c_double, C.c_int32, vp, vp, vp]
        L.uva_csr_pcg.restype = C.c_int32
        L.uva_quality_scratch_bytes.argtypes = [C.c_int64, C.c_int64, vp]
        L.uva_quality_scratch_bytes.restype = C.c_int32
        L.uva_chart_quality.argtypes = [vp, vp, vp, vp, vp, C.c_int64, vp]
        L.uva_chart_quality.restype = C.c_int32
        L._uva_param_sig = True
    return L


def _t(a, dtype, dev):
    if a is None:
        return None
    return torch.from_numpy(np.ascontiguousarray(a, dtype)).to(dev)


def _p(t):
    return C.c_void_p(t.data_ptr()) if t is not None else None


def _stream(dev):
    return C.c_void_p(torch.cuda.current_stream(dev).cuda_stream)


def _op(op, T, n, out_shape, arg=0, P=None, U=None, D=None, X=None, cots=None, R=None, area=None, out2_shape=None):
    L = _sig()
    dev = require_cuda()
    Tt = _t(np.asarray(T, np.int64).reshape(-1, 3), np.int64, dev)
    t = int(Tt.shape[0])
    args = [_t(P, np.float64, dev), _t(U, np.float64, dev), _t(D, np.float64, dev), _t(X, np.float64, dev),
            _t(cots, np.float64, dev), _t(R, np.float64, dev), _t(area, np.float64, dev)]
    out = torch.empty(out_shape, dtype=torch.float64, device=dev) if np.prod(out_shape) else torch.empty(1, dtype=torch.float64, device=dev)
    out2 = torch.empty(out2_shape, dtype=torch.float64, device=dev) if out2_shape else None
    _lib.check(L.uva_chart_op(op, arg, _p(args[0]), _p(Tt), _p(args[1]), _p(args[2]), _p(args[3]), _p(args[4]),
                              _p(args[5]), _p(args[6]), int(n), t, _p(out), _p(out2), _stream(dev)), "uva_chart_op")
    return out, out2


# ------------------------------------------------------------------ geometry
def local_frames(P, T):
    """Isometric 2D coordinates of each triangle (t,3,2), corner 0 at the
    origin, and the 3D areas (engine/param.py:19-32)."""
    T = np.asarray(T, np.int64).reshape(-1, 3)
    X, area = _op(OP_FRAMES, T, len(P), (len(T), 3, 2), P=P, out2_shape=(len(T),))
    return X.cpu().numpy(), area.cpu().numpy()


def cot_weights(X):
    """Cotangents of the angle opposite edge k, clipped to +-1e4 (engine/param.py:35-44)."""
    X = np.asarray(X, np.float64).reshape(-1, 3, 2)
    out, _ = _op(OP_COTS, np.zeros((len(X), 3), np.int64), 0, (len(X), 3), X=X)
    return out.cpu().numpy()


def _lap_triplets(T, cots):
    """(rows, cols, values) of the cotangent Laplacian (engine/param.py:47-51):
    per triangle edge k (corners k+1, k+2, half cotangent w of the opposite
    angle) the entries -w at (i, j) and (j, i) and +w at (i, i) and (j, j),
    edge by edge. Summing duplicates gives the Laplacian."""
    T = np.asarray(T, np.int64).reshape(-1, 3)
    w = 0.5 * np.asarray(cots, np.float64).reshape(-1, 3)
    i = T[:, [1, 2, 0]].reshape(-1)
    j = T[:, [2, 0, 1]].reshape(-1)
    wk = w.reshape(-1)
    rows = np.stack([i, j, i, j], 1).reshape(-1)
    cols = np.stack([j, i, i, j], 1).reshape(-1)
    vals = np.stack([-wk, -wk, wk, wk], 1).reshape(-1)
    return rows, cols, vals


def cot_laplacian(n, T, cots):
    """The cotangent Laplacian as scipy CSC (engine/param.py:54-56): the
    symmetric matrix of summed half cotangents W per undirected edge, L =
    diag(row sums of W) - W."""
    T = np.asarray(T, np.int64).reshape(-1, 3)
    w = 0.5 * np.asarray(cots, np.float64).reshape(-1, 3)
    i = T[:, [1, 2, 0]].reshape(-1)
    j = T[:, [2, 0, 1]].reshape(-1)
    W = sp.coo_matrix((w.reshape(-1), (i, j)), shape=(n, n)).tocsr()
    W = W + W.T
    return (sp.diags(np.asarray(W.sum(axis=1)).reshape(-1)) - W).tocsc()


def boundary_edges_oriented(T):
    """Directed half-edges (i -> j) whose reverse is absent, in triangle-edge
    order: all corner 0 -> 1 edges, then 1 -> 2, then 2 -> 0 (engine/param.py:
    59-68). The twin test is the uva_boundary_mask hash kernel."""
    T = np.asarray(T, np.int64).reshape(-1, 3)
    if T.size == 0:
        raise ValueError("boundary_edges_oriented: empty triangle list")
    keep = meshops.boundary_mask(T).cpu().numpy()
    a = T.T.reshape(-1)
    b = T[:, [1, 2, 0]].T.reshape(-1)
    return a[keep], b[keep]


def boundary_loops(T):
    """Boundary loops as vertex arrays (engine/param.py:71-94). A loop starts
    at the first unused boundary source in half-edge order and follows, from
    each vertex, its first outgoing boundary half-edge (half-edge order) to a
    vertex not yet used, or back to the start, which closes the loop."""
    bi, bj = boundary_edges_oriented(T)
    return _trace_loops(bi, bj)


def _trace_loops(bi, bj):
    """The loop walk of boundary_loops over directed boundary half-edges."""
    bi = np.asarray(bi, np.int64)
    bj = np.asarray(bj, np.int64)
    if len(bi) == 0:
        return []
    order = np.argsort(bi, kind="stable")          # outgoing half-edges grouped by source
    src = bi[order]
    dst = bj[order].tolist()
    starts = np.searchsorted(src, bi)              # first outgoing half-edge of each source
    ends = np.searchsorted(src, bi, side="right")
    first = dict(zip(bi.tolist(), zip(starts.tolist(), ends.tolist())))
    used = set()
    loops = []
    for s0 in bi.tolist():
        if s0 in used:
            continue
        used.add(s0)
        loop = [s0]
        v = s0
        while True:
            a, b = first.get(v, (0, 0))
            nxt = next((x for x in dst[a:b] if x == s0 or x not in used), None)
            if nxt is None or nxt == s0:
                break
            loop.append(nxt)
            used.add(nxt)
            v = nxt
        loops.append(np.asarray(loop, np.int64))
    return loops


def signed_areas(U, T):
    """Signed UV area per triangle (engine/param.py:97-99)."""
    T = np.asarray(T, np.int64).reshape(-1, 3)
    out, _ = _op(OP_SIGNED_AREA, T, len(U), (len(T),), U=U)
    return out.cpu().numpy()


# ------------------------------------------------------------------ solvers
class SPDSolver:
    """Reusable solver for a fixed SPD matrix (engine/param.py:103-132): FP64
    Jacobi-PCG on the device; up to DIRECT_LIMIT unknowns it iterates to
    1e-12 relative residual in place of the reference's sparse LU."""

    def __init__(self, A):
        self.n = A.shape[0]
        self.A = A.tocsc()
        csr = A.tocsr()
        csr.sum_duplicates()
        dev = require_cuda()
        self.dev = dev
        self.rp = torch.from_numpy(csr.indptr.astype(np.int32)).to(dev)
        self.ci = torch.from_numpy(csr.indices.astype(np.int32)).to(dev)
        self.val = torch.from_numpy(csr.data.astype(np.float64)).to(dev)
        self.lu = None

    def solve(self, b, x0=None, tol=1e-7, maxiter=None):
        L = _sig()
        b = np.asarray(b, np.float64)
        B = b if b.ndim == 2 else b[:, None]
        ncol = B.shape[1]
        tol_eff = 1e-12 if self.n <= DIRECT_LIMIT else tol
        iters = maxiter or max(2000, 4 * self.n)
        bt = torch.from_numpy(np.ascontiguousarray(B.T)).to(self.dev)
        if x0 is None:
            xt = torch.zeros_like(bt)
        else:
            X0 = np.asarray(x0, np.float64)
            X0 = X0 if X0.ndim == 2 else X0[:, None]
            xt = torch.from_numpy(np.ascontiguousarray(X0.T)).to(self.dev)
        scratch = torch.empty(3 * max(self.n, 1) * ncol, dtype=torch.float64, device=self.dev)
        it = torch.zeros(ncol, dtype=torch.int32, device=self.dev)
        _lib.check(L.uva_csr_pcg(self.n, _p(self.rp), _p(self.ci), _p(self.val), _p(bt), _p(xt), ncol, float(tol_eff),
                                 int(iters), _p(scratch), _p(it), _stream(self.dev)), "uva_csr_pcg")
        x = xt.cpu().numpy().T
        return x if b.ndim == 2 else x[:, 0]


class _ChartSolver:
    """What ``refine`` returns as ``solver``: the chart's device batch (topology
    plan, frames, Laplacian), reused when the caller passes it back."""

    def __init__(self, P, T):
        P = np.asarray(P, np.float64)
        T = np.asarray(T, np.int64)
        self.key = (len(P), T.shape[0], hash(T.tobytes()), hash(P.tobytes()))
        self.db = DeviceBatch(P, T, [0, len(P)], [0, len(T)], semantics=_lib.SEM_PARAM)

    def matches(self, P, T):
        P = np.asarray(P, np.float64)
        T = np.asarray(T, np.int64)
        return self.key == (len(P), T.shape[0], hash(T.tobytes()), hash(P.tobytes()))


def _chart(P, T, solver=None):
    if isinstance(solver, _ChartSolver) and solver.matches(P, T):
        return solver
    return _ChartSolver(P, T)


# ------------------------------------------------------------------ LSCM
def lscm(P, T, X=None, cots=None, pins=None):
    """LSCM with two hard pins (engine/param.py:136-169). Raises ValueError
    for a chart without boundary."""
    P = np.asarray(P, np.float64)
    T = np.asarray(T, np.int64)
    ch = _ChartSolver(P, T)
    db = ch.db
    if pins is not None:
        db.pins[0, 1] = int(pins[0])
        db.pins[0, 2] = int(pins[1])
    db.lscm(tol=LSCM_TOL)
    st = db.island_status()
    if st["flags"][0] & _lib.ST_NOBOUNDARY:
        raise ValueError("chart has no boundary (closed surface): needs a cut")
    return db.uvs()


def _far_pair(P, cand):
    """Boundary vertex farthest from the boundary centroid, then the one
    farthest from it (engine/param.py:172-179)."""
    Q = P[cand]
    c = Q.mean(0)
    i = cand[np.argmax(((Q - c) ** 2).sum(1))]
    j = cand[np.argmax(((Q - P[i]) ** 2).sum(1))]
    if i == j:
        j = cand[0] if cand[0] != i else cand[-1]
    return int(i), int(j)


def tutte(P, T):
    """Uniform-weight Tutte embedding onto a circle (engine/param.py:182-202)."""
    T = np.asarray(T, np.int64)
    loops = boundary_loops(T)
    loop = max(loops, key=len)
    n = len(P)
    P = np.asarray(P, np.float64)
    seg = np.linalg.norm(P[np.roll(loop, -1)] - P[loop], axis=1)
    t = np.r_[0, np.cumsum(seg)[:-1]] / max(seg.sum(), 1e-300) * 2 * np.pi
    r = seg.sum() / (2 * np.pi)
    Ub = np.stack([np.cos(t), np.sin(t)], 1) * r
    I = np.concatenate([T[:, 0], T[:, 1], T[:, 2], T[:, 1], T[:, 2], T[:, 0]])
    J = np.concatenate([T[:, 1], T[:, 2], T[:, 0], T[:, 0], T[:, 1], T[:, 2]])
    A = sp.csr_matrix((np.ones(len(I)), (I, J)), shape=(n, n))
    A.data[:] = 1.0
    deg = np.asarray(A.sum(1)).ravel()
    Lu = sp.diags(deg) - A
    fixed = np.zeros(n, bool)
    fixed[loop] = True
    U = np.zeros((n, 2))
    U[loop] = Ub
    fr = ~fixed
    rhs = -Lu[fr][:, fixed] @ Ub
    U[fr] = SPDSolver(Lu[fr][:, fr]).solve(rhs)
    return U


# ------------------------------------------------------------------ local step kernels
def _arap_rotations(U, T, X, cots, mode, sd_weights):
    """Per-triangle target rotation and weight matrices (engine/param.py:206-256):
    mode 0 the closest rotation and identity weights, mode 1 the SVD-based
    rotation and the SLIM symmetric-Dirichlet weights."""
    T = np.asarray(T, np.int64).reshape(-1, 3)
    if mode == 1:
        R, Wm = _op(OP_ROTATIONS, T, len(U), (len(T), 2, 2), arg=1, U=U, X=X, out2_shape=(len(T), 2, 2))
        return R.cpu().numpy(), Wm.cpu().numpy()
    R, _ = _op(OP_ROTATIONS, T, len(U), (len(T), 2, 2), U=U, X=X)
    Wm = np.broadcast_to(np.eye(2), (len(T), 2, 2)).copy()
    return R.cpu().numpy(), Wm


def _max_step(U, D, T):
    """Flip-safe step bound (engine/param.py:259-291)."""
    T = np.asarray(T, np.int64).reshape(-1, 3)
    out, _ = _op(OP_MAX_STEP, T, len(U), (1,), U=U, D=D)
    return float(out.item())


def _energy(U, T, X, area, kind):
    """ARAP (kind 0) or symmetric Dirichlet (kind 1) energy (engine/param.py:294-319)."""
    T = np.asarray(T, np.int64).reshape(-1, 3)
    out, _ = _op(OP_ENERGY, T, len(U), (1,), arg=int(kind), U=U, X=X, area=area)
    return float(out.item())


def _arap_rhs(n, T, X, cots, R):
    """ARAP right-hand side (engine/param.py:457-474)."""
    T = np.asarray(T, np.int64).reshape(-1, 3)
    out, _ = _op(OP_RHS, T, n, (n, 2), X=X, cots=cots, R=R)
    return out.cpu().numpy()


def refine(P, T, U, iters=10, method="arap", X=None, area=None, cots=None, solver=None, line_search=True, tol=1e-5,
           pin=None):
    """Local-global refinement (engine/param.py:379-454). Returns (U, solver)."""
    if method == "slim":
        # SLIM (param.py:415-454): the reference solves each global step
        # exactly when 2n <= DIRECT_LIMIT, else CG rtol 1e-6, 500 iterations
        ch = _chart(P, T, solver)
        db = ch.db
        db.U[:db.n].copy_(torch.from_numpy(np.asarray(U, np.float64).reshape(-1, 2)))
        direct = 2 * db.n <= DIRECT_LIMIT
        db.slim(iters=int(iters), energy_tol=float(tol), cg_tol=1e-12 if direct else 1e-6,
                cg_max=50000 if direct else 500)
        return db.uvs(), None
    if method != "arap":
        raise ValueError(f"unknown refine method {method!r}")
    ch = _chart(P, T, solver)
    db = ch.db
    db.U[:db.n].copy_(torch.from_numpy(np.asarray(U, np.float64).reshape(-1, 2)))
    db.pins[0, 0] = 0 if pin is None else int(pin)
    db.arap(iters=int(iters), line_search=bool(line_search), energy_tol=float(tol), tol=1e-10)
    return db.uvs(), ch


# ------------------------------------------------------------------ flip repair
def repair_flips(U, T, rounds=60):
    """Move interior vertices of folded triangles to their 1-ring centroid, in
    triangle order (engine/param.py:504-516)."""
    U = np.asarray(U, np.float64)
    T = np.asarray(T, np.int64)
    db = DeviceBatch(np.zeros((len(U), 3)), T, [0, len(U)], [0, len(T)], U=U, semantics=_lib.SEM_PARAM)
    db.repair_flips(int(rounds), serial=True)
    return db.uvs()


# ------------------------------------------------------------------ chart quality
def chart_quality(P, T, U, X=None, area=None):
    """Area-weighted distortion of one chart (engine/param.py:520-551)."""
    ch = _ChartSolver(P, T)
    q = chart_quality_batch(ch.db, np.asarray(U, np.float64))
    return q[0]


def chart_quality_batch(db, U=None):
    """chart_quality of every island of a PARAM-semantics device batch."""
    L = _sig()
    if U is not None:
        db.U[:db.n].copy_(torch.from_numpy(np.asarray(U, np.float64).reshape(-1, 2)))
    dev = db.dev
    nb = C.c_int64()
    _lib.check(L.uva_quality_scratch_bytes(db.t, db.nc, C.byref(nb)), "uva_quality_scratch_bytes")
    scratch = torch.empty(max(int(nb.value), 256), dtype=torch.uint8, device=dev)
    out = torch.zeros((max(db.nc, 1), 8), dtype=torch.float64, device=dev)
    pa = torch.empty(max(db.t, 1), dtype=torch.float64, device=dev)
    pr = torch.empty(max(db.t, 1), dtype=torch.float64, device=dev)
    _lib.check(L.uva_chart_quality(C.byref(db.desc), _p(out), _p(pa), _p(pr), _p(scratch), nb.value, _stream(dev)),
               "uva_chart_quality")
    # per-triangle values into page-locked host memory (torch's caching host
    # allocator reuses it once the caller drops the arrays): no page faults
    # on fresh pageable memory, asynchronous DMA on the current stream
    from ..device import host_empty
    pa_h, pr_h = host_empty(db.t, np.float64), host_empty(db.t, np.float64)
    if db.t:
        torch.from_numpy(pa_h).copy_(pa[:db.t], non_blocking=True)
        torch.from_numpy(pr_h).copy_(pr[:db.t], non_blocking=True)
    o = out.cpu().numpy()   # synchronises the stream: the copies above are done
    pa, pr = pa_h, pr_h
    tofs = db.plan.tofs
    res = []
    for i in range(db.nc):
        sl = slice(tofs[i], tofs[i + 1])
        res.append({"flips": int(o[i, 0]), "aniso_p95": float(o[i, 1]), "aniso_mean": float(o[i, 2]),
                    "area_p95": float(o[i, 3]), "area_logdev": float(o[i, 4]), "stretch": float(o[i, 5]),
                    "scale": float(o[i, 6]), "per_tri_aniso": pa[sl], "per_tri_area": pr[sl]})
    return res
