"""Drop-in replacement of the reference's ``engine/gpu.py`` (batched GPU ARAP).

Same public surface as the reference module (engine/gpu.py:16-299):
``csr32``, ``spmm``, ``device``, ``unique_edges``, ``sym_csr`` and the
``Batch`` class with ``arap``, ``repair_flips``, ``orient_positive``,
``shrink``, ``chart_uvs``, ``flips_per_chart``, ``signed_area``,
``jacobians`` and the attributes callers read.

What changes underneath: every Batch computation runs in the uva_b200 CUDA
kernels (sm_100a) on a device-resident batch. A global step is solved per
island to ||b - L x|| <= 2e-7 ||b|| per column, checked in FP64 (FP32 CG with
FP64 residual refinement), instead of at most 40 CG iterations with a 1e-6
stop test on the whole batch and a host sync per iteration. UVs are kept in FP64 on the device;
``U`` returns them in the Batch dtype. There is no CPU path: constructing a
Batch without a CUDA device raises RuntimeError.
"""
from __future__ import annotations

import contextlib
import ctypes as C

import numpy as np
import torch

from .. import _lib, meshops
from ..device import ChartArrays, DeviceBatch, DevicePlan, Plan, require_cuda


def csr32(A):
    """The matrix as a torch CSR tensor with int32 row offsets and columns:
    the layout the uva_csr_spmm kernel reads (engine/gpu.py:16-20)."""
    if A.layout != torch.sparse_csr:
        A = (A.coalesce() if A.layout == torch.sparse_coo else A).to_sparse_csr()
    crow, col = A.crow_indices(), A.col_indices()
    if crow.dtype == torch.int32 and col.dtype == torch.int32:
        return A
    return torch.sparse_csr_tensor(crow.to(torch.int32), col.to(torch.int32), A.values(), A.shape)


def spmm(L, X):
    """L @ X for a vector or a few dense columns (engine/gpu.py:23-28): one
    uva_csr_spmm launch reads the matrix once for all columns."""
    return meshops.csr_spmm(csr32(L), X)


def device():
    """engine/gpu.py:30-36, without the CPU fallback: the B200 path needs CUDA."""
    try:
        import comfy.model_management as mm  # noqa: F401 - optional host app
        d = mm.get_torch_device()
        if d.type == "cuda":
            return d
    except Exception:  # noqa: BLE001 - no ComfyUI
        pass
    return require_cuda()


def unique_edges(T, n):
    """Unique undirected edges (ea < eb ascending), the edge of each of the
    3t half-edges (k t + f: triangle f's edge opposite corner k) and the use
    count of each edge (engine/gpu.py:39-49), by the uva_unique_edges
    counting-sort kernels. Results live on T's device."""
    T = torch.as_tensor(T)
    out = meshops.unique_edges(T, n)
    return tuple(o.to(T.device) for o in out) if not T.is_cuda else out


def sym_csr(n, ea, eb, off, diag):
    """Symmetric CSR (int32 indices) with ``off`` at (ea, eb) and (eb, ea)
    and ``diag`` on the diagonal (engine/gpu.py:52-63), assembled by the
    uva_sym_csr kernels."""
    return meshops.sym_csr(n, ea, eb, off, diag)


class Batch:
    """charts: list of (P (k,3), T (t,3), U (k,2)) -> one device-resident batch.

    ``U`` may be None for a chart; call ``lscm()`` to initialise every chart
    with batched LSCM (an addition: the reference initialises per chart on
    the CPU with param.lscm before building the Batch).
    """

    def __init__(self, charts, dev=None, dtype=torch.float32, stream=None, plan_on="device"):
        self.dev = require_cuda(dev if dev is not None else device())
        self.dt = dtype
        ca = ChartArrays(charts)
        vofs, tofs = ca.vofs, ca.tofs
        self.nc = len(charts)
        self.offsets = vofs.copy()
        self.n = int(vofs[-1])
        self._tofs = tofs
        # The topology plan is built on the device from the triangles: its
        # build runs while the host copies the positions (float32 charts
        # travel as float32) and uploads them. plan_on="host" builds the same
        # arrays on the host cores and copies them range by range.
        ctx = torch.cuda.stream(stream) if stream is not None else contextlib.nullcontext()
        plan = None
        if plan_on == "device":
            plan = DevicePlan(ca.chart_tris[:2], vofs, tofs, device=self.dev, stream=stream, finish=False)
        P, U = ca.points(fp32=plan_on == "device")
        with ctx:
            P_dev = torch.from_numpy(P).to(self.dev, non_blocking=True) if self.n else None
        if plan is not None:
            plan.finish()
        else:
            plan = Plan(None, vofs, tofs, chart_tris=ca.chart_tris[:2], device=self.dev, stream=stream)
        self.db = DeviceBatch(P_dev if P_dev is not None else P, None, vofs, tofs, U=U, semantics=_lib.SEM_BATCH,
                              device=self.dev, stream=stream, plan=plan)
        self.db._host_src = (P, U)          # the asynchronous copies read these until they finish
        if P_dev is not None:
            self.db.h2d_bytes += P.nbytes
        self.last_status = None

    # ------------------------------------------------------------ attributes
    @property
    def U(self):
        return self.db.U[:self.n].to(self.dt)

    @U.setter
    def U(self, value):
        v = torch.as_tensor(value).to(self.dev, torch.float64).reshape(-1, 2)
        self.db.U[:self.n].copy_(v)

    @property
    def T(self):
        tri = self.db.tri4[:self.db.t, :3].to(torch.int64)
        return tri + self.db.vofs[:-1].to(torch.int64)[self.db.tri4[:self.db.t, 3].to(torch.int64)][:, None]

    @property
    def cv(self):
        return torch.repeat_interleave(torch.arange(self.nc, device=self.dev),
                                       torch.as_tensor(np.diff(self.offsets), device=self.dev))

    @property
    def ct(self):
        return self.db.tri4[:self.db.t, 3].to(torch.int64)

    @property
    def area(self):
        return self.db.frame[:self.db.t, 3].to(self.dt)

    @property
    def ok(self):
        return self.db.wtri[:self.db.t, 3] != 0

    @property
    def w(self):
        return self.db.wtri[:self.db.t, :3].to(self.dt)

    @property
    def x1(self):
        return self.db.frame[:self.db.t, 0].to(self.dt)

    @property
    def x2(self):
        return self.db.frame[:self.db.t, 1].to(self.dt)

    @property
    def y2(self):
        return self.db.frame[:self.db.t, 2].to(self.dt)

    @property
    def X(self):
        fr = self.db.frame[:self.db.t]
        X = torch.zeros((self.db.t, 3, 2), dtype=self.dt, device=self.dev)
        okm = self.ok
        X[:, 1, 0] = torch.where(okm, fr[:, 0], 0).to(self.dt)
        X[:, 2, 0] = fr[:, 1].to(self.dt)
        X[:, 2, 1] = torch.where(okm, fr[:, 2], 0).to(self.dt)
        return X

    @property
    def scale(self):
        return self.db.tscale[:self.db.t].to(self.dt)

    @property
    def pins(self):
        return torch.as_tensor(self.offsets[:-1], device=self.dev)

    @property
    def wpin(self):
        return self.db.wpin[0].to(self.dt) if self.nc else torch.tensor(1e-12, dtype=self.dt, device=self.dev)

    def _diag(self, self_loops):
        """FP64 diagonal of the soft-pinned Laplacian (gpu.py:131-140): the
        summed edge weights at both endpoints of every edge, plus the pin
        weights. With self_loops the edges of degenerate triangles that join
        a vertex to itself count too, as in the reference's diagonal; their
        off-diagonal entries cancel them in its matrix."""
        ea, eb, _ = self._edges
        w = self.db.wedge[:self.db.plan.E]
        if not self_loops:
            keep = ea != eb
            ea, eb, w = ea[keep], eb[keep], w[keep]
        w = w.contiguous()
        d = meshops.segment_sum(w, ea, self.n) + meshops.segment_sum(w, eb, self.n)
        d[self.pins] += self.db.wpin[:self.nc]
        return d

    @property
    def dinv(self):
        return (1.0 / self._diag(True).clamp_min(1e-30)).to(self.dt)

    @property
    def L(self):
        """The soft-pinned cotangent Laplacian as an int32 sparse CSR tensor:
        the batch's summed edge weights off the diagonal, their row sums plus
        the pin weights on it (self-loop edges of degenerate triangles cancel
        and are left out)."""
        ea, eb, _ = self._edges
        wsum = self.db.wedge[:self.db.plan.E].to(self.dt)
        keep = ea != eb
        return sym_csr(self.n, ea[keep], eb[keep], -wsum[keep], self._diag(False).to(self.dt))

    @property
    def _edges(self):
        """(ea, eb, cnt) of the unique edges in global vertex ids
        (gpu.py:128-129), read off the plan's own edge numbering: the plan
        numbers each island's edges in ascending (lo, hi) order and the
        islands in order, which is the ascending global order."""
        E = self.db.plan.E
        ea = torch.empty(E, dtype=torch.int64, device=self.dev)
        eb = torch.empty_like(ea)
        cnt = torch.empty_like(ea)
        _lib.check(_lib.lib().uva_batch_edges(C.byref(self.db.desc), meshops._p(ea), meshops._p(eb), meshops._p(cnt),
                                              meshops._stream(self.dev)), "uva_batch_edges")
        return ea, eb, cnt

    # ------------------------------------------------------------ pieces
    def jacobians(self, U=None):
        U = self.db.U if U is None else U
        J = self.db.jacobians(U)
        return tuple(J[:, k].to(self.dt) for k in range(4))

    def signed_area(self, U=None):
        return self.db.signed_area(U).to(self.dt)

    def flips_per_chart(self, U=None):
        if U is not None:
            keep = self.db.U[:self.n].clone()
            self.U = U
            out = self.db.flips_per_chart().to(self.dt)
            self.db.U[:self.n].copy_(keep)
            return out
        return self.db.flips_per_chart().to(self.dt)

    # ------------------------------------------------------------ solvers
    def lscm(self, tol=None):
        """Batched LSCM initialisation of every chart (hard far-pair pins)."""
        self.db.lscm(tol=tol)
        st = self.db.island_status()
        if (st["flags"] & _lib.ST_NOBOUNDARY).any():
            raise ValueError("chart has no boundary (closed surface): needs a cut")
        self.last_status = st
        return self.U

    def arap(self, iters=8, line_search=True, cg_iters=40, tol=None):
        """ARAP local/global iterations (engine/gpu.py:230-249).

        ``cg_iters`` is accepted for signature compatibility; convergence is
        decided per island by the FP64 residual test (``tol``, default 2e-7).
        """
        self.db.arap(iters=iters, line_search=line_search, tol=tol)
        return self.U

    def status(self):
        """Per-island solver status of the last solve (host structured array)."""
        return self.db.island_status()

    def repair_flips(self, rounds=60):
        self.db.repair_flips(rounds)
        return self.U

    def orient_positive(self):
        self.db.orient_positive()

    def shrink(self, tri_idx, factor=0.6, floor=0.05, rings=3):
        if len(tri_idx) == 0:
            return
        self.db.shrink(tri_idx, factor, floor, rings)

    def boundary_intersections(self, max_report=1000):
        """charts.boundary_intersections (engine/charts.py:596-608) of every
        chart of the batch at its current UVs, in one launch: numpy int64 per
        chart (-1 where the reference would raise for non-finite UVs). An
        addition: the reference calls it chart by chart on the host."""
        return self.db.boundary_hits(_lib.SEG_COUNT, max_report).cpu().numpy()

    def chart_uvs(self):
        U = self.db.uvs()
        return [U[a:b] for a, b in zip(self.offsets[:-1], self.offsets[1:])]
