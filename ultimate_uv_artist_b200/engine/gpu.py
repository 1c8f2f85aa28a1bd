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

import numpy as np
import torch

from .. import _lib
from ..device import DeviceBatch, Plan, concat_charts, require_cuda


def csr32(A):
    """CSR with int32 indices (engine/gpu.py:16-20)."""
    A = A.to_sparse_csr() if A.layout != torch.sparse_csr else A
    return torch.sparse_csr_tensor(A.crow_indices().to(torch.int32), A.col_indices().to(torch.int32),
                                   A.values(), A.shape)


def spmm(L, X):
    """L @ X for a few dense columns (engine/gpu.py:23-28)."""
    if X.dim() == 1:
        return L @ X
    return torch.stack([L @ X[:, k].contiguous() for k in range(X.shape[1])], 1)


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
    """Undirected unique edges, inverse map and use counts (engine/gpu.py:39-49)."""
    a = torch.cat([T[:, 1], T[:, 2], T[:, 0]])
    b = torch.cat([T[:, 2], T[:, 0], T[:, 1]])
    key = torch.minimum(a, b) * n + torch.maximum(a, b)
    uk, inv = torch.unique(key, return_inverse=True)
    cnt = torch.bincount(inv, minlength=len(uk))
    return uk // n, uk % n, inv, cnt


def sym_csr(n, ea, eb, off, diag):
    """Symmetric int32 CSR from unique edges (engine/gpu.py:52-63)."""
    dev = ea.device
    rows = torch.cat([ea, eb, torch.arange(n, device=dev)])
    cols = torch.cat([eb, ea, torch.arange(n, device=dev)])
    vals = torch.cat([off, off, diag])
    order = torch.argsort(rows * n + cols)
    rows, cols, vals = rows[order], cols[order], vals[order]
    crow = torch.zeros(n + 1, dtype=torch.int64, device=dev)
    crow[1:] = torch.cumsum(torch.bincount(rows, minlength=n), 0)
    return torch.sparse_csr_tensor(crow.to(torch.int32), cols.to(torch.int32), vals, (n, n))


class Batch:
    """charts: list of (P (k,3), T (t,3), U (k,2)) -> one device-resident batch.

    ``U`` may be None for a chart; call ``lscm()`` to initialise every chart
    with batched LSCM (an addition: the reference initialises per chart on
    the CPU with param.lscm before building the Batch).
    """

    def __init__(self, charts, dev=None, dtype=torch.float32, stream=None):
        self.dev = require_cuda(dev if dev is not None else device())
        self.dt = dtype
        # positions (and UVs) are concatenated; the topology plan reads every
        # chart's triangles where they are; the positions' upload runs while
        # the plan is built, and each finished range of the plan's arrays is
        # copied while the next one is exported
        P, Tc, U, vofs, tofs = concat_charts(charts, with_t=False)
        self.nc = len(charts)
        self.offsets = vofs.copy()
        self.n = int(vofs[-1])
        self._tofs = tofs
        with (torch.cuda.stream(stream) if stream is not None else contextlib.nullcontext()):
            P_dev = torch.from_numpy(P).to(self.dev, non_blocking=True) if self.n else None
        plan = Plan(None, vofs, tofs, chart_tris=Tc[:2], device=self.dev, stream=stream)   # export || copies
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

    def _wdiag_by_vertex(self):
        """Row sums of the weights, reordered from solver rows to vertices."""
        vr = self.db.vert_row[:self.n].to(torch.int64)
        base = torch.repeat_interleave(self.db.vofs[:-1].to(torch.int64),
                                       torch.as_tensor(np.diff(self.offsets), device=self.dev))
        return self.db.wdiag[:self.n][base + vr]

    @property
    def dinv(self):
        d = self._wdiag_by_vertex().clone()
        d[self.pins] += self.db.wpin[:self.nc]
        return (1.0 / d.clamp_min(1e-30)).to(self.dt)

    @property
    def L(self):
        """The soft-pinned cotangent Laplacian as an int32 sparse CSR tensor."""
        ea, eb, _ = self._edges
        p = self.db.plan
        wsum = self.db.wedge[:p.E].to(self.dt)
        keep = ea != eb
        diag = self._wdiag_by_vertex().clone()
        diag[self.pins] += self.db.wpin[:self.nc]
        return sym_csr(self.n, ea[keep], eb[keep], -wsum[keep], diag.to(self.dt))

    @property
    def _edges(self):
        """(ea, eb, cnt) of the unique edges, global vertex ids (gpu.py:129)."""
        ea, eb, _, cnt = unique_edges(self.T, self.n)
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
