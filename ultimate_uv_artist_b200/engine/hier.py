"""Drop-in replacement of the per-chart validity checks of the reference's
``engine/hier.py``: ``boundary_directed`` (:158-180), ``charts_collide``
(:183-225) and ``chart_checks`` (:269-353), with the reference's signatures
and results.

The topology (which corner edges are boundary edges, Euler characteristic,
boundary loops) is integer work over face arrays, done here with vectorised
numpy on the host like the reference's host code; the geometric test, "do
two boundary segments of the chart cross", runs on the GPU for all charts
in one launch (uva_boundary_hits, mode any, exact FP64 without fused
multiply-add). As in the reference, a chart with fewer than 3 boundary
segments never collides; in chart_checks one whose segment extent is not
below 1e300 (the caller substitutes 1e301 for non-finite UVs) always does,
while charts_collide tests such a chart's pairs like any other.
"""
from __future__ import annotations

import numpy as np

from .. import segments


def _boundary_corners(F, FF, faces, loc, chart, CV, nv=None):
    """isb (n, 3): corner edge k of local face i is a boundary edge unless the
    neighbour across it (FF) is a face of the same chart whose corner on the
    shared vertex F[f, k] (its first match) has the same UV vertex
    (engine/hier.py:275-291). With ``nv``, also vchart (nv,): the chart of
    the last corner (face order) naming each UV vertex, -1 for none. One
    device pass (uva_hier_boundary_corners)."""
    import ctypes as C
    import torch
    from .. import _lib
    from ..device import require_cuda
    F = np.asarray(F, np.int64).reshape(-1, 3)
    FF = np.asarray(FF, np.int64).reshape(-1, 3)
    faces = np.asarray(faces, np.int64).reshape(-1)
    loc = np.asarray(loc, np.int64).reshape(-1)
    chart = np.asarray(chart, np.int64).reshape(-1)
    CV = np.asarray(CV, np.int64).reshape(-1, 3)
    n, nf = len(faces), len(F)
    nvv = 0 if nv is None else int(nv)
    if n == 0:
        isb = np.zeros((0, 3), bool)
        return isb if nv is None else (isb, -np.ones(nvv, np.int64))
    if len(CV) != n or len(chart) != n or len(FF) != nf:
        raise ValueError("hier: faces, CV, chart or FF of inconsistent lengths")
    if faces.min() < -nf or faces.max() >= nf:
        raise IndexError("hier: faces out of range")
    faces = np.where(faces < 0, faces + nf, faces)        # numpy indexing counts from the end
    if len(loc) < nf:   # only the neighbours' entries are read
        if (FF[faces] >= len(loc)).any():
            raise IndexError("hier: loc shorter than a neighbour face id")
        loc = np.concatenate([loc, -np.ones(nf - len(loc), np.int64)])
    dev = require_cuda(None)
    up = lambda a: torch.from_numpy(np.ascontiguousarray(a, np.int32)).to(dev)
    Fd, FFd, fd, ld, cd, cvd = up(F), up(FF), up(faces), up(loc), up(chart), up(CV)
    isb = torch.empty((n, 3), dtype=torch.uint8, device=dev)
    vchart = torch.empty(max(nvv, 1), dtype=torch.int32, device=dev)
    flags = torch.empty(1, dtype=torch.int32, device=dev)
    st = torch.cuda.current_stream(dev)
    _lib.check(_lib.lib().uva_hier_boundary_corners(Fd.data_ptr(), FFd.data_ptr(), nf, fd.data_ptr(), ld.data_ptr(),
                                                    cd.data_ptr(), cvd.data_ptr(), n, nvv, isb.data_ptr(),
                                                    vchart.data_ptr(), flags.data_ptr(), C.c_void_p(st.cuda_stream)),
               "uva_hier_boundary_corners")
    out = isb.cpu().numpy().astype(bool)
    if int(flags.item()):
        raise IndexError("hier: an FF, loc or CV index is out of range")
    if nv is None:
        return out
    return out, vchart[:nvv].cpu().numpy().astype(np.int64)


def boundary_directed(F, FF, faces, loc, chart, CV):
    """Directed boundary edges (local vertex ids) of all charts, face by face
    (engine/hier.py:158-180)."""
    CV = np.asarray(CV, np.int64).reshape(-1, 3)
    isb = _boundary_corners(F, FF, faces, loc, chart, CV)
    ba = CV[isb]
    bb = CV[:, [1, 2, 0]][isb]
    return ba.copy(), bb.copy()


def _collide(UV, ba, bb, bc, nchart, mode=segments.ANY):
    """GPU test (mode ANY or ANY_ALL) of the segments (ba -> bb) of chart bc."""
    order = np.argsort(bc, kind="stable")
    counts = np.bincount(bc, minlength=nchart) if len(bc) else np.zeros(nchart, np.int64)
    sofs = np.zeros(nchart + 1, np.int64)
    np.cumsum(counts, out=sofs[1:])
    seg = np.stack([ba[order], bb[order]], 1) if len(ba) else np.zeros((0, 2), np.int64)
    out = segments.boundary_hits(np.asarray(UV, np.float64).reshape(-1, 2), sofs, seg, mode)
    if (out < 0).any():
        raise IndexError("hier: a boundary vertex id is outside UV")
    return out > 0


def charts_collide(CV, UV, chart, nchart, nv):
    """Per chart: True if its UV boundary self-intersects (exact segment test);
    boundary half-edges are corner edges whose reverse is absent
    (engine/hier.py:183-225)."""
    CV = np.asarray(CV, np.int64).reshape(-1, 3)
    chart = np.asarray(chart, np.int64)
    nchart, nv = int(nchart), int(nv)
    if nchart == 0:
        return np.zeros(0, bool)
    a = CV.reshape(-1)
    b = CV[:, [1, 2, 0]].reshape(-1)
    keep = ~np.isin(b * nv + a, a * nv + b)
    bc = np.repeat(chart, 3)[keep]
    return _collide(UV, a[keep], b[keep], bc, nchart, segments.ANY_ALL)


def _components(ba, bb, nv):
    """Roots of a union-find over the boundary edges, in the reference's
    order (engine/hier.py:320-324): parent array after all unions."""
    p = np.arange(nv, dtype=np.int64)

    def find(x):
        r = x
        while p[r] != r:
            r = p[r]
        while p[x] != r:
            nx = p[x]
            p[x] = r
            x = nx
        return r

    for q in range(len(ba)):
        ra, rb = find(int(ba[q])), find(int(bb[q]))
        if ra != rb:
            p[rb] = ra
    return p, find


def chart_checks(F, FF, faces, loc, chart, CV, UV, nchart, nv):
    """Linear-time per-chart checks -> (collide, chi, loops)
    (engine/hier.py:269-353): boundary edges from face adjacency, Euler
    characteristic chi = V - E + F, boundary loops (connected components of
    the boundary edges), and the exact boundary self-intersection test."""
    chi, loops, ba, bb, bc = _boundary_topology(F, FF, faces, loc, chart, CV, nchart, nv)
    collide = _collide(UV, ba, bb, bc, int(nchart))
    return collide, chi, loops


def _boundary_topology(F, FF, faces, loc, chart, CV, nchart, nv):
    """chart_checks without the segment test: (chi, loops, ba, bb, bc) with
    the boundary edges ba -> bb of chart bc in face order. The corner test
    and the vertex charts run on the device; the per-chart counts and the
    boundary loops on the host."""
    CV = np.asarray(CV, np.int64).reshape(-1, 3)
    chart = np.asarray(chart, np.int64)
    nchart, nv = int(nchart), int(nv)
    n = len(CV)
    # vchart[v]: chart of the last corner (face order) that names v
    isb, vchart = _boundary_corners(F, FF, faces, loc, chart, CV, nv)
    Fc = np.bincount(chart, minlength=nchart).astype(np.int64) if n else np.zeros(nchart, np.int64)
    nb_c = np.bincount(chart, weights=isb.sum(1), minlength=nchart).astype(np.int64) if n else np.zeros(nchart, np.int64)
    Vc = np.bincount(vchart[vchart >= 0], minlength=nchart).astype(np.int64)
    chi = Vc - (3 * Fc + nb_c) // 2 + Fc
    ba = CV[isb]
    bb = CV[:, [1, 2, 0]][isb]
    bc = np.repeat(chart, 3).reshape(-1, 3)[isb]
    # loops: components of the boundary edges, each counted for the chart of
    # its root. When every component lies in one chart the root's chart does
    # not depend on the union order; otherwise replay the reference's order.
    loops = np.zeros(nchart, np.int64)
    if len(ba):
        import scipy.sparse as sp
        from scipy.sparse.csgraph import connected_components
        verts = np.unique(np.concatenate([ba, bb]))
        idx = np.searchsorted(verts, ba), np.searchsorted(verts, bb)
        m = len(verts)
        G = sp.coo_matrix((np.ones(len(ba)), idx), shape=(m, m))
        ncomp, lab = connected_components(G, directed=False)
        vc = vchart[verts]
        lo = np.full(ncomp, np.iinfo(np.int64).max)
        hi = np.full(ncomp, np.iinfo(np.int64).min)
        np.minimum.at(lo, lab, vc)
        np.maximum.at(hi, lab, vc)
        if (lo == hi).all():
            np.add.at(loops, lo, 1)
        else:
            order = np.argsort(bc, kind="stable")   # the reference groups the edges by chart
            p, find = _components(ba[order], bb[order], nv)
            for v in verts.tolist():
                if find(v) == v:
                    loops[vchart[v]] += 1
    return chi, loops, ba, bb, bc


# ------------------------------------------------------------------ GPU relaxation of a face subset
class Solver:
    """Drop-in for engine/hier.py:357-593: ``relax`` runs ARAP on any subset
    of a mesh's charts, ``lscm`` maps every chart at once, ``bad_fraction``
    reports the last relax's distortion.

    ``relax`` lays the charts out as one device batch (islands = charts, in
    chart order, each chart's UV vertices in id order) and runs the batch
    kernels: orientation (uva_orient_positive), flip repair
    (uva_repair_flips) before, halfway and after, and ARAP iterations
    (uva_arap) with the reference's step rule, the flip-safe step
    min(1, 0.9 t_max) except for charts that are folded at the start of the
    iteration, which take the full step (``fold_step``). As in the drop-in
    ``gpu.Batch``, each global step is solved per chart to a 2e-7 relative
    residual checked in FP64, where the reference runs ``cg_iters`` (20)
    Jacobi-CG iterations on the whole subset in FP32; ``cg_iters`` is kept
    for signature compatibility. ``lscm`` assembles the reference's
    soft-pinned LSCM system on the device (uva_hier_lscm: weights, pins,
    unknowns grouped by chart, CSR) and solves it with the FP64 Jacobi-PCG
    kernel, one CTA per chart, to a 1e-10 relative residual per chart, where
    the reference stops its FP32 CG on the whole system at 1e-6 or 600
    iterations.
    """

    def __init__(self, topo, dev=None):
        from ..device import require_cuda
        self.dev = require_cuda(dev)
        self.V = np.asarray(topo.V, np.float64)
        self.F = np.asarray(topo.F, np.int64)
        self._q = None

    # ---------------------------------------------------------------- layout
    def _layout(self, faces, CV, nv, chart, nchart):
        """Charts as batch islands: (order, P, T_local, vofs, tofs, forder)
        with order = the UV vertices in batch order and forder = the faces in
        batch order."""
        faces = np.asarray(faces, np.int64)
        CV = np.asarray(CV, np.int64).reshape(-1, 3)
        chart = np.asarray(chart, np.int64)
        n = len(faces)
        if n and (CV.min() < 0 or CV.max() >= nv or chart.min() < 0 or chart.max() >= nchart):
            raise ValueError("hier.Solver: CV or chart out of range")
        vchart = -np.ones(nv, np.int64)
        if n:   # any naming face's chart: the check below rejects vertices named by two charts
            vchart[CV.reshape(-1)] = np.repeat(chart, 3)
        if n and (vchart[CV] != chart[:, None]).any():
            raise ValueError("hier.Solver: a UV vertex is shared by faces of different charts")
        used = np.nonzero(vchart >= 0)[0]
        order = used[np.argsort(vchart[used], kind="stable")]           # by chart, then id
        newid = -np.ones(nv, np.int64)
        newid[order] = np.arange(len(order))
        vofs = np.zeros(nchart + 1, np.int64)
        np.cumsum(np.bincount(vchart[used], minlength=nchart), out=vofs[1:])
        forder = np.argsort(chart, kind="stable")
        tofs = np.zeros(nchart + 1, np.int64)
        np.cumsum(np.bincount(chart, minlength=nchart), out=tofs[1:])
        Tb = newid[CV[forder]]
        T_local = Tb - vofs[chart[forder]][:, None]
        corner = np.empty(nv, np.int64)   # a corner naming each UV vertex (the last one)
        corner[CV.reshape(-1)] = np.arange(3 * n)
        c = corner[order]
        P = self.V[self.F[faces[c // 3], c % 3]]
        return order, P, T_local, vofs, tofs, forder

    # ---------------------------------------------------------------- relax
    def relax(self, faces, CV, nv, chart, nchart, U0, iters=6, cg_iters=20, repair_rounds=24):
        """faces (n,) global ids, CV (n,3) local vertex ids, chart (n,) local
        chart ids, U0 (nv,2) initial UVs -> (U (nv,2) float64, flips per
        chart, UV / 3D area scale per chart) (engine/hier.py:389-509)."""
        import torch
        from .. import _lib
        from ..device import DeviceBatch
        nv, nchart = int(nv), int(nchart)
        U0 = np.asarray(U0, np.float64).reshape(-1, 2)
        order, P, T_local, vofs, tofs, forder = self._layout(faces, CV, nv, chart, nchart)
        out = U0.copy()
        flips = np.zeros(nchart)
        scale = np.zeros(nchart)
        if len(order) == 0 or len(T_local) == 0:
            self._q = None
            return out, flips, scale
        db = DeviceBatch(P, T_local, vofs, tofs, U=U0[order], semantics=_lib.SEM_BATCH, device=self.dev)
        db.orient_positive()
        db.repair_flips(repair_rounds)
        first = min(int(iters), int(iters) // 2 + 1)
        if first > 0:
            db.arap(iters=first, line_search=True, fold_step=True)
            db.repair_flips(repair_rounds)           # after iteration iters // 2
        if int(iters) - first > 0:
            db.arap(iters=int(iters) - first, line_search=True, fold_step=True)
        db.repair_flips(repair_rounds)
        # per-chart quality (engine/hier.py:493-508)
        sa = db.signed_area().cpu().numpy()
        J = db.jacobians().cpu().numpy()
        area = db.frame[:db.t, 3].cpu().numpy()
        ok = (db.wtri[:db.t, 3] != 0).cpu().numpy()
        ct = np.repeat(np.arange(nchart), np.diff(tofs))
        j00, j01, j10, j11 = J[:, 0], J[:, 1], J[:, 2], J[:, 3]
        E = (j00 + j11) / 2; Fq = (j00 - j11) / 2; G = (j10 + j01) / 2; H = (j10 - j01) / 2
        Q = np.sqrt(E * E + H * H); R = np.sqrt(Fq * Fq + G * G)
        s1 = Q + R; s2 = np.abs(Q - R)
        ar3 = area * ok
        uva = np.bincount(ct, np.abs(sa) * ok, nchart)
        a3 = np.bincount(ct, ar3, nchart)
        scale = uva / np.maximum(a3, 1e-30)
        with np.errstate(divide="ignore", invalid="ignore"):
            aniso = s1 / np.maximum(s2, 1e-12)
            arat = (s1 * s2) / np.maximum(scale[ct], 1e-30)
        flips = np.bincount(ct, ((sa < 0) & ok).astype(np.float64), nchart)
        self._q = (aniso, arat, ar3, ct, nchart, a3)
        out[order] = db.uvs()
        torch.cuda.current_stream(self.dev).synchronize()
        return out, flips, scale

    def bad_fraction(self, max_aniso, max_area):
        """Area fractions of each chart above the anisotropy / area-ratio
        limits in the last relax (engine/hier.py:585-591)."""
        if self._q is None:
            return np.zeros(0), np.zeros(0)
        aniso, arat, ar3, ct, nchart, a3 = self._q
        badA = np.bincount(ct, ar3 * (aniso > max_aniso), nchart)
        badR = np.bincount(ct, ar3 * ((arat > max_area) | (arat < 1.0 / max_area)), nchart)
        return badA / np.maximum(a3, 1e-30), badR / np.maximum(a3, 1e-30)

    # ---------------------------------------------------------------- lscm
    def lscm(self, faces, CV, nv, chart, nchart, U0, ba, bb, iters=600):
        """Free-boundary conformal map of every chart at once: the LSCM energy
        with two soft pins per chart, the boundary vertices of smallest and
        largest initial u (engine/hier.py:534-585). The system is assembled
        and solved on the device (uva_hier_lscm); ``iters`` is accepted for
        signature compatibility (see the class docstring)."""
        import ctypes as C
        import torch
        from .. import _lib
        nv, nchart = int(nv), int(nchart)
        faces = np.asarray(faces, np.int64).reshape(-1)
        CV = np.asarray(CV, np.int64).reshape(-1, 3)
        chart = np.asarray(chart, np.int64).reshape(-1)
        U0 = np.ascontiguousarray(np.asarray(U0, np.float64).reshape(-1, 2))
        ba = np.asarray(ba, np.int64).reshape(-1); bb = np.asarray(bb, np.int64).reshape(-1)
        if nv == 0:
            return U0.copy()
        t, nb = len(faces), len(ba)
        if len(CV) != t or len(chart) != t or len(bb) != nb or len(U0) != nv:
            raise ValueError("hier.Solver.lscm: faces, CV, chart, ba / bb or U0 of inconsistent lengths")
        for name, a, hi in (("faces", faces, len(self.F)), ("CV", CV, nv), ("ba", ba, nv), ("bb", bb, nv)):
            if a.size and (a.min() < -hi or a.max() >= hi):
                raise IndexError(f"hier.Solver.lscm: {name} out of range")
        # negative indices count from the end, as numpy indexing does
        faces = np.where(faces < 0, faces + len(self.F), faces)
        CV = np.where(CV < 0, CV + nv, CV)
        ba = np.where(ba < 0, ba + nv, ba); bb = np.where(bb < 0, bb + nv, bb)
        d = self.dev
        Vd, Fd = self._mesh_on_device()
        up = lambda a, dt: torch.from_numpy(np.ascontiguousarray(a, dt)).to(d)
        fd, cvd, chd = up(faces, np.int32), up(CV, np.int32), up(chart, np.int32)
        bad, bbd, u0d = up(ba, np.int32), up(bb, np.int32), up(U0, np.float64)
        L = _lib.lib()
        nbytes = C.c_int64()
        _lib.check(L.uva_hier_lscm_scratch_bytes(nv, t, nb, nchart, C.byref(nbytes)), "uva_hier_lscm_scratch_bytes")
        scratch = torch.empty(max(int(nbytes.value), 1), dtype=torch.uint8, device=d)
        out = torch.empty((nv, 2), dtype=torch.float64, device=d)
        flags = torch.empty(1, dtype=torch.int32, device=d)
        st = torch.cuda.current_stream(d)
        maxiter = max(20000, 40 * int(np.sqrt(2 * nv)))   # 2 nv bounds the unknowns (the used ones are counted on the device)
        _lib.check(L.uva_hier_lscm(Vd.data_ptr(), len(self.V), Fd.data_ptr(), len(self.F), fd.data_ptr(),
                                   cvd.data_ptr(), chd.data_ptr(), t, nv, nchart, u0d.data_ptr(), bad.data_ptr(),
                                   bbd.data_ptr(), nb, 1e-10, maxiter, scratch.data_ptr(), int(nbytes.value),
                                   out.data_ptr(), flags.data_ptr(), C.c_void_p(st.cuda_stream)), "uva_hier_lscm")
        U = out.cpu().numpy()
        f = int(flags.item())
        if f & 6:
            raise ValueError("hier.Solver.lscm: a mesh face index or chart id out of range")
        if f & 1:
            raise ValueError("hier.Solver.lscm: a UV vertex is shared by faces of different charts")
        return U

    def _mesh_on_device(self):
        """The mesh's positions (FP64) and faces (int32) on the device, once."""
        import torch
        if getattr(self, "_dmesh", None) is None:
            if len(self.F) and (self.F.min() < 0 or self.F.max() >= len(self.V)):
                raise IndexError("hier.Solver: mesh faces out of range")
            self._dmesh = (torch.from_numpy(np.ascontiguousarray(self.V)).to(self.dev),
                           torch.from_numpy(np.ascontiguousarray(self.F, np.int32)).to(self.dev))
        return self._dmesh
