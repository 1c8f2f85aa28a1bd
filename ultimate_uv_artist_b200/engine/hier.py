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


def _boundary_corners(F, FF, faces, loc, chart, CV):
    """isb (n, 3): corner edge k of local face i is a boundary edge unless the
    neighbour across it (FF) is a face of the same chart whose corner on the
    shared vertex F[f, k] (its first match) has the same UV vertex
    (engine/hier.py:275-291)."""
    F = np.asarray(F, np.int64)
    FF = np.asarray(FF, np.int64)
    faces = np.asarray(faces, np.int64)
    loc = np.asarray(loc, np.int64)
    chart = np.asarray(chart, np.int64)
    CV = np.asarray(CV, np.int64).reshape(-1, 3)
    n = len(faces)
    if n == 0:
        return np.zeros((0, 3), bool)
    g = FF[faces]                                   # (n, 3) neighbour faces
    gs = np.where(g >= 0, g, 0)
    j = np.where(g >= 0, loc[gs], -1)               # their local indices
    js = np.where(j >= 0, j, 0)
    same = (j >= 0) & (chart[js] == chart[:, None])
    a = F[faces]                                    # (n, 3) corner vertices
    match = F[gs] == a[:, :, None]                  # (n, 3, 3): F[g, kk] == F[f, k]
    has = match.any(2)
    kk = match.argmax(2)                            # first matching corner of g
    cvj = CV[js, kk]
    interior = same & has & (cvj == CV)
    return ~interior


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
    chi, loops, ba, bb, bc = chart_topology(F, FF, faces, loc, chart, CV, nchart, nv)
    collide = _collide(UV, ba, bb, bc, int(nchart))
    return collide, chi, loops


def chart_topology(F, FF, faces, loc, chart, CV, nchart, nv):
    """The host half of chart_checks: (chi, loops, ba, bb, bc) with the
    boundary edges ba -> bb of chart bc in face order."""
    CV = np.asarray(CV, np.int64).reshape(-1, 3)
    chart = np.asarray(chart, np.int64)
    nchart, nv = int(nchart), int(nv)
    n = len(CV)
    isb = _boundary_corners(F, FF, faces, loc, chart, CV)
    Fc = np.bincount(chart, minlength=nchart).astype(np.int64) if n else np.zeros(nchart, np.int64)
    nb_c = np.bincount(chart, weights=isb.sum(1), minlength=nchart).astype(np.int64) if n else np.zeros(nchart, np.int64)
    # vchart[v]: chart of the last corner (face order) that names v
    flat = CV.reshape(-1)
    vchart = -np.ones(nv, np.int64)
    if n:
        rev = flat[::-1]
        uniq, first = np.unique(rev, return_index=True)
        vchart[uniq] = np.repeat(chart, 3)[::-1][first]
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
