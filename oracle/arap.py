"""Oracle for the ARAP / LSCM path (test infrastructure only, see package doc).

Two semantics are restated, because the reference has two solvers:

* ``BatchRef`` restates ``engine/gpu.py`` ``Batch`` (batched, block-diagonal,
  soft pin on the first vertex of every chart with one global pin weight,
  per-chart flip-safe line search, non-finite charts revert) but solves every
  global step EXACTLY (sparse LU in FP64) instead of running 40 CG iterations.
  It is the FP64 oracle the batched CUDA solver is measured against.
* ``param_*`` functions restate ``engine/param.py`` (per chart, exact LU,
  per-chart pin weight, relative-energy stop, hard-pinned LSCM).
"""
from __future__ import annotations

import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as spla


# ====================================================================== Batch
def batch_frames(P, T):
    """Isometric frames, areas, validity mask and half-cotangent weights.
    Restates engine/gpu.py:88-121 (FP64)."""
    p0, p1, p2 = P[T[:, 0]], P[T[:, 1]], P[T[:, 2]]
    e1 = p1 - p0
    e2 = p2 - p0
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
    w = np.empty((len(T), 3))
    for k in range(3):
        i, j, o = (k + 1) % 3, (k + 2) % 3, k
        a = X[:, i] - X[:, o]
        b = X[:, j] - X[:, o]
        cr = np.maximum(np.abs(a[:, 0] * b[:, 1] - a[:, 1] * b[:, 0]), 1e-30)
        w[:, k] = 0.5 * np.clip((a * b).sum(1) / cr, -1e4, 1e4)
    w[~ok] = 0.0
    x1 = np.maximum(X[:, 1, 0], 1e-30)
    x2 = X[:, 2, 0].copy()
    y2 = np.where(np.abs(X[:, 2, 1]) > 1e-30, X[:, 2, 1], 1e-30)
    return {"X": X, "area": 0.5 * dbl, "ok": ok, "w": w, "x1": x1, "x2": x2, "y2": y2}


class BatchRef:
    """FP64 restatement of engine/gpu.py:66-299 with exact global solves."""

    def __init__(self, charts, wpin=None):
        """``wpin`` overrides the soft-pin weight (the reference takes the max
        |w| of the whole batch; a sub-batch checked against a larger batch
        passes that batch's value)."""
        self._wpin_override = wpin
        P, T, U, cv, ct = [], [], [], [], []
        off = 0
        for i, (p, t, u) in enumerate(charts):
            P.append(np.asarray(p, np.float64))
            U.append(np.asarray(u, np.float64))
            T.append(np.asarray(t, np.int64) + off)
            cv.append(np.full(len(p), i, np.int64))
            ct.append(np.full(len(t), i, np.int64))
            off += len(p)
        self.nc = len(charts)
        self.offsets = np.cumsum([0] + [len(p) for p, _, _ in charts])
        self.n = off
        self.P = np.concatenate(P)
        self.T = np.concatenate(T)
        self.U = np.concatenate(U)
        self.cv = np.concatenate(cv)
        self.ct = np.concatenate(ct)
        fr = batch_frames(self.P, self.T)
        self.X, self.area, self.ok, self.w = fr["X"], fr["area"], fr["ok"], fr["w"]
        self.x1, self.x2, self.y2 = fr["x1"], fr["x2"], fr["y2"]
        self.scale = np.ones(len(self.T))
        self._build_laplacian()

    def _build_laplacian(self):
        """engine/gpu.py:126-142: cotangent Laplacian summed over unique edges,
        soft pin (weight = global max |w|) on the first vertex of each chart."""
        T, w, n = self.T, self.w, self.n
        a = np.concatenate([T[:, 1], T[:, 2], T[:, 0]])
        b = np.concatenate([T[:, 2], T[:, 0], T[:, 1]])
        W = np.concatenate([w[:, 0], w[:, 1], w[:, 2]])
        key = np.minimum(a, b) * n + np.maximum(a, b)
        uk, inv = np.unique(key, return_inverse=True)
        wsum = np.bincount(inv, weights=W, minlength=len(uk))
        ea, eb = uk // n, uk % n
        self.edges = (ea, eb, np.bincount(inv, minlength=len(uk)))
        diag = np.bincount(ea, weights=wsum, minlength=n) + np.bincount(eb, weights=wsum, minlength=n)
        self.pins = self.offsets[:-1].copy()
        self.wpin = max(float(np.abs(W).max()) if len(W) else 0.0, 1e-12)
        if self._wpin_override is not None:
            self.wpin = float(self._wpin_override)
        diag[self.pins] += self.wpin
        rows = np.concatenate([ea, eb, np.arange(n)])
        cols = np.concatenate([eb, ea, np.arange(n)])
        vals = np.concatenate([-wsum, -wsum, diag])
        self.L = sp.csc_matrix((vals, (rows, cols)), shape=(n, n))
        self.diag = diag
        self._lu = None

    def _solve(self, b):
        if self._lu is None:
            self._lu = spla.splu(self.L, permc_spec="MMD_AT_PLUS_A", options={"SymmetricMode": True})
        return self._lu.solve(b)

    def signed_area(self, U):
        """engine/gpu.py:153-156."""
        a, b, c = U[self.T[:, 0]], U[self.T[:, 1]], U[self.T[:, 2]]
        return 0.5 * ((b[:, 0] - a[:, 0]) * (c[:, 1] - a[:, 1]) - (c[:, 0] - a[:, 0]) * (b[:, 1] - a[:, 1]))

    def jacobians(self, U):
        """engine/gpu.py:145-151."""
        T = self.T
        a0, a1, a2 = U[T[:, 0]], U[T[:, 1]], U[T[:, 2]]
        j00 = (a1[:, 0] - a0[:, 0]) / self.x1
        j10 = (a1[:, 1] - a0[:, 1]) / self.x1
        j01 = ((a2[:, 0] - a0[:, 0]) - j00 * self.x2) / self.y2
        j11 = ((a2[:, 1] - a0[:, 1]) - j10 * self.x2) / self.y2
        return j00, j01, j10, j11

    def flips_per_chart(self, U=None):
        """engine/gpu.py:158-163."""
        U = self.U if U is None else U
        bad = (self.signed_area(U) < 0) & self.ok
        return np.bincount(self.ct, weights=bad.astype(np.float64), minlength=self.nc)

    def rhs(self, U):
        """engine/gpu.py:165-182: closest rotation of the conformal part of J,
        scaled, times the weighted frame edges, scattered to both endpoints;
        plus the soft-pin term."""
        j00, j01, j10, j11 = self.jacobians(U)
        ca = j00 + j11
        cb = j10 - j01
        h = np.hypot(ca, cb)
        good = self.ok & np.isfinite(h) & (h > 0)
        c = np.where(good, ca / np.where(good, h, 1.0), 1.0) * self.scale
        s = np.where(good, cb / np.where(good, h, 1.0), 0.0) * self.scale
        X, T, w = self.X, self.T, self.w
        b = np.zeros((self.n, 2))
        for k in range(3):
            i, j = (k + 1) % 3, (k + 2) % 3
            dx = X[:, i] - X[:, j]
            rx = (c * dx[:, 0] - s * dx[:, 1]) * w[:, k]
            ry = (s * dx[:, 0] + c * dx[:, 1]) * w[:, k]
            np.add.at(b[:, 0], T[:, i], rx); np.add.at(b[:, 1], T[:, i], ry)
            np.add.at(b[:, 0], T[:, j], -rx); np.add.at(b[:, 1], T[:, j], -ry)
        b[self.pins] += self.wpin * U[self.pins]
        return b

    def max_step(self, U, D):
        """engine/gpu.py:204-227: per chart, the smallest positive root of the
        signed-area quadratic over triangles that are positive now."""
        T = self.T
        u0, u1, u2 = U[T[:, 0]], U[T[:, 1]], U[T[:, 2]]
        d0, d1, d2 = D[T[:, 0]], D[T[:, 1]], D[T[:, 2]]
        ux1, uy1 = u1[:, 0] - u0[:, 0], u1[:, 1] - u0[:, 1]
        ux2, uy2 = u2[:, 0] - u0[:, 0], u2[:, 1] - u0[:, 1]
        dx1, dy1 = d1[:, 0] - d0[:, 0], d1[:, 1] - d0[:, 1]
        dx2, dy2 = d2[:, 0] - d0[:, 0], d2[:, 1] - d0[:, 1]
        C = ux1 * uy2 - ux2 * uy1
        B = ux1 * dy2 + dx1 * uy2 - ux2 * dy1 - dx2 * uy1
        A = dx1 * dy2 - dx2 * dy1
        big = np.full_like(C, 1e30)
        with np.errstate(divide="ignore", invalid="ignore"):
            lin = np.where((np.abs(A) < 1e-30) & (B < 0), -C / np.where(B != 0, B, 1.0), big)
            disc = B * B - 4 * A * C
            sq = np.sqrt(np.maximum(disc, 0))
            A2 = np.where(np.abs(A) < 1e-30, 1.0, 2 * A)
            r1 = (-B - sq) / A2
            r2 = (-B + sq) / A2
        quad = np.minimum(np.where(r1 > 0, r1, big), np.where(r2 > 0, r2, big))
        quad = np.where((disc >= 0) & (np.abs(A) >= 1e-30), quad, big)
        t = np.minimum(lin, quad)
        t = np.where(C > 0, t, big)
        out = np.full(self.nc, 1e30)
        np.minimum.at(out, self.ct, t)
        return out

    def arap(self, iters=8, line_search=True):
        """engine/gpu.py:230-249 with the CG replaced by an exact solve."""
        U = self.U
        for _ in range(iters):
            b = self.rhs(U)
            Un = self._solve(b)
            badv = ~np.isfinite(Un).all(1)
            if badv.any():
                badc = np.zeros(self.nc, bool)
                badc[self.cv[badv]] = True
                Un = np.where(badc[self.cv][:, None], U, Un)
            if line_search:
                D = Un - U
                step = np.minimum(0.9 * self.max_step(U, D), 1.0)
                U = U + D * step[self.cv][:, None]
            else:
                U = Un
        self.U = U
        return U

    def repair_flips(self, rounds=60):
        """engine/gpu.py:251-273: Jacobi moves of interior vertices of folded
        triangles to their 1-ring mean (unique-edge neighbours)."""
        ea, eb, cnt = self.edges
        n = self.n
        bnd = np.zeros(n, bool)
        one = cnt == 1
        bnd[ea[one]] = True
        bnd[eb[one]] = True
        A = sp.csr_matrix((np.ones(2 * len(ea)), (np.r_[ea, eb], np.r_[eb, ea])), shape=(n, n))
        deg = np.maximum(np.asarray(A.sum(1)).ravel(), 1)
        U = self.U
        for _ in range(rounds):
            bad = (self.signed_area(U) < 0) & self.ok
            if not bad.any():
                break
            mv = np.zeros(n, bool)
            mv[self.T[bad].reshape(-1)] = True
            mv &= ~bnd
            mean = (A @ U) / deg[:, None]
            U = np.where(mv[:, None], mean, U)
        self.U = U
        return U

    def orient_positive(self):
        """engine/gpu.py:275-281."""
        sa = self.signed_area(self.U)
        s = np.bincount(self.ct, weights=np.sign(sa) * self.area, minlength=self.nc)
        flip = (s < 0)[self.cv]
        self.U = np.where(flip[:, None], self.U * np.array([1.0, -1.0]), self.U)

    def shrink(self, tri_idx, factor=0.6, floor=0.05, rings=3):
        """engine/gpu.py:283-295."""
        if len(tri_idx) == 0:
            return
        mark = np.zeros(self.n, bool)
        sel = np.zeros(len(self.T), bool)
        sel[np.asarray(tri_idx)] = True
        for _ in range(rings):
            mark[self.T[sel].reshape(-1)] = True
            sel = mark[self.T].any(1)
        self.scale = np.where(sel, np.maximum(self.scale * factor, floor), self.scale)

    def chart_uvs(self):
        """engine/gpu.py:297-299."""
        return [self.U[a:b].copy() for a, b in zip(self.offsets[:-1], self.offsets[1:])]

    def residual(self, b, x):
        """FP64 relative residual ||b - L x|| / ||b|| per column, per chart."""
        r = b - self.L @ x
        rn = np.sqrt(np.stack([np.bincount(self.cv, weights=r[:, k] ** 2, minlength=self.nc) for k in range(2)], 1))
        bn = np.sqrt(np.stack([np.bincount(self.cv, weights=b[:, k] ** 2, minlength=self.nc) for k in range(2)], 1))
        return rn / np.maximum(bn, 1e-300)


# ====================================================================== param
def local_frames(P, T):
    """engine/param.py:19-32."""
    p0, p1, p2 = P[T[:, 0]], P[T[:, 1]], P[T[:, 2]]
    e1 = p1 - p0
    e2 = p2 - p0
    l1 = np.linalg.norm(e1, axis=1)
    n = np.cross(e1, e2)
    nn = np.linalg.norm(n, axis=1)
    ex = e1 / np.maximum(l1, 1e-300)[:, None]
    ey = np.cross(n / np.maximum(nn, 1e-300)[:, None], ex)
    X = np.zeros((len(T), 3, 2))
    X[:, 1, 0] = l1
    X[:, 2, 0] = (e2 * ex).sum(1)
    X[:, 2, 1] = (e2 * ey).sum(1)
    return X, 0.5 * nn


def cot_weights(X):
    """engine/param.py:35-44."""
    cots = np.empty((len(X), 3))
    for k in range(3):
        i, j, o = (k + 1) % 3, (k + 2) % 3, k
        a = X[:, i] - X[:, o]
        b = X[:, j] - X[:, o]
        cr = np.abs(a[:, 0] * b[:, 1] - a[:, 1] * b[:, 0])
        cots[:, k] = (a * b).sum(1) / np.maximum(cr, 1e-300)
    return np.clip(cots, -1e4, 1e4)


def lap_triplets(T, cots):
    """engine/param.py:47-51."""
    i = np.concatenate([T[:, 1], T[:, 2], T[:, 0]])
    j = np.concatenate([T[:, 2], T[:, 0], T[:, 1]])
    w = 0.5 * np.concatenate([cots[:, 0], cots[:, 1], cots[:, 2]])
    return np.concatenate([i, j, i, j]), np.concatenate([j, i, i, j]), np.concatenate([-w, -w, w, w])


def boundary_edges_oriented(T):
    """engine/param.py:59-68: directed half-edges whose reverse is absent."""
    a = np.concatenate([T[:, 0], T[:, 1], T[:, 2]])
    b = np.concatenate([T[:, 1], T[:, 2], T[:, 0]])
    n = int(max(a.max(), b.max())) + 1
    has_twin = np.isin(b * n + a, a * n + b)
    return a[~has_twin], b[~has_twin]


def signed_areas(U, T):
    """engine/param.py:97-99."""
    a, b, c = U[T[:, 0]], U[T[:, 1]], U[T[:, 2]]
    return 0.5 * ((b[:, 0] - a[:, 0]) * (c[:, 1] - a[:, 1]) - (c[:, 0] - a[:, 0]) * (b[:, 1] - a[:, 1]))


def far_pair(P, cand):
    """engine/param.py:172-179: boundary vertex farthest from the boundary
    centroid, then the boundary vertex farthest from it."""
    Q = P[cand]
    c = Q.mean(0)
    i = cand[np.argmax(((Q - c) ** 2).sum(1))]
    j = cand[np.argmax(((Q - P[i]) ** 2).sum(1))]
    if i == j:
        j = cand[0] if cand[0] != i else cand[-1]
    return int(i), int(j)


def lscm(P, T, X=None, cots=None, pins=None):
    """engine/param.py:136-169: conformal energy H = [[L, -B], [B, L]] with the
    boundary area term, two hard pins (p0 -> (0,0), p1 -> (|P[p1]-P[p0]|, 0)),
    exact solve of the free unknowns."""
    P = np.asarray(P, np.float64)
    T = np.asarray(T, np.int64)
    n = len(P)
    if X is None:
        X, _ = local_frames(P, T)
    if cots is None:
        cots = cot_weights(X)
    bi, bj = boundary_edges_oriented(T)
    if len(bi) == 0:
        raise ValueError("chart has no boundary (closed surface): needs a cut")
    I, J, W = lap_triplets(T, cots)
    hb = np.full(len(bi), 0.5)
    rows = np.concatenate([I, I + n, bi, bj, bi + n, bj + n])
    cols = np.concatenate([J, J + n, bj + n, bi + n, bj, bi])
    vals = np.concatenate([W, W, -hb, hb, hb, -hb])
    if pins is None:
        pins = far_pair(P, np.unique(bi))
    p0, p1 = pins
    d = np.linalg.norm(P[p1] - P[p0])
    pin_idx = np.array([p0, p1, p0 + n, p1 + n])
    pin_val = np.zeros(2 * n)
    pin_val[p1] = d
    keep = np.ones(2 * n, bool)
    keep[pin_idx] = False
    newid = np.full(2 * n, -1)
    newid[keep] = np.arange(int(keep.sum()))
    rf = newid[rows]
    cf = newid[cols]
    both = (rf >= 0) & (cf >= 0)
    nf = int(keep.sum())
    Hff = sp.csc_matrix((vals[both], (rf[both], cf[both])), shape=(nf, nf))
    pc = (rf >= 0) & (cf < 0)
    rhs = -np.bincount(rf[pc], weights=vals[pc] * pin_val[cols[pc]], minlength=nf)
    sol = spla.splu(Hff, permc_spec="MMD_AT_PLUS_A", options={"SymmetricMode": True}).solve(rhs)
    x = pin_val.copy()
    x[keep] = sol
    return np.stack([x[:n], x[n:]], 1)


def lscm_batch(P, T, X, cots):
    """LSCM of one chart with explicit weights (used for batched parity where
    the weights follow the Batch frame rules)."""
    return lscm(P, T, X=X, cots=cots)


def arap_rotations(U, T, X):
    """engine/param.py:206-233 (mode 0): closest rotation from the conformal
    part of J; identity for frame-less or zero-Jacobian triangles."""
    x1 = X[:, 1, 0]; x2 = X[:, 2, 0]; y2 = X[:, 2, 1]
    du1 = U[T[:, 1]] - U[T[:, 0]]
    du2 = U[T[:, 2]] - U[T[:, 0]]
    good = np.abs(x1 * y2) >= 1e-300
    x1s = np.where(good, x1, 1.0); y2s = np.where(good, y2, 1.0)
    j00 = du1[:, 0] / x1s; j10 = du1[:, 1] / x1s
    j01 = (du2[:, 0] - j00 * x2) / y2s; j11 = (du2[:, 1] - j10 * x2) / y2s
    ca = j00 + j11; cb = j10 - j01
    h = np.sqrt(ca * ca + cb * cb)
    small = h < 1e-300
    ca = np.where(small, 1.0, ca); cb = np.where(small, 0.0, cb); h = np.where(small, 1.0, h)
    R = np.empty((len(T), 2, 2))
    R[:, 0, 0] = ca / h; R[:, 0, 1] = -cb / h; R[:, 1, 0] = cb / h; R[:, 1, 1] = ca / h
    R[~good] = np.eye(2)
    return R


def arap_rhs(n, T, X, cots, R):
    """engine/param.py:457-474."""
    b = np.zeros((n, 2))
    for k in range(3):
        ii, jj = (k + 1) % 3, (k + 2) % 3
        w = 0.5 * cots[:, k]
        dx = X[:, ii] - X[:, jj]
        rx = R[:, 0, 0] * dx[:, 0] + R[:, 0, 1] * dx[:, 1]
        ry = R[:, 1, 0] * dx[:, 0] + R[:, 1, 1] * dx[:, 1]
        np.add.at(b[:, 0], T[:, ii], w * rx); np.add.at(b[:, 1], T[:, ii], w * ry)
        np.add.at(b[:, 0], T[:, jj], -w * rx); np.add.at(b[:, 1], T[:, jj], -w * ry)
    return b


def max_step_param(U, D, T):
    """engine/param.py:259-291 (serial semantics, vectorised)."""
    a, b, c = T[:, 0], T[:, 1], T[:, 2]
    ux1 = U[b, 0] - U[a, 0]; uy1 = U[b, 1] - U[a, 1]
    ux2 = U[c, 0] - U[a, 0]; uy2 = U[c, 1] - U[a, 1]
    dx1 = D[b, 0] - D[a, 0]; dy1 = D[b, 1] - D[a, 1]
    dx2 = D[c, 0] - D[a, 0]; dy2 = D[c, 1] - D[a, 1]
    C = ux1 * uy2 - ux2 * uy1
    Bq = ux1 * dy2 + dx1 * uy2 - ux2 * dy1 - dx2 * uy1
    A = dx1 * dy2 - dx2 * dy1
    tmax = 1e30
    pos = C > 0
    lin = pos & ((A == 0.0) | (np.abs(A) < 1e-30 * np.maximum(np.abs(Bq), 1e-300)))
    with np.errstate(divide="ignore", invalid="ignore"):
        rl = np.where(lin & (Bq < 0), -C / np.where(Bq != 0, Bq, 1.0), np.inf)
        quad = pos & ~lin
        disc = Bq * Bq - 4 * A * C
        quad &= disc >= 0
        sq = np.sqrt(np.where(quad, disc, 0.0))
        A2 = np.where(quad, 2 * A, 1.0)
        r1 = (-Bq - sq) / A2; r2 = (-Bq + sq) / A2
    r1 = np.where(quad & (r1 > 0), r1, np.inf)
    r2 = np.where(quad & (r2 > 0), r2, np.inf)
    m = min(float(rl.min(initial=np.inf)), float(r1.min(initial=np.inf)), float(r2.min(initial=np.inf)))
    return min(tmax, m)


def energy(U, T, X, area, kind):
    """engine/param.py:294-319."""
    x1 = X[:, 1, 0]; x2 = X[:, 2, 0]; y2 = X[:, 2, 1]
    good = np.abs(x1 * y2) >= 1e-300
    x1s = np.where(good, x1, 1.0); y2s = np.where(good, y2, 1.0)
    du1 = U[T[:, 1]] - U[T[:, 0]]
    du2 = U[T[:, 2]] - U[T[:, 0]]
    j00 = du1[:, 0] / x1s; j10 = du1[:, 1] / x1s
    j01 = (du2[:, 0] - j00 * x2) / y2s; j11 = (du2[:, 1] - j10 * x2) / y2s
    if kind == 0:
        qe = 0.5 * (j00 + j11); qh = 0.5 * (j10 - j01)
        rf = 0.5 * (j00 - j11); rg = 0.5 * (j10 + j01)
        q = np.sqrt(qe * qe + qh * qh); r = np.sqrt(rf * rf + rg * rg)
        e = area * ((q + r - 1) ** 2 + (q - r - 1) ** 2)
    else:
        dj = j00 * j11 - j01 * j10
        fro = j00 * j00 + j01 * j01 + j10 * j10 + j11 * j11
        with np.errstate(divide="ignore", invalid="ignore"):
            e = np.where(dj <= 0, np.inf, area * (fro + fro / (dj * dj) - 4.0))
    return float(np.where(good, e, 0.0).sum())


def refine_arap(P, T, U, iters=10, line_search=True, tol=1e-5, pin=None):
    """engine/param.py:379-414 (method='arap'): soft pin (per-chart weight
    max |W|), exact LU, flip-safe line search when the start is flip-free,
    relative-energy stop."""
    P = np.asarray(P, np.float64); T = np.asarray(T, np.int64); U = np.asarray(U, np.float64)
    n = len(P)
    X, area = local_frames(P, T)
    cots = cot_weights(X)
    flips0 = int((signed_areas(U, T) <= 0).sum())
    use_ls = line_search and flips0 == 0
    pin = 0 if pin is None else pin
    I, J, W = lap_triplets(T, cots)
    wpin = float(np.abs(W).max()) if len(W) else 1.0
    L = sp.csc_matrix((np.r_[W, wpin], (np.r_[I, pin], np.r_[J, pin])), shape=(n, n))
    lu = spla.splu(L, permc_spec="MMD_AT_PLUS_A", options={"SymmetricMode": True})
    prev = energy(U, T, X, area, 0)
    for _ in range(iters):
        R = arap_rotations(U, T, X)
        b = arap_rhs(n, T, X, cots, R)
        b[pin] += wpin * U[pin]
        Un = lu.solve(b)
        if use_ls:
            D = Un - U
            step = min(1.0, 0.9 * max_step_param(U, D, T))
            Un = U + step * D
        e = energy(Un, T, X, area, 0)
        U = Un
        if abs(prev - e) <= tol * max(prev, 1e-300):
            break
        prev = e
    return U


def slim_local(U, T, X):
    """engine/param.py:206-256 (mode 1): per triangle the signed SVD of the
    Jacobian J = U_f M^-1 (numpy svd, last singular value negated when
    det(U V^T) < 0), the rotation U V^T and the SLIM weights
    W = U diag(w) U^T with w = sqrt((s - s^-3) / (s - 1)) of |s| clamped at
    1e-8 (2 when |s - 1| < 1e-6). Frame-less triangles get R = W = I."""
    t = len(T)
    x1 = X[:, 1, 0]; x2 = X[:, 2, 0]; y2 = X[:, 2, 1]
    good = np.abs(x1 * y2) >= 1e-300
    x1s = np.where(good, x1, 1.0); y2s = np.where(good, y2, 1.0)
    du1 = U[T[:, 1]] - U[T[:, 0]]
    du2 = U[T[:, 2]] - U[T[:, 0]]
    j00 = du1[:, 0] / x1s; j10 = du1[:, 1] / x1s
    j01 = (du2[:, 0] - j00 * x2) / y2s; j11 = (du2[:, 1] - j10 * x2) / y2s
    J = np.stack([np.stack([j00, j01], 1), np.stack([j10, j11], 1)], 1)
    Us, S, Vt = np.linalg.svd(J)
    neg = np.linalg.det(Us @ Vt) < 0
    Us[neg, :, 1] *= -1.0
    S[neg, 1] *= -1.0
    R = Us @ Vt
    s = np.maximum(np.abs(S), 1e-8)
    with np.errstate(divide="ignore", invalid="ignore"):
        w = np.where(np.abs(s - 1.0) < 1e-6, 2.0, np.sqrt(np.maximum((s - s ** -3) / (s - 1.0), 1e-12)))
    W = np.einsum("tij,tj,tkj->tik", Us, w, Us)
    eye = np.broadcast_to(np.eye(2), (t, 2, 2))
    R = np.where(good[:, None, None], R, eye)
    W = np.where(good[:, None, None], W, eye)
    return R, W


def slim_system(n, T, X, area, R, W):
    """engine/param.py:341-377: rows sqrt(area) (W (J - R)) over the 2n
    unknowns [u; v]; returns A (4t x 2n) and b."""
    t = len(T)
    x1 = X[:, 1, 0]; x2 = X[:, 2, 0]; y2 = X[:, 2, 1]
    G = np.zeros((t, 2, 3))
    G[:, 0, 0] = -1 / x1; G[:, 0, 1] = 1 / x1
    G[:, 1, 0] = (-1 + x2 / x1) / y2; G[:, 1, 1] = (-x2 / x1) / y2; G[:, 1, 2] = 1 / y2
    sq = np.sqrt(area)
    WR = W @ R
    rows, cols, vals, rhs = [], [], [], []
    for si in range(2):
        for c in range(2):
            r0 = (2 * si + c) * t + np.arange(t)
            for comp in range(2):
                for k in range(3):
                    rows.append(r0); cols.append(T[:, k] + comp * n)
                    vals.append(sq * W[:, si, comp] * G[:, c, k])
            rhs.append(sq * WR[:, si, c])
    A = sp.csr_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))), shape=(4 * t, 2 * n))
    return A, np.concatenate(rhs)


def refine_slim(P, T, U, iters=10, tol=1e-5):
    """engine/param.py:415-454 (method='slim'), exact solves: normal
    equations (A^T A + 1e-12 sum(area) I) x = A^T b + 1e-12 sum(area) x0,
    flip-safe step min(1, 0.9 tmax), halving up to 12 times while the
    symmetric Dirichlet energy is not below the previous one, relative-energy
    stop. A start with an inverted triangle is returned unchanged."""
    P = np.asarray(P, np.float64); T = np.asarray(T, np.int64); U = np.asarray(U, np.float64).copy()
    n = len(P)
    X, area = local_frames(P, T)
    prev = energy(U, T, X, area, 1)
    if not np.isfinite(prev):
        return U
    reg = 1e-12 * area.sum()
    for _ in range(iters):
        R, W = slim_local(U, T, X)
        A, b = slim_system(n, T, X, area, R, W)
        M = (A.T @ A).tocsc() + sp.identity(2 * n, format="csc") * reg
        x0 = np.r_[U[:, 0], U[:, 1]]
        x = spla.spsolve(M, A.T @ b + reg * x0)
        D = np.stack([x[:n], x[n:]], 1) - U
        step = min(1.0, 0.9 * max_step_param(U, D, T))
        e = energy(U + step * D, T, X, area, 1)
        k = 0
        while (not np.isfinite(e) or e > prev) and k < 12:
            step *= 0.5
            e = energy(U + step * D, T, X, area, 1)
            k += 1
        if not np.isfinite(e) or e > prev:
            break
        U = U + step * D
        if abs(prev - e) <= tol * prev:
            break
        prev = e
    return U


def repair_flips_param(U, T, rounds=60):
    """engine/param.py:477-516: Gauss-Seidel 1-ring moves in triangle order."""
    U = np.array(U, np.float64, copy=True)
    T = np.asarray(T, np.int64)
    n = len(U)
    I = np.concatenate([T[:, 0], T[:, 1], T[:, 2], T[:, 1], T[:, 2], T[:, 0]])
    J = np.concatenate([T[:, 1], T[:, 2], T[:, 0], T[:, 0], T[:, 1], T[:, 2]])
    key = np.unique(I * n + J)
    I, J = key // n, key % n
    ptr = np.zeros(n + 1, np.int64)
    np.add.at(ptr, I + 1, 1)
    ptr = np.cumsum(ptr)
    bi, bj = boundary_edges_oriented(T)
    is_bnd = np.zeros(n, bool); is_bnd[bi] = True; is_bnd[bj] = True
    nb = [J[ptr[v]:ptr[v + 1]].tolist() for v in range(n)]
    Tl = T.tolist()
    for _ in range(rounds):
        bad = 0
        for (a, b, c) in Tl:
            ar = (U[b, 0] - U[a, 0]) * (U[c, 1] - U[a, 1]) - (U[c, 0] - U[a, 0]) * (U[b, 1] - U[a, 1])
            if ar > 0:
                continue
            bad += 1
            for v in (a, b, c):
                if is_bnd[v]:
                    continue
                lst = nb[v]
                if lst:
                    sx = 0.0; sy = 0.0
                    for q in lst:
                        sx += U[q, 0]; sy += U[q, 1]
                    U[v, 0] = sx / len(lst); U[v, 1] = sy / len(lst)
        if bad == 0:
            break
    return U


# ====================================================================== helpers
def chart_quality(P, T, U):
    """engine/param.py:519-551: flips against the majority orientation, the
    closed-form singular values s1 >= s2 of each triangle's Jacobian,
    anisotropy s1 / s2 and area ratio s1 s2 / scale with its area-weighted
    p95 (argsort, cumulative weights, first index reaching 0.95 of the total)
    and means, stretch and scale."""
    P = np.asarray(P, np.float64)
    U = np.asarray(U, np.float64)
    T = np.asarray(T, np.int64)
    X, area = local_frames(P, T)
    sa = signed_areas(U, T)
    A = area.sum()
    npos, nneg = int((sa > 0).sum()), int((sa < 0).sum())
    flips = int((sa <= 0).sum()) if npos >= nneg else int((sa >= 0).sum())
    x1, x2, y2 = X[:, 1, 0], X[:, 2, 0], X[:, 2, 1]
    ok = np.abs(x1 * y2) > 1e-300
    x1s, y2s = np.where(ok, x1, 1.0), np.where(ok, y2, 1.0)
    d1 = U[T[:, 1]] - U[T[:, 0]]
    d2 = U[T[:, 2]] - U[T[:, 0]]
    j00, j10 = d1[:, 0] / x1s, d1[:, 1] / x1s
    j01, j11 = (d2[:, 0] - j00 * x2) / y2s, (d2[:, 1] - j10 * x2) / y2s
    q = np.sqrt(((j00 + j11) / 2) ** 2 + ((j10 - j01) / 2) ** 2)
    r = np.sqrt(((j00 - j11) / 2) ** 2 + ((j10 + j01) / 2) ** 2)
    s1, s2 = q + r, np.abs(q - r)
    sc = np.abs(sa).sum() / max(A, 1e-300)
    w = area / max(A, 1e-300)
    an = s1 / np.maximum(s2, 1e-12)
    ar = s1 * s2 / max(sc, 1e-300)
    lar = np.abs(np.log2(np.maximum(ar, 1e-12)))

    def p95(x):
        o = np.argsort(x)
        cw = np.cumsum(w[o])
        return float(x[o][min(np.searchsorted(cw, 0.95 * cw[-1]), len(o) - 1)])

    st2 = (s1 ** 2 + s2 ** 2) / 2 / max(sc, 1e-300)
    return {"flips": flips, "aniso_p95": p95(an), "aniso_mean": float((an * w).sum()),
            "area_p95": float(2 ** p95(lar)), "area_logdev": float((lar * w).sum()),
            "stretch": float(np.sqrt((st2 * w).sum())), "scale": float(np.sqrt(sc)),
            "per_tri_aniso": an, "per_tri_area": ar}


def uv_rel_error(U, Uref, offsets):
    """Per chart max |U - Uref| divided by the chart's UV extent; returns the
    max over charts."""
    worst = 0.0
    for a, b in zip(offsets[:-1], offsets[1:]):
        if b <= a:
            continue
        ext = float((Uref[a:b].max(0) - Uref[a:b].min(0)).max())
        err = float(np.abs(U[a:b] - Uref[a:b]).max())
        worst = max(worst, err / max(ext, 1e-300))
    return worst
