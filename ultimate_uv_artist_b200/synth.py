"""Seeded synthetic meshes for the five workloads of the parameterization and
validation path.

No benchmark meshes ship with the reference (its chest / fox / wolf / tree
scans are not public), so every workload here is generated from a seed.
Positions are float32, as a mesh loaded from a GLB would be.

* ``hemisphere_patch``  one 50x50 grid (4,802 triangles) mapped onto a
  hemisphere of radius 1, positions jittered N(0, 0.01).
* ``uneven_islands``    2,000 disk grid patches displaced by 8 Gaussian bumps
  (amplitude U(0, 0.5)); the square grid behind each disk has a triangle count
  drawn log-uniformly from 20 to 20,000, the inscribed digital disk keeps about
  pi/4 of it (about 4.5M triangles in total).
* ``validation_atlas``  5,000 grid-patch islands (about 1M triangles) shelf
  packed on a 4096 atlas with 4-texel padding, with overlaps, folds, mirrored
  islands and out-of-range vertices injected from the seed.
* ``energy_islands``    512 smooth displaced grids of 500 to 50,000 triangles
  with 5 % near-degenerate triangles.
* ``noisy_sphere_charts`` a closed sphere displaced by 3D value noise, cut into
  charts by k-means on vertex normals.
"""
from __future__ import annotations

import numpy as np


# ------------------------------------------------------------------ grids
def _grid_faces(nx, ny, alt=False):
    """Triangles of an (nx x ny)-vertex grid, two per cell, row-major vertices."""
    idx = np.arange(nx * ny, dtype=np.int64).reshape(ny, nx)
    a = idx[:-1, :-1]; b = idx[:-1, 1:]; c = idx[1:, 1:]; d = idx[1:, :-1]
    if alt:
        # alternate the diagonal per cell so the triangulation has no preferred direction
        par = ((np.arange(ny - 1)[:, None] + np.arange(nx - 1)[None, :]) % 2).astype(bool)
        t1 = np.where(par[..., None], np.stack([a, b, c], -1), np.stack([a, b, d], -1))
        t2 = np.where(par[..., None], np.stack([a, c, d], -1), np.stack([b, c, d], -1))
    else:
        t1 = np.stack([a, b, c], -1); t2 = np.stack([a, c, d], -1)
    return np.concatenate([t1.reshape(-1, 3), t2.reshape(-1, 3)])


def _compact(V, F):
    used, inv = np.unique(F, return_inverse=True)
    return V[used], inv.reshape(-1, 3).astype(np.int64)


def hemisphere_patch(seed=1000, n=50, jitter=0.01):
    """n x n grid mapped onto a hemisphere of radius 1 (disk topology)."""
    rng = np.random.default_rng(seed)
    s = np.linspace(-1.0, 1.0, n)
    u, v = np.meshgrid(s, s)
    u = u.ravel(); v = v.ravel()
    # square -> disk (elliptical map), then lift onto the upper hemisphere
    x = u * np.sqrt(1.0 - 0.5 * v * v)
    y = v * np.sqrt(1.0 - 0.5 * u * u)
    z = np.sqrt(np.maximum(1.0 - x * x - y * y, 0.0))
    V = np.stack([x, y, z], 1) + rng.normal(0.0, jitter, (n * n, 3))
    F = _grid_faces(n, n)
    return V.astype(np.float32), F


def disk_patch(rng, target_tris, bumps=8, amp=0.5, extent=1.0):
    """Digital disk of whole grid cells (pinch-free, one boundary loop) cut from
    a square grid holding about ``target_tris`` triangles, z-displaced by a sum
    of Gaussian bumps."""
    cells = max(2, int(round(np.sqrt(max(target_tris, 2) / 2.0))))
    nx = cells + 1
    s = np.linspace(-extent, extent, nx)
    X, Y = np.meshgrid(s, s)
    V = np.stack([X.ravel(), Y.ravel(), np.zeros(nx * nx)], 1)
    F = _grid_faces(nx, nx, alt=True)
    # keep both triangles of every cell whose centre lies in the inscribed circle
    cc = (np.arange(cells) + 0.5) / cells * 2 - 1
    keep_cell = (cc[None, :] ** 2 + cc[:, None] ** 2) <= 1.0
    if keep_cell.sum() < 1:
        keep_cell[cells // 2, cells // 2] = True
    kc = keep_cell.ravel()
    F = F[np.concatenate([kc, kc])]
    c = rng.uniform(-extent, extent, (bumps, 2))
    a = rng.uniform(0.0, amp, bumps)
    sg = rng.uniform(0.15, 0.45, bumps) * extent
    d2 = ((V[:, None, :2] - c[None]) ** 2).sum(-1)
    V[:, 2] = (a[None] * np.exp(-d2 / (2 * sg[None] ** 2))).sum(1)
    V, F = _compact(V, F)
    return V.astype(np.float32), F


def uneven_islands(seed=2000, count=2000, tmin=20, tmax=20000):
    """List of (P, T) disk islands with log-uniform square-grid triangle counts."""
    rng = np.random.default_rng(seed)
    targets = np.exp(rng.uniform(np.log(tmin), np.log(tmax), count))
    return [disk_patch(rng, t) for t in targets]


# ------------------------------------------------------------------ validation atlas
def validation_atlas(seed=3000, islands=5000, tris_per_island=200, atlas=4096, padding=4,
                     overlap_rate=1e-4, fold_rate=1e-5, mirrored=3, outside=20):
    """UV atlas of grid-patch islands, shelf packed, with injected faults.

    Returns (V (n,3) f32, F (m,3) i64, UV (n,2) f32, info dict).
    Fault injection (all from the seed):
    * overlaps: each island is shifted by U(0, 8) texels with probability
      ``overlap_rate`` per triangle of the island (so about rate*m islands);
    * folds: one vertex of a triangle reflected across its opposite edge, at
      ``fold_rate`` per triangle;
    * ``mirrored`` islands mirrored u -> 1 - u inside their bounding box;
    * ``outside`` vertices near the atlas border pushed 1-4 texels outside [0, 1].
    """
    rng = np.random.default_rng(seed)
    side = max(2, int(round(np.sqrt(tris_per_island / 2.0))))
    Vs, Fs, Us = [], [], []
    # island footprint in texels (square-ish, varied)
    sizes = rng.uniform(0.6, 1.4, islands)
    off = 0
    for i in range(islands):
        nx = side + 1
        s = np.linspace(0.0, 1.0, nx)
        X, Y = np.meshgrid(s, s)
        uv = np.stack([X.ravel(), Y.ravel()], 1)
        F = _grid_faces(nx, nx, alt=True)
        z = 0.1 * np.sin(3 * X.ravel() + i) * np.cos(2 * Y.ravel())
        P = np.stack([X.ravel() + 2.0 * (i % 100), Y.ravel() + 2.0 * (i // 100), z], 1)
        Vs.append(P); Fs.append(F + off); Us.append(uv * sizes[i]); off += len(P)
    # shelf packing in texel units (island sizes scaled so they fill most of the atlas)
    ext = np.array([[u[:, 0].max(), u[:, 1].max()] for u in Us])
    total = float((ext[:, 0] + padding / atlas) @ (ext[:, 1] + padding / atlas))
    scale = np.sqrt(0.55 * 1.0 / total)
    pad = padding / atlas
    order = np.argsort(-ext[:, 1], kind="stable")
    x = pad; y = pad; row_h = 0.0
    place = np.zeros((islands, 2))
    for i in order:
        w, h = ext[i] * scale
        if x + w + pad > 1.0:
            x = pad; y += row_h + pad; row_h = 0.0
        place[i] = (x, y)
        x += w + pad; row_h = max(row_h, h)
    if y + row_h > 1.0:
        raise RuntimeError("validation atlas does not fit; lower the fill factor")
    UV = [Us[i] * scale + place[i] for i in range(islands)]
    V = np.concatenate(Vs); F = np.concatenate(Fs); U = np.concatenate(UV)
    vofs = np.cumsum([0] + [len(p) for p in Vs])
    tofs = np.cumsum([0] + [len(f) for f in Fs])
    m = len(F)
    info = {"shifted": [], "folded": [], "mirrored": [], "outside": []}
    # overlaps: shift whole islands by U(0, 8) texels (u and v)
    n_shift = int(rng.binomial(m, overlap_rate))
    if overlap_rate > 0:
        n_shift = max(1, n_shift)
    for i in rng.choice(islands, n_shift, replace=False):
        d = rng.uniform(0, 8, 2) / atlas
        U[vofs[i]:vofs[i + 1]] += d
        info["shifted"].append(int(i))
    # mirrored islands
    for i in rng.choice(islands, mirrored, replace=False):
        seg = U[vofs[i]:vofs[i + 1]]
        lo, hi = seg[:, 0].min(), seg[:, 0].max()
        seg[:, 0] = lo + hi - seg[:, 0]
        info["mirrored"].append(int(i))
    # folds: reflect one vertex of a triangle across the opposite edge
    n_fold = int(rng.binomial(m, fold_rate))
    if fold_rate > 0:
        n_fold = max(1, n_fold)
    for t in rng.choice(m, n_fold, replace=False):
        a, b, c = F[t]
        p, q = U[b], U[c]
        e = q - p
        r = U[a] - p
        proj = p + e * (r @ e) / max(e @ e, 1e-30)
        U[a] = 2 * proj - U[a]
        info["folded"].append(int(t))
    # out of range vertices: vertices of islands next to the atlas border,
    # pushed 1-4 texels past that border
    lo_v = np.argsort(U[:, 1])[: max(outside * 50, 1)]
    for vtx in rng.choice(lo_v, min(outside, len(lo_v)), replace=False):
        U[vtx, 1] = -rng.uniform(1.0, 4.0) / atlas
        info["outside"].append(int(vtx))
    return V.astype(np.float32), F.astype(np.int64), U.astype(np.float32), {**info, "vofs": vofs, "tofs": tofs}


# ------------------------------------------------------------------ energies
def energy_islands(seed=4000, count=512, tmin=500, tmax=50000, degenerate=0.05, max_aspect=1e3):
    """Smooth displaced grids with a fraction of near-degenerate triangles.

    Near-degenerate triangles are made by sliding one vertex of a triangle
    towards the midpoint of its opposite edge until the aspect ratio reaches
    U(10, max_aspect); a move that would invert an incident triangle of the
    xy projection is skipped, so the projection stays a flip-free
    parameterization. Returns a list of (P, T)."""
    rng = np.random.default_rng(seed)
    targets = np.exp(rng.uniform(np.log(tmin), np.log(tmax), count))
    out = []
    for t in targets:
        P, T = disk_patch(rng, t / 0.785, bumps=8, amp=0.3)
        P = P.astype(np.float64)
        # faces incident to each vertex (CSR: vertex -> its corners' faces)
        corner_v = T.reshape(-1)
        by_v = np.argsort(corner_v, kind="stable")
        vstart = np.searchsorted(corner_v[by_v], np.arange(len(P) + 1))
        inc_f = by_v // 3
        k = int(degenerate * len(T))
        for f in rng.choice(len(T), k, replace=False):
            a, b, c = T[f]
            mid = 0.5 * (P[b] + P[c])
            base = np.linalg.norm(P[c] - P[b])
            h = np.linalg.norm(P[a] - mid)
            target_h = base / rng.uniform(10.0, max_aspect)
            if h <= target_h:
                continue
            old = P[a].copy()
            P[a] = mid + (P[a] - mid) * (target_h / h)
            tri = T[inc_f[vstart[a]:vstart[a + 1]]]
            u = P[tri][:, :, :2].astype(np.float32).astype(np.float64)   # as stored
            sa = (u[:, 1, 0] - u[:, 0, 0]) * (u[:, 2, 1] - u[:, 0, 1]) - (u[:, 2, 0] - u[:, 0, 0]) * (u[:, 1, 1] - u[:, 0, 1])
            if (sa <= 0).any():
                P[a] = old
        out.append((P.astype(np.float32), T))
    return out


# ------------------------------------------------------------------ dense scan
def _value_noise3(p, rng, octaves=4):
    """Trilinear value noise, ``octaves`` octaves, lattice values from the seed."""
    out = np.zeros(len(p))
    amp = 1.0; freq = 2.0; norm = 0.0
    for _ in range(octaves):
        n = int(freq) + 2
        lat = rng.uniform(-1, 1, (n, n, n))
        q = (p * 0.5 + 0.5) * freq
        i0 = np.clip(np.floor(q).astype(int), 0, n - 2)
        f = q - i0
        f = f * f * (3 - 2 * f)
        acc = np.zeros(len(p))
        for dx in (0, 1):
            for dy in (0, 1):
                for dz in (0, 1):
                    w = (f[:, 0] if dx else 1 - f[:, 0]) * (f[:, 1] if dy else 1 - f[:, 1]) * \
                        (f[:, 2] if dz else 1 - f[:, 2])
                    acc += w * lat[i0[:, 0] + dx, i0[:, 1] + dy, i0[:, 2] + dz]
        out += amp * acc; norm += amp
        amp *= 0.5; freq *= 2.0
    return out / norm


def noisy_sphere(seed=5000, tris=5_000_000, amp=0.05):
    """Closed UV-sphere-like surface (cube-sphere, no poles) with about ``tris``
    triangles, displaced radially by 4-octave value noise."""
    rng = np.random.default_rng(seed)
    k = max(2, int(round(np.sqrt(tris / 12.0))))
    s = np.linspace(-1.0, 1.0, k + 1)
    A, B = np.meshgrid(s, s)
    A = A.ravel(); B = B.ravel()
    Vs, Fs = [], []
    off = 0
    for axis in range(3):
        for sgn in (-1.0, 1.0):
            P = np.zeros((len(A), 3))
            o = [i for i in range(3) if i != axis]
            P[:, axis] = sgn; P[:, o[0]] = A; P[:, o[1]] = B
            F = _grid_faces(k + 1, k + 1, alt=True)
            if sgn * (1 if axis != 1 else -1) < 0:
                F = F[:, ::-1]
            Vs.append(P); Fs.append(F + off); off += len(P)
    V = np.concatenate(Vs); F = np.concatenate(Fs)
    key = np.round(V * 1e6).astype(np.int64)
    _, idx, inv = np.unique(key, axis=0, return_index=True, return_inverse=True)
    V = V[idx]; F = inv.reshape(-1)[F]
    V = V / np.linalg.norm(V, axis=1, keepdims=True)
    V = V * (1.0 + amp * _value_noise3(V, rng))[:, None]
    return V.astype(np.float32), F.astype(np.int64)


def kmeans_charts(V, F, k=3000, seed=5001, iters=8, device=None):
    """Cut a closed mesh into charts: k-means on face normals (plus a weak
    position term so charts stay compact), then split labels into connected
    components. Returns a list of face-index arrays. With a torch ``device``
    the assignment steps run there (test-data generation at 5M faces)."""
    import scipy.sparse as sp
    from scipy.sparse.csgraph import connected_components
    rng = np.random.default_rng(seed)
    P = V.astype(np.float64)
    e1 = P[F[:, 1]] - P[F[:, 0]]; e2 = P[F[:, 2]] - P[F[:, 0]]
    nrm = np.cross(e1, e2); nrm /= np.maximum(np.linalg.norm(nrm, axis=1, keepdims=True), 1e-30)
    cen = P[F].mean(1)
    feat = np.concatenate([nrm, 0.5 * cen], 1)
    C = feat[rng.choice(len(F), k, replace=False)]
    lab = np.zeros(len(F), np.int64)
    chunk = 1 << 18
    if device is not None:
        import torch
        X = torch.from_numpy(feat).to(device)
        x2 = (X * X).sum(1)
    for _ in range(iters):
        if device is not None:
            Ct = torch.from_numpy(C).to(device)
            c2 = (Ct * Ct).sum(1)
            lt = torch.empty(len(F), dtype=torch.int64, device=device)
            for s in range(0, len(F), chunk):
                d = x2[s:s + chunk, None] - 2 * X[s:s + chunk] @ Ct.T + c2[None]
                lt[s:s + chunk] = d.argmin(1)
            lab = lt.cpu().numpy()
        else:
            for s in range(0, len(F), chunk):
                x = feat[s:s + chunk]
                d = (x * x).sum(1)[:, None] - 2 * x @ C.T + (C * C).sum(1)[None]
                lab[s:s + chunk] = d.argmin(1)
        cnt = np.bincount(lab, minlength=k)
        for j in range(feat.shape[1]):
            C[:, j] = np.bincount(lab, weights=feat[:, j], minlength=k) / np.maximum(cnt, 1)
    # connected components inside each label (faces sharing an edge)
    a = np.concatenate([F[:, 0], F[:, 1], F[:, 2]]); b = np.concatenate([F[:, 1], F[:, 2], F[:, 0]])
    fid = np.tile(np.arange(len(F)), 3)
    key = np.minimum(a, b) * len(V) + np.maximum(a, b)
    o = np.argsort(key, kind="stable")
    ks = key[o]; fs = fid[o]
    same = ks[1:] == ks[:-1]
    f0 = fs[:-1][same]; f1 = fs[1:][same]
    link = lab[f0] == lab[f1]
    G = sp.coo_matrix((np.ones(int(link.sum())), (f0[link], f1[link])), shape=(len(F), len(F)))
    _, comp = connected_components(G, directed=False)
    order = np.argsort(comp, kind="stable")
    cuts = np.flatnonzero(np.diff(comp[order])) + 1
    return np.split(order, cuts)


def disk_charts(V, F, charts, min_tris=20):
    """(P, T) of every chart (face-index array) that is a topological disk:
    one boundary loop and Euler characteristic 1, at least ``min_tris``
    triangles (the dense-scan workload keeps disks only)."""
    out = []
    for fidx in charts:
        if len(fidx) < min_tris:
            continue
        P, T = _compact(V, F[fidx])
        a = np.concatenate([T[:, 0], T[:, 1], T[:, 2]]); b = np.concatenate([T[:, 1], T[:, 2], T[:, 0]])
        key = np.minimum(a, b) * len(P) + np.maximum(a, b)
        uk, cnt = np.unique(key, return_counts=True)
        if len(P) - len(uk) + len(T) != 1 or (cnt > 2).any():
            continue
        # boundary half-edges (edges used once) must form a single loop
        once = np.isin(key, uk[cnt == 1])
        ba, bb = a[once], b[once]
        if len(ba) == 0:
            continue
        nxt = dict(zip(ba.tolist(), bb.tolist()))
        if len(nxt) != len(ba):
            continue
        start = int(ba[0]); v = start; steps = 0
        while True:
            v = nxt.get(v, -1); steps += 1
            if v == start or v < 0 or steps > len(ba):
                break
        if v == start and steps == len(ba):
            out.append((P.astype(np.float32), T))
    return out


def shelf_pack(uvs, atlas=4096, padding=4, fill=0.6):
    """Shelf packing of per-chart UV arrays into [0, 1]^2 with ``padding``
    texels between charts (test data for validation; not a product packer)."""
    lo = [u.min(0) for u in uvs]
    ext = np.array([u.max(0) - l for u, l in zip(uvs, lo)])
    pad = padding / atlas
    total = float(((ext[:, 0] + pad) * (ext[:, 1] + pad)).sum())
    scale = np.sqrt(fill / max(total, 1e-30))
    for _ in range(20):
        x = pad; y = pad; row_h = 0.0
        place = np.zeros((len(uvs), 2))
        for i in np.argsort(-ext[:, 1], kind="stable"):
            w, h = ext[i] * scale
            if x + w + pad > 1.0:
                x = pad; y += row_h + pad; row_h = 0.0
            place[i] = (x, y)
            x += w + pad; row_h = max(row_h, h)
        if y + row_h + pad <= 1.0:
            return [(u - l) * scale + place[i] for i, (u, l) in enumerate(zip(uvs, lo))]
        scale *= 0.9
    raise RuntimeError("shelf_pack: charts do not fit")


def mesh_charts(seed=6000, nx=256, ny=256, block=32, fold_every=2):
    """A bumpy grid mesh cut into block charts, in the input layout of
    engine/hier.py (Solver.relax, chart_checks): returns (V, F, FF, faces,
    loc, chart, CV, nv, nchart, U0). Every chart has its own UV vertices
    (CV); U0 is the planar position with small noise, and every
    ``fold_every``-th chart has two vertices reflected through its centre
    (folds). Vectorised, for bench sizes."""
    rng = np.random.default_rng(seed)
    s = np.arange(nx + 1, dtype=np.float64)
    X, Y = np.meshgrid(s, np.arange(ny + 1, dtype=np.float64))
    V2 = np.stack([X.ravel(), Y.ravel()], 1) + rng.uniform(-0.2, 0.2, ((nx + 1) * (ny + 1), 2))
    z = 0.6 * np.sin(V2[:, 0] / 4.0) * np.cos(V2[:, 1] / 5.0)
    V = np.concatenate([V2, z[:, None]], 1)
    cx, cy = np.meshgrid(np.arange(nx), np.arange(ny))
    cx, cy = cx.ravel(), cy.ravel()
    a = cy * (nx + 1) + cx
    b, c, d = a + 1, a + nx + 1, a + nx + 2
    F = np.stack([np.stack([a, b, d], 1), np.stack([a, d, c], 1)], 1).reshape(-1, 3).astype(np.int64)
    fx, fy = np.repeat(cx, 2), np.repeat(cy, 2)
    m = len(F)
    # face adjacency: the face across corner edge k (F[f,k] -> F[f,k+1])
    key = F * (len(V)) + F[:, [1, 2, 0]]
    rkey = F[:, [1, 2, 0]] * (len(V)) + F
    order = np.argsort(key.ravel())
    sk = key.ravel()[order]
    pos = np.searchsorted(sk, rkey.ravel())
    pos = np.minimum(pos, len(sk) - 1)
    hit = sk[pos] == rkey.ravel()
    FF = np.where(hit, order[pos] // 3, -1).reshape(m, 3)
    nbx = (nx + block - 1) // block
    lab = (fx // block) + (fy // block) * nbx
    faces = np.arange(m, dtype=np.int64)
    loc = np.arange(m, dtype=np.int64)
    _, chart = np.unique(lab, return_inverse=True)
    nchart = int(chart.max()) + 1
    ck = chart[:, None] * len(V) + F                      # (chart, mesh vertex) per corner
    uk, CV = np.unique(ck.ravel(), return_inverse=True)
    CV = CV.reshape(m, 3).astype(np.int64)
    nv = len(uk)
    vmesh = uk % len(V)
    vch = uk // len(V)
    U0 = V2[vmesh] * 0.9 + rng.normal(0, 0.03, (nv, 2))
    for ch in range(0, nchart, max(int(fold_every), 1)):
        ids = np.nonzero(vch == ch)[0]
        mv = rng.choice(ids, 2, replace=False)
        ctr = U0[ids].mean(0)
        U0[mv] = ctr + (ctr - U0[mv]) * 0.3
    return V, F, FF, faces, loc, chart.astype(np.int64), CV, int(nv), nchart, U0
