"""Generate the golden fixtures of the report and bookkeeping functions by
running the REFERENCE implementation (Ultimate UV Artist, engine/*.py):

* metrics.seam_report / preservation_report / full_report
  (engine/metrics.py:226-311), including full_report with in_v / in_f as the
  ComfyUI node calls it (nodes.py:222, :294);
* validate.validate_uvs with in_v / in_f / in_normals / out_normals /
  in_colors / out_colors (the preservation branch, engine/validate.py:191-199):
  exact, a moved corner, a NaN corner, +-0.0 corners, mismatched colours, a
  dropped triangle;
* param.tutte, boundary_edges_oriented, boundary_loops, cot_laplacian
  (engine/param.py:47-94, 182-202) on disks, an annulus, a bow-tie,
  duplicated and degenerate triangles;
* gpu.unique_edges, sym_csr, csr32, spmm (engine/gpu.py:16-63) on CPU torch.

    NUMBA_CACHE_DIR=/tmp/nb python tests/golden/make_golden_reports.py /path/to/ultimate_uv_artist

The reference is only read here; the tests compare the CUDA path against the
committed golden_reports.npz.
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from ultimate_uv_artist_b200 import synth  # noqa: E402


def grid_mesh(nx, ny):
    """Welded planar grid (z = a smooth bump) of (nx-1)(ny-1)*2 triangles."""
    x, y = np.meshgrid(np.linspace(-1, 1, nx), np.linspace(-1, 1, ny))
    V = np.stack([x.ravel(), y.ravel(), 0.3 * np.exp(-2 * (x.ravel() ** 2 + y.ravel() ** 2))], 1)
    F = synth._grid_faces(nx, ny)
    return V.astype(np.float32), F.astype(np.int64)


def box_mesh(k):
    """Closed welded box of 6 k x k grids (a regression-style closed mesh)."""
    s = np.linspace(-1, 1, k)
    a, b = np.meshgrid(s, s)
    a, b = a.ravel(), b.ravel()
    F0 = synth._grid_faces(k, k)
    Vs, Fs, off = [], [], 0
    for axis in range(3):
        for sgn in (-1.0, 1.0):
            P = np.zeros((len(a), 3))
            P[:, axis] = sgn
            o = [i for i in range(3) if i != axis]
            P[:, o[0]], P[:, o[1]] = a, b
            Vs.append(P)
            Fs.append((F0 if sgn > 0 else F0[:, ::-1]) + off)
            off += len(P)
    V = np.concatenate(Vs)
    F = np.concatenate(Fs)
    key = np.round(V * 1e6).astype(np.int64)
    _, first, inv = np.unique(key, axis=0, return_index=True, return_inverse=True)
    return V[first].astype(np.float32), inv.reshape(-1)[F].astype(np.int64)


def cut_unwrap(V, F, chart, tiles):
    """Seam-cut mesh: every chart gets its own copies of its vertices; UVs are
    a planar projection of the chart fitted into its atlas tile."""
    out_v, out_f, out_uv, xref = [], np.empty_like(F), [], []
    base = 0
    nt = int(np.ceil(np.sqrt(tiles)))
    for c in range(int(chart.max()) + 1):
        fs = np.nonzero(chart == c)[0]
        used, inv = np.unique(F[fs], return_inverse=True)
        P = V[used].astype(np.float64)
        n = np.cross(V[F[fs][:, 1]] - V[F[fs][:, 0]], V[F[fs][:, 2]] - V[F[fs][:, 0]]).sum(0)
        ax = int(np.argmax(np.abs(n)))
        q = P[:, [i for i in range(3) if i != ax]]
        q = (q - q.min(0)) / max(float(np.ptp(q, 0).max()), 1e-9)
        ty, tx = divmod(c, nt)
        uv = (q * 0.8 + 0.1 + np.array([tx, ty])) / nt
        out_f[fs] = inv.reshape(-1, 3) + base
        out_v.append(V[used])
        out_uv.append(uv)
        xref.append(used)
        base += len(used)
    return (np.concatenate(out_v), out_f, np.concatenate(out_uv).astype(np.float32),
            np.concatenate(xref).astype(np.int64))


def topology_cases():
    """Triangle lists with boundaries of every kind the helpers meet."""
    rng = np.random.default_rng(41)
    Pd, Td = synth.disk_patch(rng, 300)
    _, Tg = grid_mesh(9, 7)
    # annulus: the grid with its centre cells removed
    Va, Ta = grid_mesh(12, 12)
    c = Va[Ta].mean(1)
    Ta = Ta[np.hypot(c[:, 0], c[:, 1]) > 0.4]
    # bow-tie: two fans sharing one vertex
    Tb = np.array([[0, 1, 2], [0, 2, 3], [0, 4, 5], [0, 5, 6]], np.int64)
    # duplicated and reversed-duplicate triangles, a repeated-vertex triangle
    Tx = np.concatenate([Tg, Tg[:3], Tg[3:5, ::-1], [[0, 0, 1], [4, 5, 4]]])
    return {"disk": Td, "grid": Tg, "annulus": Ta, "bowtie": Tb, "dups": Tx}


def main(ref_root):
    sys.path.insert(0, ref_root)
    import torch
    from engine import gpu, metrics, param, validate

    out = {}
    # ------------------------------------------------------------ param helpers
    for name, T in topology_cases().items():
        bi, bj = param.boundary_edges_oriented(T)
        loops = param.boundary_loops(T)
        out[f"t_{name}_T"] = T
        out[f"t_{name}_bi"] = bi
        out[f"t_{name}_bj"] = bj
        out[f"t_{name}_loops"] = np.concatenate(loops) if loops else np.zeros(0, np.int64)
        out[f"t_{name}_loop_len"] = np.array([len(x) for x in loops], np.int64)
    P, T = synth.hemisphere_patch(seed=13, n=12, jitter=0.01)
    P = P.astype(np.float64)
    X, _ = param.local_frames(P, T)
    cots = param.cot_weights(X)
    Lc = param.cot_laplacian(len(P), T, cots)
    out.update(l_P=P, l_T=T, l_cots=cots, l_dense=Lc.toarray())
    out["u_tutte_hemi"] = param.tutte(P, T)
    rng = np.random.default_rng(43)
    Pd, Td = synth.disk_patch(rng, 500, amp=0.4)
    Pd = Pd.astype(np.float64)
    out.update(u_P=Pd, u_T=Td, u_tutte_disk=param.tutte(Pd, Td), u_hP=P, u_hT=T)

    # ------------------------------------------------------------ gpu helpers (CPU torch)
    Tg = topology_cases()["dups"]
    n = int(Tg.max()) + 1
    ea, eb, inv, cnt = gpu.unique_edges(torch.from_numpy(Tg), n)
    out.update(g_T=Tg, g_n=np.array(n), g_ea=ea.numpy(), g_eb=eb.numpy(), g_inv=inv.numpy(), g_cnt=cnt.numpy())
    keep = (ea != eb)
    off = torch.from_numpy(np.random.default_rng(44).normal(size=int(keep.sum())))
    diag = torch.from_numpy(np.random.default_rng(45).normal(size=n)) + 5.0
    S = gpu.sym_csr(n, ea[keep], eb[keep], off, diag)
    out.update(g_off=off.numpy(), g_diag=diag.numpy(), g_crow=S.crow_indices().numpy(), g_col=S.col_indices().numpy(),
               g_val=S.values().numpy())
    X2 = torch.from_numpy(np.random.default_rng(46).normal(size=(n, 3)))
    out["g_X"] = X2.numpy()
    out["g_spmm64"] = gpu.spmm(gpu.csr32(S), X2).numpy()
    S32 = gpu.csr32(torch.sparse_csr_tensor(S.crow_indices(), S.col_indices(), S.values().float(), S.shape))
    out["g_spmm32"] = gpu.spmm(S32, X2.float()).numpy()
    out["g_spmv32"] = gpu.spmm(S32, X2[:, 0].float().contiguous()).numpy()
    coo = S.to_sparse_coo()
    out.update(g_coo_idx=coo.indices().numpy(), g_coo_val=coo.values().numpy())

    # ------------------------------------------------------------ reports
    meshes = {}
    Vg, Fg = grid_mesh(17, 13)
    cg = ((Vg[Fg].mean(1)[:, 0] > 0).astype(np.int64) + 2 * (Vg[Fg].mean(1)[:, 1] > 0.3))
    meshes["plane"] = (Vg, Fg, cg, 4)
    Vb, Fb = box_mesh(6)
    nb_ = np.abs(np.cross(Vb[Fb[:, 1]] - Vb[Fb[:, 0]], Vb[Fb[:, 2]] - Vb[Fb[:, 0]]))
    meshes["box"] = (Vb, Fb, np.argmax(nb_, 1) * 2 + (Vb[Fb].mean(1)[np.arange(len(Fb)), np.argmax(nb_, 1)] > 0), 6)
    # a non-manifold fin on the plane: a third face on an interior edge
    e = Fg[40, :2]
    Vf = np.concatenate([Vg, [[0.1, 0.1, 1.0]]]).astype(np.float32)
    Ff = np.concatenate([Fg, [[e[0], e[1], len(Vg)]]])
    meshes["fin"] = (Vf, Ff, np.concatenate([cg, [4]]), 5)
    for name, (V, F, chart, tiles) in meshes.items():
        ov, of, ouv, xref = cut_unwrap(V, F, chart, tiles)
        rep = metrics.seam_report(ov, of, ouv)
        wk = np.random.default_rng(47).permutation(len(V))[xref]     # weld keys: arbitrary labels of the source vertex
        repw = metrics.seam_report(ov, of, ouv, weld_keys=wk)
        full, isl = metrics.full_report(ov, of, ouv, raster_res=256, in_v=V, in_f=F)
        out.update({f"r_{name}_V": V, f"r_{name}_F": F, f"r_{name}_ov": ov, f"r_{name}_of": of,
                    f"r_{name}_ouv": ouv, f"r_{name}_xref": xref, f"r_{name}_wk": wk, f"r_{name}_isl": isl})
        for tag, r in (("seam", rep), ("seamw", repw), ("full", full)):
            keys = sorted(k for k in r if isinstance(r[k], (int, float, bool, np.integer, np.floating)))
            out[f"r_{name}_{tag}_keys"] = np.array(keys)
            out[f"r_{name}_{tag}_vals"] = np.array([float(r[k]) for k in keys])

    # preservation_report cases on the plane
    V, F, chart, tiles = meshes["plane"]
    ov, of, ouv, xref = cut_unwrap(V, F, chart, tiles)
    nrm = np.random.default_rng(48).normal(size=(len(V), 3)).astype(np.float32)
    col = np.random.default_rng(49).integers(0, 255, size=(len(V), 4)).astype(np.uint8)
    cases = {}
    cases["exact"] = (V, F, ov, of, {"normals": nrm, "colors": col}, {"normals": nrm[xref], "colors": col[xref]})
    moved = ov.copy(); moved[7, 1] = np.nextafter(moved[7, 1], np.float32(2))
    cases["moved"] = (V, F, moved, of, {"normals": nrm}, {"normals": nrm[xref]})
    vn = V.copy(); vn[int(F[5, 1])] = np.nan
    cases["nan"] = (vn, F, np.where(np.isnan(vn[xref]), np.nan, ov).astype(np.float32), of, None, None)
    vz = V.copy(); vz[int(F[0, 0]), 0] = 0.0
    oz = vz[xref].copy(); oz[np.nonzero(xref == int(F[0, 0]))[0], 0] = -0.0
    cases["signed_zero"] = (vz, F, oz, of, None, None)
    c2 = col[xref].copy(); c2[3, 2] ^= 1
    cases["colors"] = (V, F, ov, of, {"colors": col, "extra": None}, {"colors": c2})
    cases["missing"] = (V, F, ov, of, {"normals": nrm}, {})
    cases["dropped"] = (V, F[:-1], ov, of, None, None)
    cases["dtype"] = (V.astype(np.float64), F, ov, of, {"normals": nrm.astype(np.float64)}, {"normals": nrm[xref]})
    for name, (iv, iff, o_v, o_f, ia, oa) in cases.items():
        r = metrics.preservation_report(iv, iff, o_v, o_f, ia, oa)
        keys = sorted(r)
        out[f"p_{name}_keys"] = np.array(keys)
        out[f"p_{name}_vals"] = np.array([bool(r[k]) for k in keys])
        out[f"p_{name}_in_v"] = iv
        out[f"p_{name}_in_f"] = iff
        out[f"p_{name}_out_v"] = o_v
        out[f"p_{name}_out_f"] = o_f
        for side, d in (("ia", ia), ("oa", oa)):
            for k, a in (d or {}).items():
                out[f"p_{name}_{side}_{k}"] = a if a is not None else np.zeros(0)
            out[f"p_{name}_{side}_names"] = np.array(sorted((d or {}).keys()))
            out[f"p_{name}_{side}_none"] = np.array([k for k, a in (d or {}).items() if a is None])

    # validate_uvs preservation branch (atlas 512, padding 4), on the box
    V, F, chart, tiles = meshes["box"]
    ov, of, ouv, xref = cut_unwrap(V, F, chart, tiles)
    nrm = np.random.default_rng(50).normal(size=(len(V), 3)).astype(np.float32)
    col = np.random.default_rng(51).integers(0, 255, size=(len(V), 3)).astype(np.uint8)
    vcases = {}
    vcases["exact"] = dict(in_v=V, in_f=F, in_normals=nrm, out_normals=nrm[xref], in_colors=col, out_colors=col[xref])
    moved = ov.copy(); moved[11, 0] += np.float32(1e-3)
    vcases["moved"] = dict(v=moved, in_v=V, in_f=F)
    vn = V.astype(np.float64).copy(); vn[int(F[2, 2]), 1] = np.nan
    vcases["nan"] = dict(in_v=vn, in_f=F)
    vz = V.copy(); k0 = int(F[0, 0]); vz[k0, 0] = 0.0
    oz = vz[xref].copy(); oz[np.nonzero(xref == k0)[0], 0] = -0.0
    vcases["signed_zero"] = dict(v=oz, in_v=vz, in_f=F)
    c2 = col[xref].copy(); c2[0, 0] ^= 4
    vcases["colors"] = dict(in_v=V, in_f=F, in_colors=col, out_colors=c2, in_normals=nrm, out_normals=nrm[xref])
    vcases["dropped"] = dict(in_v=V, in_f=F[1:])
    out.update(vv_ov=ov, vv_of=of, vv_ouv=ouv, vv_V=V, vv_F=F, vv_nrm=nrm, vv_col=col, vv_xref=xref)
    for name, kw in vcases.items():
        v = kw.pop("v", ov)
        rep, prob = validate.validate_uvs(v, of, ouv, atlas=512, padding=4, **kw)
        keys = sorted(k for k in rep if isinstance(rep[k], (int, float, bool, np.integer, np.floating)))
        out[f"vv_{name}_keys"] = np.array(keys)
        out[f"vv_{name}_vals"] = np.array([float(rep[k]) for k in keys])
        out[f"vv_{name}_prob"] = prob
        out[f"vv_{name}_v"] = v
        for k, a in kw.items():
            out[f"vv_{name}_{k}"] = a
    path = os.path.join(HERE, "golden_reports.npz")
    np.savez_compressed(path, **out)
    print("wrote", path, os.path.getsize(path), "bytes")


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.environ.get("UVA_REFERENCE", ""))
