"""Block-Jacobi smoother of the island PCG: the FP16 block inverses that
uva_batch_setup writes, applied by the warp-level MMA product, against the
FP64 inverses of the same diagonal blocks (numpy), and its effect on the
solves (same tolerances, fewer iterations than point Jacobi)."""
import ctypes as C

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _batch(seed=11, block_jacobi=True):
    from ultimate_uv_artist_b200 import synth, _lib
    from ultimate_uv_artist_b200.device import DeviceBatch, concat_charts
    isl = synth.uneven_islands(seed=seed, count=24, tmin=8, tmax=5000)
    isl.append(synth.hemisphere_patch(seed=3, n=12))
    P, T, U, vofs, tofs = concat_charts([(p, t) for p, t in isl], with_uv=False)
    return DeviceBatch(P, T, vofs, tofs, semantics=_lib.SEM_BATCH, device=torch.device("cuda", 0),
                       block_jacobi=block_jacobi)


def _blocks(db, op):
    """FP64 inverses of every slice's diagonal block, assembled like the
    solver's operator from the device slot weights."""
    pl = db.plan
    cw = db.slot_cw.cpu().numpy()
    col = cw[:, 0] & 0xFFFFFF
    c2 = (cw[:, 0] >> 24).astype(np.float64)
    w = cw[:, 1].view(np.float32).astype(np.float64)
    pins = db.pins.cpu().numpy()
    wpin = db.wpin.cpu().numpy()
    out = {}
    for isl in range(pl.nc):
        v0, n = int(pl.vofs[isl]), int(pl.vofs[isl + 1] - pl.vofs[isl])
        vr = pl.vert_row[v0:v0 + n]
        pin = vr[pins[isl, 0]] if n else -1
        hard = {int(vr[p]) for p in pins[isl, 1:] if p >= 0}
        for ls in range((n + 31) // 32):
            gs = int(pl.sofs[isl]) + ls
            q0, q1 = int(pl.slice_ptr[gs]), int(pl.slice_ptr[gs + 1])
            width = (q1 - q0) // 32
            B = np.zeros((32, 32), np.complex128)
            dead = []
            for lane in range(32):
                r = 32 * ls + lane
                if r >= n or (op == 1 and r in hard):
                    dead.append(lane)
                    continue
                q = q0 + lane + 32 * np.arange(width)
                keep = col[q] != r
                d = w[q][keep].sum() + (wpin[isl] if op == 0 and r == pin else 0.0)
                for cc, ww, cq in zip(col[q][keep], w[q][keep], c2[q][keep]):
                    if cc // 32 == ls:
                        B[lane, cc % 32] -= ww + (0.5j * cq if op == 1 else 0.0)
                B[lane, lane] = d
                if not d > 0:
                    dead.append(lane)
            for lane in dead:   # identity rows and columns
                B[lane, :] = 0
                B[:, lane] = 0
                B[lane, lane] = 1
            out[(isl, ls)] = np.linalg.inv(B)
    return out


@pytest.mark.parametrize("op", [0, 1])
def test_block_inverses_apply(cuda, op):
    from ultimate_uv_artist_b200 import _lib
    db = _batch()
    rng = np.random.default_rng(op)
    pl = db.plan
    r = rng.standard_normal((db.n, 2)).astype(np.float32)
    # a slice of tiny and one of huge values: the per-slice power-of-two scale
    r[:32] *= 1e-20
    r[32:64] *= 1e20
    if op == 1:   # hard-pinned rows carry no residual
        pins = db.pins.cpu().numpy()
        for isl in range(pl.nc):
            v0 = int(pl.vofs[isl])
            for p in pins[isl, 1:]:
                if p >= 0:
                    r[v0 + pl.vert_row[v0 + p]] = 0
    rd = torch.from_numpy(r).to(cuda)
    zd = torch.full_like(rd, float("nan"))
    s = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    _lib.check(_lib.lib().uva_bjac_apply(C.byref(db.desc), op, rd.data_ptr(), zd.data_ptr(), s), "uva_bjac_apply")
    z = zd.cpu().numpy().astype(np.float64)
    assert np.isfinite(z).all()
    worst = 0.0
    for (isl, ls), Ci in _blocks(db, op).items():
        v0, n = int(pl.vofs[isl]), int(pl.vofs[isl + 1] - pl.vofs[isl])
        rows = np.arange(32 * ls, min(32 * ls + 32, n))
        rr = np.zeros(32, np.complex128)
        rr[:len(rows)] = r[v0 + rows, 0] + 1j * r[v0 + rows, 1]
        if op == 0:   # real blocks act on u and v separately
            ref = (Ci.real @ rr.real) + 1j * (Ci.real @ rr.imag)
        else:
            ref = Ci @ rr
        ref = ref[:len(rows)]
        got = z[v0 + rows, 0] + 1j * z[v0 + rows, 1]
        scale = np.abs(Ci).max() * np.abs(rr).max() + 1e-300
        worst = max(worst, float(np.abs(got - ref).max() / scale))
    # FP16 block entries (11 bits) and a 22-bit split of r, FP32 accumulation
    assert worst < 2e-3, worst


def test_block_jacobi_solves(cuda):
    """LSCM and ARAP with the block smoother reach the same tolerances and
    agree with the point-Jacobi solves; LSCM needs clearly fewer iterations."""
    a = _batch(seed=5, block_jacobi=True)
    b = _batch(seed=5, block_jacobi=False)
    for db in (a, b):
        db.lscm()
    sa, sb = a.island_status(), b.island_status()
    assert (sa["flags"] & 3 == 0).all() and (sb["flags"] & 3 == 0).all()
    assert (sa["resid"] <= 1e-9 * 1.001).all()
    ext = float((b.U.max(0).values - b.U.min(0).values).max())
    assert float((a.U - b.U).abs().max()) / ext < 1e-6
    big = np.diff(a.plan.vofs) > 256
    ia, ib = int(sa["cg_iters"][big].sum()), int(sb["cg_iters"][big].sum())
    assert ia < 0.85 * ib, (ia, ib)
    for db in (a, b):
        db.arap(iters=5)
    sa, sb = a.island_status(), b.island_status()
    assert (sa["resid"] <= 2e-7 * 1.001).all() and (sb["resid"] <= 2e-7 * 1.001).all()
    assert float((a.U - b.U).abs().max()) / ext < 1e-5
