"""The topology plan built on the device (uva_dplan_build / uva_dplan_slots)
against the host plan (uva_plan_create / uva_plan_export): every array equal,
element for element, on uneven islands, on islands large enough for wider
aggregates, and on the topologies the host plan handles specially
(duplicated and reversed triangles, repeated-vertex triangles, non-manifold
edges, bow-ties, isolated vertices, several components, empty islands)."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

ARRAYS = ("tri4", "tri_edge", "sofs", "slice_ptr", "slot_col", "slot_edge", "slot_c", "vt_ptr", "vt", "vflags",
          "bofs", "bverts")


def _plans(charts):
    from ultimate_uv_artist_b200.device import DevicePlan, Plan, concat_charts
    P, Tc, U, vofs, tofs = concat_charts([(p, t) for p, t in charts], with_uv=False, with_t=False)
    dev = torch.device("cuda", 0)
    host = Plan(None, vofs, tofs, chart_tris=Tc[:2])
    devp = DevicePlan(Tc[:2], vofs, tofs, device=dev)
    torch.cuda.synchronize()
    return host, devp


def _compare(host, devp):
    for k in ("nc", "n", "t", "E", "nslices", "nslots", "nbverts", "maxrows", "ncoarse"):
        assert getattr(host, k) == getattr(devp, k), k
    for k in ARRAYS:
        a = np.asarray(getattr(host, k)).reshape(-1)
        b = np.asarray(getattr(devp, k)).reshape(-1)[:a.size]
        assert a.shape == b.shape and np.array_equal(a, b), (k, np.flatnonzero(a != b)[:10])
    for k in ("row_vert", "vert_row", "agg_rows", "cofs"):
        a = np.asarray(getattr(host, k)).reshape(-1)
        b = getattr(devp, k).cpu().numpy().reshape(-1)[:a.size]
        assert np.array_equal(a, b), (k, np.flatnonzero(a != b)[:10])
    assert np.array_equal(host.order, devp.order) and np.array_equal(host.class_ofs, devp.class_ofs)


def test_device_plan_uneven_islands(cuda):
    from ultimate_uv_artist_b200 import synth
    charts = synth.uneven_islands(seed=31, count=80, tmin=20, tmax=20000)
    _compare(*_plans(charts))


def test_device_plan_large_island(cuda):
    """About 35k vertices: 192-row aggregates, global-memory BFS state."""
    from ultimate_uv_artist_b200 import synth
    rng = np.random.default_rng(32)
    charts = [synth.disk_patch(rng, 90000), synth.disk_patch(rng, 300)]
    _compare(*_plans(charts))


def test_device_plan_topologies(cuda):
    rng = np.random.default_rng(33)
    from ultimate_uv_artist_b200 import synth
    P0, T0 = synth.disk_patch(rng, 400)
    n0 = len(P0)
    # duplicated, reversed and repeated-vertex triangles, a non-manifold fin
    Tdup = np.concatenate([T0, T0[:5], T0[5:9, ::-1], [[0, 0, 1], [2, 3, 2]], [[T0[20, 0], T0[20, 1], n0]]])
    Pdup = np.concatenate([P0, [[0.0, 0.0, 1.0]]]).astype(np.float32)
    # bow-tie plus an isolated vertex and a second component
    Pb = rng.normal(size=(12, 3)).astype(np.float32)
    Tb = np.array([[0, 1, 2], [0, 2, 3], [0, 4, 5], [0, 5, 6], [8, 9, 10], [8, 10, 11]], np.int64)
    # an island of 300 vertices and two components (blobs cross components)
    P1, T1 = synth.disk_patch(rng, 300)
    P2, T2 = synth.disk_patch(rng, 300)
    Pc = np.concatenate([P1, P2]).astype(np.float32)
    Tc = np.concatenate([T1, T2 + len(P1)])
    # an island with vertices and no triangles, and an empty one
    Pe = rng.normal(size=(3, 3)).astype(np.float32)
    Te = np.zeros((0, 3), np.int64)
    charts = [(Pdup, Tdup), (Pb, Tb), (Pc, Tc), (Pe, Te), (np.zeros((0, 3), np.float32), Te), (P0, T0.astype(np.int32))]
    _compare(*_plans(charts))


def test_device_plan_rejects_bad_index(cuda):
    from ultimate_uv_artist_b200.device import DevicePlan, concat_charts
    P = np.zeros((4, 3), np.float32)
    T = np.array([[0, 1, 2], [1, 2, 7]], np.int64)
    _, Tc, _, vofs, tofs = concat_charts([(P, T)], with_uv=False, with_t=False)
    with pytest.raises(ValueError, match="outside its island"):
        DevicePlan(Tc[:2], vofs, tofs, device=torch.device("cuda", 0))


def test_batch_on_device_plan_matches_host_plan(cuda):
    """gpu.Batch over either plan: bitwise the same LSCM + ARAP UVs."""
    from ultimate_uv_artist_b200 import synth
    from ultimate_uv_artist_b200.engine import gpu
    isl = synth.uneven_islands(seed=34, count=40, tmin=20, tmax=12000)
    out = []
    for where in ("host", "device"):
        b = gpu.Batch([(p, t, None) for p, t in isl], plan_on=where)
        b.lscm()
        b.arap(5, line_search=True)
        out.append(np.concatenate(b.chart_uvs()))
    assert np.array_equal(out[0], out[1])
