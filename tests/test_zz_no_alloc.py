"""The no-allocation ARAP entry point (uva_arap_noalloc) against the regular
one (uva_arap).

uva_arap_noalloc serves callers that cannot allocate device memory while
they run, such as a host application that owns a fixed device pool: it
borrows one static device array for the solver scratch instead of taking
scratch buffers from the caller. This file is named so that pytest collects
it last; it passes alone in a fresh process and after the other tests.
"""
import ctypes as C

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

TOL = 1e-12   # same kernel, same per-island arithmetic: agreement to round-off


# the caller's solver scratch, which the entry point must not read: a caller
# without device scratch passes null for all of it
SCRATCH_FIELDS = ("work", "cpart", "x64", "b64", "rc", "r32", "d32", "p32", "q32", "hist")


def _batch():
    from ultimate_uv_artist_b200 import synth
    from ultimate_uv_artist_b200.device import DeviceBatch, concat_charts
    rng = np.random.default_rng(516)
    isl = synth.uneven_islands(seed=515, count=10, tmin=20, tmax=4000)
    # one island above UVA_CLASS_BIG (8,192 vertices): a whole CTA with its CG
    # vectors in global memory, here in the static array
    isl.append(synth.disk_patch(rng, 25000))
    P, T, _, vofs, tofs = concat_charts([(p, t) for p, t in isl], with_uv=False)
    assert vofs[-1] <= 32768 and tofs[-1] <= 65536
    assert int(np.diff(vofs).max()) > 8192
    db = DeviceBatch(P, T, vofs, tofs)
    db.lscm()
    return db, vofs


def test_noalloc_matches_allocating_entry_point(cuda):
    from ultimate_uv_artist_b200 import _lib
    L = _lib.lib()
    db, vofs = _batch()
    U0 = db.U.clone()
    prm = db.params("arap", iters=6, line_search=True)
    stream = db._stream()
    _lib.check(L.uva_arap(C.byref(db.desc), C.byref(prm), stream), "uva_arap")
    Uref = db.U.clone()
    st_ref = db.island_status()
    ext = float((Uref.max(0).values - Uref.min(0).values).max())
    for call in range(2):
        db.U.copy_(U0)
        status = torch.zeros_like(db.status)
        desc = _lib.BatchDesc.from_buffer_copy(db.desc)
        desc.status = status.data_ptr()
        for f in SCRATCH_FIELDS:
            setattr(desc, f, None)
        _lib.check(L.uva_arap_noalloc(C.byref(desc), C.byref(prm), stream), "uva_arap_noalloc")
        torch.cuda.synchronize()
        err = float((db.U - Uref).abs().max()) / ext
        assert err <= TOL, f"call {call}: relative UV difference {err:.3e}"
        raw = status[:db.nc].cpu().numpy()
        st = raw.view(st_ref.dtype).reshape(-1)
        assert np.array_equal(st["outer_iters"], st_ref["outer_iters"])
        assert (st["resid"] <= 1e-6 + 1e-12).all()


def test_noalloc_rejects_oversize_batch(cuda):
    from ultimate_uv_artist_b200 import _lib
    L = _lib.lib()
    db, _ = _batch()
    desc = _lib.BatchDesc.from_buffer_copy(db.desc)
    desc.n = 40000          # checked before anything touches the device
    prm = db.params("arap", iters=1)
    rc = L.uva_arap_noalloc(C.byref(desc), C.byref(prm), db._stream())
    assert rc == _lib.UVA_E_TOOBIG
    assert b"32768" in L.uva_last_error()
    # more islands than the fixed x64 / b64 rows can hold (max(n, nc) rows)
    desc = _lib.BatchDesc.from_buffer_copy(db.desc)
    desc.nc = 40000
    rc = L.uva_arap_noalloc(C.byref(desc), C.byref(prm), db._stream())
    assert rc == _lib.UVA_E_TOOBIG
