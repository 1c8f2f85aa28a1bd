"""Re-entrant calls: the reference pipeline calls the per-chart API from
ThreadPoolExecutor workers (engine/pipeline.py:608-610, :721-722,
engine/merge.py:114). Eight threads call param.lscm, param.refine (with the
solver handed back), param.chart_quality and validate.validate_uvs on
different charts at once; every result equals the serial call's bit for bit
(the kernels reduce in a fixed order, and validation is exact)."""
from concurrent.futures import ThreadPoolExecutor

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _chart_job(P, T):
    from ultimate_uv_artist_b200.engine import param as Pm
    from ultimate_uv_artist_b200.engine import validate as Vd
    P = P.astype(np.float64)
    U0 = Pm.lscm(P, T)
    U1, solver = Pm.refine(P, T, U0, iters=5, tol=0.0)
    U2, _ = Pm.refine(P, T, U1, iters=3, tol=0.0, solver=solver)
    q = Pm.chart_quality(P, T, U2)
    lo, ext = U2.min(0), np.ptp(U2, 0).max()
    uv = ((U2 - lo) / ext * 0.9 + 0.05).astype(np.float32)
    rep, prob = Vd.validate_uvs(P, T, uv, atlas=1024, padding=4)
    return U0, U2, q["aniso_p95"], rep, prob


def test_concurrent_calls_match_serial(cuda):
    from ultimate_uv_artist_b200 import synth
    rng = np.random.default_rng(77)
    charts = [synth.disk_patch(rng, t) for t in rng.integers(200, 6000, 16)]
    serial = [_chart_job(P, T) for P, T in charts]
    with ThreadPoolExecutor(8) as ex:
        par = list(ex.map(lambda c: _chart_job(*c), charts))
    for (a0, a2, aq, arep, aprob), (b0, b2, bq, brep, bprob) in zip(serial, par):
        assert np.array_equal(a0, b0) and np.array_equal(a2, b2)
        assert aq == bq
        assert arep == brep and np.array_equal(aprob, bprob)
