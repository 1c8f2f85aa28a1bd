"""The drop-in modules against the reference's API surface
(tests/golden/api_surface.json, read statically from the reference's source
by make_api_surface.py): every call the reference's pipeline, node and
tests make into engine/param.py, gpu.py, validate.py, metrics.py and
pack.py binds to this package's function of the same name (same
positional count, same keywords), and every public function of those
modules exists here with the reference's parameter names. charts.py,
hier.py and overlapfix.py are function-level replacements (the charting and
overlap-repair logic around them is outside the path): each function they
provide binds like the reference's. No GPU needed: signatures only."""
import importlib
import inspect
import json
import os

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
FULL = ("param", "gpu", "validate", "metrics", "pack")
PARTIAL = ("charts", "hier", "overlapfix")


@pytest.fixture(scope="module")
def surface():
    with open(os.path.join(HERE, "golden", "api_surface.json")) as fh:
        return json.load(fh)


def _mod(name):
    return importlib.import_module(f"ultimate_uv_artist_b200.engine.{name}")


def _binds(obj, npos, keywords):
    inspect.signature(obj).bind_partial(*([None] * npos), **{k: None for k in keywords})


@pytest.mark.parametrize("m", FULL)
def test_every_reference_call_binds(surface, m):
    mod = _mod(m)
    calls = surface["calls"].get(m, {})
    for f, rec in calls.items():
        obj = getattr(mod, f, None)
        assert obj is not None, f"{m}.{f} missing (called at {rec['sites'][:3]})"
        _binds(obj, rec["npos"], rec["keywords"])


@pytest.mark.parametrize("m", FULL)
def test_public_functions_keep_parameter_names(surface, m):
    mod = _mod(m)
    for f, sig in surface["functions"][m].items():
        if f.startswith("_"):
            continue
        obj = getattr(mod, f, None)
        assert obj is not None, f"{m}.{f} missing"
        params = inspect.signature(obj).parameters
        ours = [p for p in params if params[p].kind in (inspect.Parameter.POSITIONAL_ONLY,
                                                        inspect.Parameter.POSITIONAL_OR_KEYWORD)]
        assert ours[:len(sig["params"])] == sig["params"], (m, f, ours, sig["params"])


@pytest.mark.parametrize("m", PARTIAL)
def test_function_level_replacements_bind(surface, m):
    mod = _mod(m)
    provided = 0
    for f, sig in surface["functions"][m].items():
        obj = getattr(mod, f, None)
        if obj is None or not callable(obj):
            continue
        provided += 1
        inspect.signature(obj).bind_partial(**{p: None for p in sig["params"]})
        rec = surface["calls"].get(m, {}).get(f)
        if rec is not None:
            _binds(obj, rec["npos"], rec["keywords"])
    assert provided > 0
