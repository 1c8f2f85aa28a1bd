"""The reference's API surface for the drop-in modules, written from the
reference's SOURCE by static reading (ast, nothing of it is run): for each
drop-in module (engine/param.py, gpu.py, validate.py, metrics.py, pack.py,
charts.py, hier.py, overlapfix.py) every top-level function with its
parameters, and every call that the rest of the reference (engine/*.py,
nodes.py, tests/*.py) makes into these modules, with the number of
positional arguments and the keywords used, and where.

    python tests/golden/make_api_surface.py /path/to/ultimate_uv_artist
"""
from __future__ import annotations

import ast
import glob
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
MODULES = ("param", "gpu", "validate", "metrics", "pack", "charts", "hier", "overlapfix")


def signature_of(fn):
    a = fn.args
    pos = [x.arg for x in a.posonlyargs + a.args]
    return {"params": pos, "defaults": len(a.defaults), "vararg": a.vararg is not None,
            "kwonly": [x.arg for x in a.kwonlyargs], "kwarg": a.kwarg is not None}


def module_aliases(tree, this_module):
    """name -> module for module imports; name -> (module, function) for
    functions imported by name."""
    mods, funcs = {}, {}
    for node in ast.walk(tree):
        if isinstance(node, ast.ImportFrom):
            src = (node.module or "").split(".")[-1] if node.module else ""
            for al in node.names:
                name = al.asname or al.name
                if al.name in MODULES and src in ("", "engine"):
                    mods[name] = al.name
                elif src in MODULES and src != this_module:
                    funcs[name] = (src, al.name)
        elif isinstance(node, ast.Import):
            for al in node.names:
                last = al.name.split(".")[-1]
                if last in MODULES and al.asname:
                    mods[al.asname] = last
    return mods, funcs


def main(ref):
    out = {"functions": {}, "calls": {}}
    for m in MODULES:
        tree = ast.parse(open(os.path.join(ref, "engine", m + ".py")).read())
        out["functions"][m] = {n.name: signature_of(n) for n in tree.body if isinstance(n, ast.FunctionDef)}
    files = sorted(glob.glob(os.path.join(ref, "engine", "*.py")) + [os.path.join(ref, "nodes.py")]
                   + glob.glob(os.path.join(ref, "tests", "*.py")))
    for path in files:
        rel = os.path.relpath(path, ref)
        this = os.path.splitext(os.path.basename(path))[0] if rel.startswith("engine") else ""
        tree = ast.parse(open(path).read())
        mods, funcs = module_aliases(tree, this)
        for node in ast.walk(tree):
            if not isinstance(node, ast.Call):
                continue
            target = None
            if isinstance(node.func, ast.Attribute) and isinstance(node.func.value, ast.Name) \
                    and node.func.value.id in mods:
                target = (mods[node.func.value.id], node.func.attr)
            elif isinstance(node.func, ast.Name) and node.func.id in funcs:
                target = funcs[node.func.id]
            if target is None or target[0] == this:
                continue
            m, f = target
            rec = out["calls"].setdefault(m, {}).setdefault(f, {"npos": 0, "keywords": [], "sites": []})
            starred = any(isinstance(a, ast.Starred) for a in node.args)
            rec["npos"] = max(rec["npos"], 0 if starred else len(node.args))
            rec["keywords"] = sorted(set(rec["keywords"]) | {k.arg for k in node.keywords if k.arg})
            rec["sites"].append(f"{rel}:{node.lineno}")
    path = os.path.join(HERE, "api_surface.json")
    with open(path, "w") as fh:
        json.dump(out, fh, indent=1, sort_keys=True)
    n = sum(len(v) for v in out["calls"].values())
    print("wrote", path, n, "called functions")


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.environ.get("UVA_REFERENCE", ""))
