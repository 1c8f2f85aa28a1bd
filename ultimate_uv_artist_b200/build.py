"""Build the sm_100a shared library ``libuva_b200.so`` in-tree with nvcc.

    python -m ultimate_uv_artist_b200.build        # or: from . import build; build.build()

The library is a plain C-ABI ``.so`` (declarations in include/uva_b200.h),
loaded with ctypes by ``ultimate_uv_artist_b200._lib``. nvcc cross-compiles
for sm_100a without a GPU, so the build runs on any machine with CUDA 12.8+.
"""
from __future__ import annotations

import hashlib
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(ROOT, "include")
LIB = os.path.join(HERE, "libuva_b200.so")
PYHOST_LIB = os.path.join(HERE, "libuva_pyhost.so")   # the batch constructor's charts pass (CPython API)
BUILD_DIR = os.path.join(ROOT, "_build")

CU_SOURCES = ["capi.cu", "solve.cu", "ops.cu", "chart_ops.cu", "validate.cu", "metrics.cu", "energy.cu", "gutter.cu",
              "segments.cu", "edges.cu", "report.cu", "dplan.cu", "pack.cu", "hier.cu"]
CXX_SOURCES = ["plan.cpp"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
              "-Xptxas", "-O3"]
# validation predicates are exact FP64: no FMA contraction in those files
NO_FMA = {"validate.cu", "gutter.cu", "segments.cu", "report.cu", "pack.cu"}


def _nvcc():
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found: the uva_b200 CUDA library cannot be built")


def _sources():
    cu = [s for s in CU_SOURCES if os.path.exists(os.path.join(CSRC, s))]
    return cu, list(CXX_SOURCES)


def _digest(files, flags):
    h = hashlib.sha256()
    for f in files:
        with open(f, "rb") as fh:
            h.update(fh.read())
    h.update(" ".join(flags).encode())
    return h.hexdigest()


def build_pyhost(force=False, verbose=False):
    """csrc/pyhost.cpp into PYHOST_LIB with g++ against this interpreter's
    headers (skipped when up to date). Returns the path, or None without a
    C++ compiler or Python headers."""
    import sysconfig
    src = os.path.join(CSRC, "pyhost.cpp")
    inc = sysconfig.get_paths().get("include")
    gxx = shutil.which("g++")
    if not (os.path.exists(src) and inc and os.path.exists(os.path.join(inc, "Python.h")) and gxx):
        return None
    digest = _digest([src], [inc, sys.version])
    stamp = PYHOST_LIB + ".sha256"
    if not force and os.path.exists(PYHOST_LIB) and os.path.exists(stamp):
        with open(stamp) as fh:
            if fh.read().strip() == digest:
                return PYHOST_LIB
    tmp = PYHOST_LIB + ".tmp"
    cmd = [gxx, "-O2", "-std=c++17", "-fPIC", "-shared", "-I", inc, src, "-o", tmp]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)
    os.replace(tmp, PYHOST_LIB)
    with open(stamp, "w") as fh:
        fh.write(digest)
    return PYHOST_LIB


def build(force=False, verbose=False):
    """Compile every CUDA / C++ source into LIB (skipped when up to date),
    and the batch constructor's host helper into PYHOST_LIB."""
    build_pyhost(force, verbose)
    cu, cxx = _sources()
    deps = [os.path.join(CSRC, s) for s in cu + cxx]
    deps += [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    deps += [os.path.join(INCLUDE, f) for f in os.listdir(INCLUDE) if f.endswith(".h")]
    deps.sort()
    digest = _digest(deps, ARCH + NVCC_FLAGS)
    stamp = LIB + ".sha256"
    if not force and os.path.exists(LIB) and os.path.exists(stamp):
        with open(stamp) as fh:
            if fh.read().strip() == digest:
                return LIB
    nvcc = _nvcc()
    os.makedirs(BUILD_DIR, exist_ok=True)
    objs = []
    for s in cu:
        obj = os.path.join(BUILD_DIR, s + ".o")
        flags = list(NVCC_FLAGS)
        if s in NO_FMA:
            flags += ["--fmad=false"]
        cmd = [nvcc, *ARCH, *flags, "-I", INCLUDE, "-c", os.path.join(CSRC, s), "-o", obj]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
        objs.append(obj)
    for s in cxx:
        obj = os.path.join(BUILD_DIR, s + ".o")
        cmd = [shutil.which("g++") or "g++", "-O3", "-std=c++17", "-fPIC", "-pthread", "-I", INCLUDE, "-c",
               os.path.join(CSRC, s), "-o", obj]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
        objs.append(obj)
    tmp = LIB + ".tmp"
    cmd = [nvcc, *ARCH, "-shared", "-o", tmp, *objs, "-lcudart", "-lpthread"]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)
    os.replace(tmp, LIB)
    with open(stamp, "w") as fh:
        fh.write(digest)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
