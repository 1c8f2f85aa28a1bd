"""Build the C part of the oracle (test infrastructure only) into
oracle/liboracle_c.so with gcc, without floating-point contraction; the
overlap scan runs its cells on OpenMP threads (OMP_NUM_THREADS), as the
reference's numba prange does.

    python oracle/build_oracle.py
"""
from __future__ import annotations

import os
import shutil
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "c", "uva_oracle.c")
LIB = os.path.join(HERE, "liboracle_c.so")


def build(force=False):
    if not force and os.path.exists(LIB) and os.path.getmtime(LIB) >= os.path.getmtime(SRC):
        return LIB
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        raise RuntimeError("gcc not found: cannot build the C oracle")
    tmp = LIB + ".tmp"
    subprocess.run([cc, "-O2", "-ffp-contract=off", "-fno-fast-math", "-fopenmp", "-fPIC", "-shared", SRC, "-o", tmp,
                    "-lm"], check=True)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(force=True))
