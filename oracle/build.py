"""Build recipe of the oracle's C restatement (test infrastructure only).

``python -m oracle.build`` compiles ``oracle/loop_ref.c`` with gcc into
``oracle/_build/liboracle_ref.so`` (OpenMP, no FMA contraction, no fast-math).
The reference itself is MATLAB/GNU Octave and has nothing to compile, so there
is no ``oracle/_ref`` build.
"""
from __future__ import annotations

import os
import shutil
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
OUT_DIR = os.path.join(HERE, "_build")
LIB = os.path.join(OUT_DIR, "liboracle_ref.so")
SRC = os.path.join(HERE, "loop_ref.c")


def build(force: bool = False) -> str:
    if not force and os.path.exists(LIB) and os.path.getmtime(LIB) >= os.path.getmtime(SRC):
        return LIB
    os.makedirs(OUT_DIR, exist_ok=True)
    # the system gcc carries the OpenMP runtime; a gcc wrapper named by $CC may not
    cands = [c for c in ("/usr/bin/gcc", os.environ.get("CC"), shutil.which("gcc"), "cc") if c]
    err = None
    for cc in dict.fromkeys(cands):
        cmd = [cc, "-O2", "-fopenmp", "-ffp-contract=off", "-fno-fast-math", "-shared", "-fPIC",
               "-o", LIB + ".tmp", SRC]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode == 0:
            os.replace(LIB + ".tmp", LIB)
            return LIB
        err = r.stderr
    raise RuntimeError(f"could not build {LIB}:\n{err}")


if __name__ == "__main__":
    print(build(force=True))
