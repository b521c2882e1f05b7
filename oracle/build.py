"""Build the CPU oracle (test infrastructure) into oracle/_build/.

    python oracle/build.py

Strict IEEE single precision: no fast-math, no FMA contraction, so the
oracle performs the same FP32 additions in the same order as the reference
code it restates.
"""
from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
OUT = HERE / "_build"
LIB = OUT / "libgr_oracle.so"
SRC = [HERE / "gr_oracle.c"]
HDR = [HERE / "gr_oracle.h"]


def build(force: bool = False, verbose: bool = False) -> Path:
    OUT.mkdir(exist_ok=True)
    if not force and LIB.exists():
        t = LIB.stat().st_mtime
        if all(p.stat().st_mtime <= t for p in SRC + HDR):
            return LIB
    cmd = [os.environ.get("GR_CC", "gcc"), "-O2", "-fPIC", "-shared", "-fopenmp", "-ffp-contract=off",
           "-fno-fast-math", "-std=c11", *map(str, SRC), "-o", str(LIB), "-lm"]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
