"""Build the native library (sm_100a CUDA + C++ host code) in-tree.

    python -m iitmglobalrouter_b200.build          # library + route CLI
    python -m iitmglobalrouter_b200.build --force

Outputs (git-ignored, shipped with the source tree):
    iitmglobalrouter_b200/lib/libiitmgr_b200.so   C ABI of include/iitmgr_b200.h
    iitmglobalrouter_b200/lib/route               the `route` command line tool
"""
from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
LIB_DIR = PKG / "lib"
LIB = LIB_DIR / "libiitmgr_b200.so"
ROUTE_BIN = LIB_DIR / "route"

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CUDA_FLAGS = ARCH + [
    "-O3", "-lineinfo", "-std=c++17", "--expt-relaxed-constexpr",
    "-Xcompiler", "-fPIC,-O3,-fopenmp", "-I", str(ROOT / "include"),
]
CXX = os.environ.get("GR_CXX", "g++")
CXX_FLAGS = ["-O3", "-std=c++20", "-fPIC", "-fopenmp", "-I", str(ROOT / "include")]

LIB_CU = ["gr_capi.cu", "gr_cnn.cu"]
LIB_CPP = ["gr_io.cpp", "gr_io_capi.cpp"]
HEADERS = ["gr_device.cuh", "gr_kernels.cuh", "gr_io.hpp"]


def _newer(target: Path, deps) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(Path(d).exists() and Path(d).stat().st_mtime > t for d in deps)


def _run(cmd, verbose):
    if verbose:
        print(" ".join(str(c) for c in cmd), flush=True)
    subprocess.run([str(c) for c in cmd], check=True)


def build(force: bool = False, verbose: bool = False) -> Path:
    LIB_DIR.mkdir(exist_ok=True)
    obj_dir = LIB_DIR / "_obj"
    obj_dir.mkdir(exist_ok=True)
    hdrs = [CSRC / h for h in HEADERS if (CSRC / h).exists()] + [ROOT / "include" / "iitmgr_b200.h"]
    objs = []
    for name in LIB_CU:
        src = CSRC / name
        obj = obj_dir / (name + ".o")
        if force or _newer(obj, [src, *hdrs]):
            _run([NVCC, *CUDA_FLAGS, "-c", src, "-o", obj], verbose)
        objs.append(obj)
    for name in LIB_CPP:
        src = CSRC / name
        if not src.exists():
            continue
        obj = obj_dir / (name + ".o")
        if force or _newer(obj, [src, *hdrs]):
            _run([CXX, *CXX_FLAGS, "-c", src, "-o", obj], verbose)
        objs.append(obj)
    if force or _newer(LIB, objs):
        _run([NVCC, *ARCH, "-shared", "-Xcompiler", "-fopenmp", *objs, "-o", LIB], verbose)
    main_src = CSRC / "route_main.cpp"
    if main_src.exists() and (force or _newer(ROUTE_BIN, [main_src, LIB, *hdrs])):
        _run([CXX, *CXX_FLAGS, main_src, "-o", ROUTE_BIN, "-L", LIB_DIR, "-liitmgr_b200",
              "-Wl,-rpath,$ORIGIN"], verbose)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
