"""Recipe: build the reference router's own -bit_pmodel code path into
oracle/_ref/ref_harness (TEST INFRASTRUCTURE ONLY).

    python -m oracle.ref.build_ref [--reference /root/reference] [--force]

The reference (SammithKanur/iitmGlobalRouter) is one header-only CUDA C++
program; ref_harness.cu includes its headers where they lie and runs its
reader, batcher, per-batch GPU path and route writer (see that file). Two
of its dependencies are not in this image as such and are replaced at
compile time, without touching the reference's files:
  * Boost.Geometry (point, box, rtree + intersects, used by the batcher):
    oracle/ref/shim/boost/geometry.hpp, a linear-scan stand-in with Boost's
    closed-box intersection rule;
  * fmt (through spdlog): spdlog 1.14.1's headers as shipped in this image
    (flashinfer's data directory) with its std::format backend, plus
    oracle/ref/shim/ref_compat.h (fmt::format as std::format, a formatter
    for cudaError_t, <map> and <set>).
Built for sm_100a directly (the reference's build.sh targets sm_80) with
NDEBUG, so no device-side assert can stop a kernel. The binary is written to
oracle/_ref/ (git-ignored; it travels with the tree to a GPU machine, where
tests/golden/make_ref_fixtures.py drives it). Nothing in the product, the
GPU tests or the benchmark runs it.
"""
from __future__ import annotations

import argparse
import os
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
OUT = ROOT / "oracle" / "_ref"
BIN = OUT / "ref_harness"
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")


def spdlog_include() -> Path | None:
    for p in sys.path:
        cand = Path(p) / "flashinfer" / "data" / "spdlog" / "include"
        if (cand / "spdlog" / "spdlog.h").exists():
            return cand
    return None


def build(reference: str = "/root/reference", force: bool = False, verbose: bool = False) -> Path | None:
    """Returns the binary, or None when the reference tree or spdlog is absent."""
    ref = Path(reference)
    if not (ref / "main.cpp").exists():
        if verbose:
            print(f"build_ref: no reference tree at {ref}; skipped")
        return None
    spd = spdlog_include()
    if spd is None:
        if verbose:
            print("build_ref: spdlog headers not found; skipped")
        return None
    OUT.mkdir(parents=True, exist_ok=True)
    src = HERE / "ref_harness.cu"
    deps = [src, HERE / "shim" / "ref_compat.h", HERE / "shim" / "boost" / "geometry.hpp", Path(__file__)]
    deps += list(ref.rglob("*.hpp")) + list(ref.rglob("*.h"))
    if not force and BIN.exists() and all(BIN.stat().st_mtime >= d.stat().st_mtime for d in deps if d.exists()):
        return BIN
    cmd = [NVCC, "-std=c++20", "-x", "cu", "-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-DNDEBUG",
           "-DSPDLOG_USE_STD_FORMAT", "-Xcompiler", "-fopenmp", "-w",
           "-I", str(HERE / "shim"), "-I", str(spd), "-I", str(ref),
           "-include", str(HERE / "shim" / "ref_compat.h"), str(src), "-o", str(BIN), "-lgomp"]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)
    return BIN


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default="/root/reference")
    ap.add_argument("--force", action="store_true")
    a = ap.parse_args()
    print(build(a.reference, a.force, verbose=True))
