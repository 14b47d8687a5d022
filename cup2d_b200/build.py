"""Builds libcup2d_poisson.so in-tree for sm_100a with nvcc.

Usage: python -m cup2d_b200.build [--force] [--verbose]
"""
from __future__ import annotations

import argparse
import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
INCLUDE = PKG.parent / "include"
BUILD = PKG / "_build"
LIB = PKG / "libcup2d_poisson.so"

SOURCES = ["assemble.cu", "adapt.cu", "bicgstab.cu", "capi.cu", "noalloc.cu", "precond_tc.cu", "projection.cu",
           "server.cu", "timestep.cu", "spmv_staged.cu", "problems.cpp", "forest.cpp"]
# files whose arithmetic must round like a plain IEEE evaluation (no FMA)
FILE_FLAGS = {"projection.cu": ["--fmad=false"]}
HEADERS = ["common.cuh", "kernels.hpp", "spmv.cuh", "handle_view.hpp", "forest.hpp"]

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "--expt-relaxed-constexpr",
              "-Xcompiler", "-fPIC,-fopenmp,-O3", "-I", str(INCLUDE)]


def nvcc() -> str:
    cand = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not Path(cand).exists():
        raise RuntimeError("nvcc not found: the CUDA toolkit is required to build cup2d_b200")
    return cand


def _stale(target: Path, deps: list[Path]) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def build(force: bool = False, verbose: bool = False, ptxas_verbose: bool = False) -> Path:
    BUILD.mkdir(exist_ok=True)
    hdrs = [CSRC / h for h in HEADERS] + [INCLUDE / "cup2d_poisson.h"]
    objs = []
    for src in SOURCES:
        s = CSRC / src
        o = BUILD / (src + ".o")
        objs.append(o)
        if force or _stale(o, [s] + hdrs):
            cmd = [nvcc(), *ARCH, *NVCC_FLAGS, *FILE_FLAGS.get(src, []), "-c", str(s), "-o", str(o)]
            if ptxas_verbose and src.endswith(".cu"):
                cmd += ["-Xptxas", "-v"]
            if verbose:
                print(" ".join(cmd), flush=True)
            subprocess.run(cmd, check=True)
    if force or _stale(LIB, objs):
        cmd = [nvcc(), *ARCH, "-shared", "-o", str(LIB), *map(str, objs),
               "-Xcompiler", "-fopenmp", "-lgomp"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    return LIB


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose", action="store_true")
    ap.add_argument("--ptxas", action="store_true", help="print -Xptxas -v resource usage")
    a = ap.parse_args(argv)
    build(force=a.force, verbose=a.verbose, ptxas_verbose=a.ptxas)
    print(LIB)
    return 0


if __name__ == "__main__":
    sys.exit(main())
