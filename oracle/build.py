"""Builds the CPU oracle (test infrastructure) as oracle/liboracle.so.

FP contraction is disabled so that the restated arithmetic is plain IEEE
double, the same rounding as the reference's host code on x86-64.
"""
from __future__ import annotations

import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
SRCS = [HERE / "oracle.cpp", HERE / "projection.cpp"]
LIB = HERE / "liboracle.so"


def build(force: bool = False) -> Path:
    if force or not LIB.exists() or any(s.stat().st_mtime > LIB.stat().st_mtime for s in SRCS):
        cmd = ["g++", "-O2", "-std=c++17", "-fopenmp", "-ffp-contract=off", "-fPIC", "-shared",
               *map(str, SRCS), "-o", str(LIB)]
        subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv)
    print(LIB)
