"""ORACLE — test infrastructure only.  Builds the reference checker from
CUP2D's own Poisson sources, compiled unchanged where they lie in the
reference tree, into oracle/_ref/:

  liboracle_ref_cpu.so  ExpAMRSolver.cpp + LocalSpMatDnVec.cpp (g++) with the
                        capture stand-in of BiCGSTABSolver (no GPU needed):
                        the reference's P^-1 and assembled COO system.
  liboracle_ref_gpu.so  the same plus the reference's BiCGSTAB.cu (nvcc,
                        sm_100a, cuBLAS + cuSPARSE + cub): the reference's own
                        FP64 solve, end to end through ExpAMRSolver::solve.

What stands in for what CUP2D links against (all of it our own code):
  * Cubism (un-vendored submodule): oracle/ref/standin/Cubism/*.h;
  * MPI: oracle/ref/standin/mpi.h, one rank;
  * source/include/helper_cuda.h: oracle/ref/cuda_check.h, force-included, whose
    include guard turns the reference's #include of that header into a no-op;
  * CUDA 12.9's cusparse.h has no CUSPARSE_MV_ALG_DEFAULT (the reference's
    SpMV algorithm enum, BiCGSTAB.cu:234,249,345,383), so it is defined as
    CUSPARSE_SPMV_ALG_DEFAULT, the value that replaced it.

Arithmetic: plain IEEE double (-O2, no -ffast-math, no FMA contraction); the
reference's Release configuration adds -ffast-math -march=native
(CMakeLists.txt:93-95), which would let the compiler reorder the same
operations.

The reference tree is read from $CUP2D_REFERENCE (default /root/reference);
where it is absent (a machine that only runs the tests) the libraries already
built in oracle/_ref/ are used as they are.

Usage: python -m oracle.ref.build [--force] [--cpu-only]
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
OUT = HERE.parent / "_ref"
REFERENCE = Path(os.environ.get("CUP2D_REFERENCE", "/root/reference"))
POISSON = REFERENCE / "source" / "Poisson"
CPU_LIB = OUT / "liboracle_ref_cpu.so"
GPU_LIB = OUT / "liboracle_ref_gpu.so"
CUDA = Path(os.environ.get("CUDA_HOME", "/usr/local/cuda"))

DEFS = ["-D_DOUBLE_PRECISION_", "-D_BS_=8", "-DDIMENSION=2", "-DGPU_POISSON",
        "-DCUSPARSE_MV_ALG_DEFAULT=CUSPARSE_SPMV_ALG_DEFAULT"]
INCS = ["-I", str(HERE / "standin"), "-I", str(HERE), "-I", str(POISSON), "-I", str(CUDA / "include")]
FORCE = ["-include", str(HERE / "cuda_check.h")]
CXX = ["g++", "-O2", "-std=c++17", "-fPIC", "-fopenmp", "-ffp-contract=off", "-w"]


def reference_present() -> bool:
    return (POISSON / "ExpAMRSolver.cpp").exists()


def _deps() -> list[Path]:
    own = [HERE / "ref_driver.cpp", HERE / "solver_capture.cpp", HERE / "ref_capture.hpp",
           HERE / "cuda_check.h", HERE / "standin" / "mpi.h", HERE / "standin" / "cubism_standin.hpp"]
    ref = [POISSON / n for n in ("ExpAMRSolver.cpp", "ExpAMRSolver.h", "LocalSpMatDnVec.cpp",
                                 "LocalSpMatDnVec.h", "BiCGSTAB.cu", "BiCGSTAB.cuh")]
    return own + ref


def _stale(target: Path) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(d.exists() and d.stat().st_mtime > t for d in _deps())


def _run(cmd: list[str], verbose: bool) -> None:
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)


def _objects(verbose: bool) -> dict[str, Path]:
    OUT.mkdir(exist_ok=True)
    objs = {}
    for name, src in (("exp", POISSON / "ExpAMRSolver.cpp"), ("lsm", POISSON / "LocalSpMatDnVec.cpp"),
                      ("drv", HERE / "ref_driver.cpp"), ("cap", HERE / "solver_capture.cpp")):
        o = OUT / f"{name}.o"
        _run([*CXX, *DEFS, *INCS, *FORCE, "-c", str(src), "-o", str(o)], verbose)
        objs[name] = o
    return objs


def build(force: bool = False, cpu_only: bool = False, verbose: bool = False) -> Path | None:
    """Builds the checker libraries when the reference tree is present and
    they are missing or stale; returns the CPU library path (None when it
    neither exists nor can be built)."""
    if not reference_present():
        return CPU_LIB if CPU_LIB.exists() else None
    want_gpu = not cpu_only and shutil.which("nvcc") is not None
    if not (force or _stale(CPU_LIB) or (want_gpu and _stale(GPU_LIB))):
        return CPU_LIB
    objs = _objects(verbose)
    _run([*CXX, "-shared", "-o", str(CPU_LIB), str(objs["exp"]), str(objs["lsm"]), str(objs["drv"]),
          str(objs["cap"])], verbose)
    if want_gpu:
        bic = OUT / "bicgstab.o"
        _run(["nvcc", "-gencode", "arch=compute_100a,code=sm_100a", "-O2", "-std=c++17", "-w",
              "-Xcompiler", "-fPIC", *DEFS, *INCS, *FORCE, "-c", str(POISSON / "BiCGSTAB.cu"), "-o", str(bic)],
             verbose)
        _run(["nvcc", "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-o", str(GPU_LIB),
              str(objs["exp"]), str(objs["lsm"]), str(objs["drv"]), str(bic),
              "-L", str(CUDA / "lib64"), "-lcublas", "-lcusparse", "-Xcompiler", "-fopenmp", "-lgomp"], verbose)
    for o in OUT.glob("*.o"):
        o.unlink()
    return CPU_LIB


if __name__ == "__main__":
    lib = build(force="--force" in sys.argv, cpu_only="--cpu-only" in sys.argv, verbose=True)
    print(lib if lib else "reference tree absent and no prebuilt checker")
