"""ORACLE — test infrastructure only.  ctypes binding of the reference checker
in oracle/_ref/ (built by oracle/ref/build.py from CUP2D's own Poisson sources):

  assemble(mesh)  CPU build: the reference's P^-1 and the COO system its
                  getMat/LocalSpMatDnVec produce for the mesh (rows ascending,
                  columns ascending within a row), plus b, x0, h^2.
  solve(mesh, b)  GPU build: ExpAMRSolver::solve end to end with the
                  reference's cuBLAS/cuSPARSE BiCGSTAB (BiCGSTAB.cu:412-620),
                  returning the mean-removed solution and the statistics the
                  solver prints (parsed from its log).

Only tests/ and the fixture script under tests/golden/ use it.
"""
from __future__ import annotations

import ctypes as C
import re
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
OUT = HERE.parent / "_ref"
CPU_LIB = OUT / "liboracle_ref_cpu.so"
GPU_LIB = OUT / "liboracle_ref_gpu.so"


class RefForest(C.Structure):
    _fields_ = [("bpdx", C.c_int32), ("bpdy", C.c_int32), ("level_max", C.c_int32),
                ("periodic_x", C.c_int32), ("periodic_y", C.c_int32), ("extent", C.c_double),
                ("nblocks", C.c_int64), ("level", C.POINTER(C.c_int32)), ("bx", C.POINTER(C.c_int32)),
                ("by", C.POINTER(C.c_int32))]


_libs: dict[str, C.CDLL] = {}


def available(kind: str = "cpu") -> bool:
    """Whether the checker library of that kind is built (building it first
    when the reference tree is present)."""
    try:
        _load(kind)
        return True
    except OSError:
        return False


def _load(kind: str) -> C.CDLL:
    if kind in _libs:
        return _libs[kind]
    path = CPU_LIB if kind == "cpu" else GPU_LIB
    from . import build as _b
    _b.build(cpu_only=(kind == "cpu"))
    if not path.exists():
        raise OSError(f"reference checker {path.name} is not built (the reference tree is needed to build it)")
    L = C.CDLL(str(path))
    pd = C.POINTER(C.c_double)
    L.ref_solve.restype = C.c_int
    L.ref_solve.argtypes = [C.POINTER(RefForest), pd, pd, C.c_double, C.c_double, C.c_int, C.c_int,
                            C.c_char_p, C.c_int64]
    L.ref_solve_mc.restype = C.c_int
    L.ref_solve_mc.argtypes = [C.POINTER(RefForest), pd, pd, C.c_double, C.c_double, C.c_int, C.c_int, C.c_int,
                               C.c_char_p, C.c_int64]
    L.ref_mean_row.restype = C.c_int
    L.ref_copy_pinv.restype = C.c_int
    L.ref_copy_pinv.argtypes = [pd]
    L.ref_system_size.restype = C.c_int
    L.ref_system_size.argtypes = [C.POINTER(C.c_int64), C.POINTER(C.c_int64)]
    L.ref_copy_system.restype = C.c_int
    L.ref_copy_system.argtypes = [C.POINTER(C.c_int32), C.POINTER(C.c_int32), pd, pd, pd, pd]
    _libs[kind] = L
    return L


def _forest(mesh):
    arrs = tuple(np.ascontiguousarray(a, dtype=np.int32) for a in (mesh.level, mesh.bx, mesh.by))
    f = RefForest(mesh.bpdx, mesh.bpdy, mesh.level_max, int(mesh.periodic_x), int(mesh.periodic_y),
                  float(mesh.extent), mesh.nblocks, *(a.ctypes.data_as(C.POINTER(C.c_int32)) for a in arrs))
    return f, arrs


def _pd(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _run(L, mesh, b, x, tol_abs, tol_rel, max_restarts, step, mean_constraint=0):
    f, keep = _forest(mesh)
    buf = C.create_string_buffer(1 << 20)
    rc = L.ref_solve_mc(C.byref(f), _pd(b), _pd(x), tol_abs, tol_rel, max_restarts, step, int(mean_constraint), buf,
                        len(buf))
    log = buf.value.decode(errors="replace")
    if rc != 0:
        raise RuntimeError("reference checker failed: " + log.strip().splitlines()[-1] if log.strip() else "")
    return log


def assemble(mesh, b: np.ndarray | None = None, mean_constraint: int = 0) -> dict:
    """The reference's P^-1 and assembled system for the mesh (CPU build);
    with mean_constraint also the row getMat picks ("mean_row")."""
    L = _load("cpu")
    n = mesh.nblocks * 64
    b = np.zeros(n) if b is None else np.ascontiguousarray(b, dtype=np.float64)
    x = np.zeros(n)
    _run(L, mesh, b, x, 0.0, 0.0, 100, 10, mean_constraint)
    mean_row = int(L.ref_mean_row())
    P = np.empty(64 * 64)
    if L.ref_copy_pinv(_pd(P)) != 0:
        raise RuntimeError("reference checker recorded no P^-1")
    m, nnz = C.c_int64(), C.c_int64()
    if L.ref_system_size(C.byref(m), C.byref(nnz)) != 0:
        raise RuntimeError("reference checker recorded no system")
    row = np.empty(nnz.value, dtype=np.int32)
    col = np.empty(nnz.value, dtype=np.int32)
    val = np.empty(nnz.value)
    bb, x0, h2 = np.empty(m.value), np.empty(m.value), np.empty(m.value // 64)
    L.ref_copy_system(row.ctypes.data_as(C.POINTER(C.c_int32)), col.ctypes.data_as(C.POINTER(C.c_int32)),
                      _pd(val), _pd(bb), _pd(x0), _pd(h2))
    return {"pinv": P.reshape(64, 64), "row": row, "col": col, "val": val, "b": bb, "x0": x0, "h2": h2,
            "mean_row": mean_row}


_NUM = r"([-+0-9.eE]+|inf|nan)"


def parse_log(log: str) -> dict:
    """Statistics from the reference solver's progress lines
    (BiCGSTAB.cu:449-452,490-493,549,600-606).  `iterations` counts completed
    iterations: the solver prints the 0-based index of the converging one."""
    st = {"norm_ax0": None, "err_init": None, "err_opt": None, "iterations": None, "converged": False,
          "restarts": len(re.findall(r"Restart at iteration", log))}
    m = re.search(r"\|\| A\*x_0 \|\| = " + _NUM, log)
    if m:
        st["norm_ax0"] = float(m.group(1))
    m = re.search(r"Initial norm: " + _NUM, log)
    if m:
        st["err_init"] = float(m.group(1))
    m = re.search(r"Converged after (\d+) iterations", log)
    if m:
        st["converged"] = True
        st["iterations"] = int(m.group(1)) + 1
    m = re.search(r"Iteration (\d+)\. Error norm", log)
    if m:
        st["iterations"] = int(m.group(1))
    m = re.search(r"Error norm \(relative\) = " + _NUM, log)
    if m:
        st["err_opt"] = float(m.group(1))
    return st


def solve(mesh, b: np.ndarray, x0: np.ndarray | None = None, tol_abs: float = 0.0, tol_rel: float = 1e-8,
          max_restarts: int = 100, mean_constraint: int = 0) -> tuple[np.ndarray, dict]:
    """ExpAMRSolver::solve with the reference's GPU BiCGSTAB (GPU build).  The
    call runs with sim.step = 10, where the caller's tolerances apply, and
    sim.bMeanConstraint = mean_constraint."""
    L = _load("gpu")
    b = np.ascontiguousarray(b, dtype=np.float64)
    x = np.zeros(mesh.nblocks * 64) if x0 is None else np.array(x0, dtype=np.float64, copy=True)
    log = _run(L, mesh, b, x, tol_abs, tol_rel, max_restarts, 10, mean_constraint)
    st = parse_log(log)
    st["log"] = log
    return x, st
