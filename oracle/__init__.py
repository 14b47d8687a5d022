"""ORACLE — test infrastructure only (reference for the parity tests and timed CPU baseline).

ctypes binding of oracle/liboracle.so, the CPU FP64 restatement of CUP2D's
GPU Poisson path (see oracle.cpp for the reference lines it follows).  Only
tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use it; the
product library never does.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "liboracle.so"


class OracleForest(C.Structure):
    _fields_ = [("bpdx", C.c_int32), ("bpdy", C.c_int32), ("level_max", C.c_int32),
                ("periodic_x", C.c_int32), ("periodic_y", C.c_int32), ("extent", C.c_double),
                ("nblocks", C.c_int64), ("level", C.POINTER(C.c_int32)), ("bx", C.POINTER(C.c_int32)),
                ("by", C.POINTER(C.c_int32))]


class OracleStats(C.Structure):
    _fields_ = [("iterations", C.c_int32), ("restarts", C.c_int32), ("converged", C.c_int32),
                ("hit_max_iter", C.c_int32), ("err_init", C.c_double), ("err_opt", C.c_double),
                ("norm_ax0", C.c_double)]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


_lib = None


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            from . import build as _b  # noqa: F401  (oracle/build.py)
            _b.build()
        L = C.CDLL(str(LIB_PATH))
        pf = C.POINTER(C.c_double)
        L.oracle_num_threads.restype = C.c_int
        L.oracle_set_threads.argtypes = [C.c_int]
        L.oracle_pinv.argtypes = [pf]
        L.oracle_assemble.restype = C.c_void_p
        L.oracle_assemble.argtypes = [C.POINTER(OracleForest)]
        L.oracle_matrix_n.restype = C.c_int64
        L.oracle_matrix_n.argtypes = [C.c_void_p]
        L.oracle_matrix_nnz.restype = C.c_int64
        L.oracle_matrix_nnz.argtypes = [C.c_void_p]
        L.oracle_matrix_copy.argtypes = [C.c_void_p, C.POINTER(C.c_int64), C.POINTER(C.c_int32), pf]
        L.oracle_matrix_free.argtypes = [C.c_void_p]
        L.oracle_spmv.argtypes = [C.c_void_p, pf, pf]
        L.oracle_precond.argtypes = [C.c_int64, pf, pf, pf]
        L.oracle_bicgstab.restype = C.c_int
        L.oracle_bicgstab.argtypes = [C.c_void_p, pf, pf, pf, C.c_double, C.c_double, C.c_int, C.c_int,
                                      C.POINTER(OracleStats)]
        L.oracle_subtract_mean.argtypes = [C.c_int64, pf, pf]
        L.oracle_bicgstab_mean.restype = C.c_int
        L.oracle_bicgstab_mean.argtypes = [C.c_void_p, pf, pf, pf, C.c_double, C.c_double, C.c_int, C.c_int,
                                           C.c_int64, pf, C.POINTER(OracleStats)]
        L.oracle_pressure_rhs.restype = C.c_int
        L.oracle_pressure_rhs.argtypes = [C.POINTER(OracleForest), C.c_double, pf, pf, pf, pf, pf, pf]
        L.oracle_pressure_correction.restype = C.c_int
        L.oracle_pressure_correction.argtypes = [C.POINTER(OracleForest), C.c_double, pf, pf]
        _lib = L
    return _lib


def _pd(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def set_threads(n: int) -> None:
    lib().oracle_set_threads(int(n))


def num_threads() -> int:
    return int(lib().oracle_num_threads())


def pinv() -> np.ndarray:
    P = np.empty(64 * 64, dtype=np.float64)
    lib().oracle_pinv(_pd(P))
    return P.reshape(64, 64)


def _forest(mesh):
    arrs = (np.ascontiguousarray(mesh.level, dtype=np.int32), np.ascontiguousarray(mesh.bx, dtype=np.int32),
            np.ascontiguousarray(mesh.by, dtype=np.int32))
    f = OracleForest(mesh.bpdx, mesh.bpdy, mesh.level_max, int(mesh.periodic_x), int(mesh.periodic_y),
                     float(mesh.extent), mesh.nblocks, *(a.ctypes.data_as(C.POINTER(C.c_int32)) for a in arrs))
    return f, arrs


def _opt(a):
    return None if a is None else _pd(a)


def pressure_rhs(mesh, dt: float, vel=None, udef=None, chi=None, pres=None, tmp=None):
    """PressureSingle.cpp:826-849 before the solve (oracle/projection.cpp).

    vel/udef: (ncells, 2) velocities, chi: (ncells,).  Returns (tmp, pold):
    tmp = updatePressureRHS of the velocities (when vel is given, else the
    given tmp), minus updatePressureRHS1 of pres (when pres is given), and
    pold = pres."""
    n = mesh.ncells
    f, keep = _forest(mesh)
    out = np.zeros(n) if tmp is None else np.array(tmp, dtype=np.float64, copy=True)
    vel = None if vel is None else np.ascontiguousarray(vel, dtype=np.float64).reshape(n, 2)
    udef = None if udef is None else np.ascontiguousarray(udef, dtype=np.float64).reshape(n, 2)
    chi = None if chi is None else np.ascontiguousarray(chi, dtype=np.float64)
    pres = None if pres is None else np.ascontiguousarray(pres, dtype=np.float64)
    pold = None if pres is None else np.empty(n)
    if lib().oracle_pressure_rhs(C.byref(f), float(dt), _opt(vel), _opt(udef), _opt(chi), _opt(pres), _pd(out),
                                 _opt(pold)) != 0:
        raise ValueError("oracle: malformed forest")
    del keep
    return out, pold


def pressure_correction(mesh, dt: float, pres, vel):
    """PressureSingle::pressureCorrection: returns vel + tmpV / h^2."""
    n = mesh.ncells
    f, keep = _forest(mesh)
    pres = np.ascontiguousarray(pres, dtype=np.float64)
    out = np.array(vel, dtype=np.float64, copy=True).reshape(n, 2)
    if lib().oracle_pressure_correction(C.byref(f), float(dt), _pd(pres), _pd(out)) != 0:
        raise ValueError("oracle: malformed forest")
    del keep
    return out


class Matrix:
    """The explicit operator of ExpAMRSolver::getMat for one forest."""

    def __init__(self, mesh):
        self._arrs = (np.ascontiguousarray(mesh.level, dtype=np.int32),
                      np.ascontiguousarray(mesh.bx, dtype=np.int32),
                      np.ascontiguousarray(mesh.by, dtype=np.int32))
        f = OracleForest(mesh.bpdx, mesh.bpdy, mesh.level_max, int(mesh.periodic_x), int(mesh.periodic_y),
                         float(mesh.extent), mesh.nblocks,
                         *(a.ctypes.data_as(C.POINTER(C.c_int32)) for a in self._arrs))
        self._h = lib().oracle_assemble(C.byref(f))
        if not self._h:
            raise ValueError("oracle: malformed forest")
        self.n = int(lib().oracle_matrix_n(self._h))
        self.nnz = int(lib().oracle_matrix_nnz(self._h))
        self.nblocks = self.n // 64

    def __del__(self):
        h = getattr(self, "_h", None)
        if h and _lib is not None:
            _lib.oracle_matrix_free(h)
            self._h = None

    def csr(self):
        rp = np.empty(self.n + 1, dtype=np.int64)
        col = np.empty(self.nnz, dtype=np.int32)
        val = np.empty(self.nnz, dtype=np.float64)
        lib().oracle_matrix_copy(self._h, rp.ctypes.data_as(C.POINTER(C.c_int64)),
                                 col.ctypes.data_as(C.POINTER(C.c_int32)), _pd(val))
        return rp, col, val

    def scipy(self):
        import scipy.sparse as sp
        rp, col, val = self.csr()
        return sp.csr_matrix((val, col, rp), shape=(self.n, self.n))

    def spmv(self, x: np.ndarray) -> np.ndarray:
        x = np.ascontiguousarray(x, dtype=np.float64)
        y = np.empty(self.n, dtype=np.float64)
        lib().oracle_spmv(self._h, _pd(x), _pd(y))
        return y

    def bicgstab(self, b: np.ndarray, x0: np.ndarray | None = None, tol_abs: float = 0.0,
                 tol_rel: float = 1e-8, max_restarts: int = 100, max_iter: int = 1000,
                 P: np.ndarray | None = None, mean_row: int = -1, h_block: np.ndarray | None = None):
        """BiCGSTABSolver::main; returns (x_opt, stats dict).  mean_row >= 0:
        the bMeanConstraint SpMV (that row is sum h^2 x, h_block per block)."""
        b = np.ascontiguousarray(b, dtype=np.float64)
        x = np.zeros(self.n) if x0 is None else np.array(x0, dtype=np.float64, copy=True)
        P = pinv() if P is None else np.ascontiguousarray(P, dtype=np.float64)
        st = OracleStats()
        if mean_row >= 0:
            h = np.ascontiguousarray(h_block, dtype=np.float64)
            lib().oracle_bicgstab_mean(self._h, _pd(P), _pd(b), _pd(x), tol_abs, tol_rel, max_restarts, max_iter,
                                       int(mean_row), _pd(h), C.byref(st))
        else:
            lib().oracle_bicgstab(self._h, _pd(P), _pd(b), _pd(x), tol_abs, tol_rel, max_restarts, max_iter,
                                  C.byref(st))
        return x, st.as_dict()


def precond(P: np.ndarray, p: np.ndarray) -> np.ndarray:
    p = np.ascontiguousarray(p, dtype=np.float64)
    z = np.empty_like(p)
    P = np.ascontiguousarray(P, dtype=np.float64)
    lib().oracle_precond(p.shape[0] // 64, _pd(P), _pd(p), _pd(z))
    return z


def subtract_mean(h_block: np.ndarray, x: np.ndarray) -> np.ndarray:
    x = np.array(x, dtype=np.float64, copy=True)
    h = np.ascontiguousarray(h_block, dtype=np.float64)
    lib().oracle_subtract_mean(h.shape[0], _pd(h), _pd(x))
    return x


def mean_row(mesh) -> int:
    """bMeanConstraint's row: cell (0,0) of the leaf whose index is (0,0)
    (ExpAMRSolver.cpp:251-256)."""
    blk = np.flatnonzero((np.asarray(mesh.bx) == 0) & (np.asarray(mesh.by) == 0))
    if blk.size != 1:
        raise ValueError("oracle: no single leaf at the domain's corner")
    return int(blk[0]) * 64


def solve(mesh, b: np.ndarray, x0=None, tol_abs=0.0, tol_rel=1e-8, max_restarts=100, max_iter=1000,
          subtract_mean_=True, mean_constraint=False):
    """ExpAMRSolver::solve end to end on the CPU: assemble, BiCGSTAB, mean removal.
    mean_constraint: getVec writes 0 into the mean row of b and the solver
    runs the bMeanConstraint SpMV."""
    A = Matrix(mesh)
    if mean_constraint:
        row = mean_row(mesh)
        b = np.array(b, dtype=np.float64, copy=True)
        b[row] = 0.0
        x, st = A.bicgstab(b, x0, tol_abs, tol_rel, max_restarts, max_iter, mean_row=row, h_block=mesh.cell_h())
    else:
        x, st = A.bicgstab(b, x0, tol_abs, tol_rel, max_restarts, max_iter)
    if subtract_mean_:
        x = subtract_mean(mesh.cell_h(), x)
    return x, st
