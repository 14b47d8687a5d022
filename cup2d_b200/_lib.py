"""ctypes binding of libcup2d_poisson.so (the C ABI in include/cup2d_poisson.h).

The library is loaded from this package directory.  There is no fallback:
if it is missing, importing the solver raises.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "libcup2d_poisson.so"

OK, NOT_CONVERGED, BREAKDOWN_LIMIT, BAD_MESH, OOM, TIMEOUT, CUDA_ERROR, INVALID_ARGUMENT, \
    NO_DEVICE, QUEUE_FULL, PENDING = range(11)
PREC_FP64, PREC_MIXED = 0, 1
GRAPH_ZERO_X = 1

P_i32 = C.POINTER(C.c_int32)
P_i64 = C.POINTER(C.c_int64)
P_f64 = C.POINTER(C.c_double)
P_f32 = C.POINTER(C.c_float)


class Forest(C.Structure):
    _fields_ = [("bpdx", C.c_int32), ("bpdy", C.c_int32), ("level_max", C.c_int32),
                ("periodic_x", C.c_int32), ("periodic_y", C.c_int32), ("extent", C.c_double),
                ("nblocks", C.c_int64), ("level", P_i32), ("bx", P_i32), ("by", P_i32)]


class SolveOpts(C.Structure):
    _fields_ = [("tol_abs", C.c_double), ("tol_rel", C.c_double), ("max_restarts", C.c_int32),
                ("max_iter", C.c_int32), ("precision", C.c_int32), ("subtract_mean", C.c_int32),
                ("reliable_delta", C.c_double), ("timeout_ms", C.c_int32), ("reliable_restart", C.c_int32),
                ("mean_constraint", C.c_int32)]


class ServerCounters(C.Structure):
    _fields_ = [(k, C.c_int64) for k in ("submitted", "admitted", "completed", "failed", "queued", "inflight",
                                        "resident_meshes", "evictions", "assemblies", "resident_bytes",
                                        "budget_bytes", "assembly_us")]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


class SolveStats(C.Structure):
    _fields_ = [("status", C.c_int32), ("iterations", C.c_int32), ("restarts", C.c_int32),
                ("refinements", C.c_int32), ("err_init", C.c_double), ("err_final", C.c_double),
                ("rel_res_inf", C.c_double), ("solve_ms", C.c_double)]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


class ServerOpts(C.Structure):
    _fields_ = [("max_inflight", C.c_int32), ("team", C.c_int32), ("blocks_per_cta", C.c_int32),
                ("solve_share", C.c_double), ("hbm_budget_bytes", C.c_int64), ("solve", SolveOpts)]


# name -> (restype, argtypes)
SIGNATURES = {
    "cup2d_version": (C.c_char_p, []),
    "cup2d_status_string": (C.c_char_p, [C.c_int]),
    "cup2d_default_opts": (None, [C.POINTER(SolveOpts)]),
    "cup2d_pinv": (C.c_int, [P_f64]),
    "cup2d_poisson_create": (C.c_int, [C.POINTER(Forest), C.POINTER(SolveOpts), C.POINTER(C.c_void_p)]),
    "cup2d_poisson_update_mesh": (C.c_int, [C.c_void_p, C.POINTER(Forest)]),
    "cup2d_poisson_adapt_disks": (C.c_int, [C.c_void_p, C.c_int32, C.POINTER(C.c_double), C.c_double,
                                            C.POINTER(C.c_int64)]),
    "cup2d_poisson_get_forest": (C.c_int, [C.c_void_p, C.POINTER(C.c_int32), C.POINTER(C.c_int32),
                                           C.POINTER(C.c_int32)]),
    "cup2d_poisson_pressure_step": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                              C.POINTER(SolveStats), C.c_void_p]),
    "cup2d_poisson_pressure_rhs": (C.c_int, [C.c_void_p, C.c_double, C.c_void_p, C.c_void_p, C.c_void_p,
                                             C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "cup2d_poisson_pressure_correction": (C.c_int, [C.c_void_p, C.c_double, C.c_void_p, C.c_void_p,
                                                    C.c_void_p]),
    "cup2d_poisson_pressure_projection": (C.c_int, [C.c_void_p, C.c_double, C.c_void_p, C.c_void_p, C.c_void_p,
                                                    C.c_void_p, C.c_void_p, C.c_void_p, C.POINTER(SolveStats),
                                                    C.c_void_p]),
    "cup2d_poisson_set_opts": (C.c_int, [C.c_void_p, C.POINTER(SolveOpts)]),
    "cup2d_poisson_num_cells": (C.c_int64, [C.c_void_p]),
    "cup2d_poisson_set_grid": (C.c_int, [C.c_void_p, C.c_int32]),
    "cup2d_poisson_destroy": (C.c_int, [C.c_void_p]),
    "cup2d_poisson_solve": (C.c_int, [C.c_void_p, P_f64, P_f64, C.POINTER(SolveStats)]),
    "cup2d_poisson_solve_device": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p,
                                             C.POINTER(SolveStats), C.c_void_p]),
    "cup2d_poisson_solve_device_noalloc": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p,
                                                     C.POINTER(SolveStats), C.c_void_p]),
    "cup2d_poisson_apply": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "cup2d_poisson_apply32": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "cup2d_poisson_precond": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "cup2d_poisson_precond32": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "cup2d_poisson_precond32_tc": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "cup2d_poisson_export_csr": (C.c_int, [C.c_void_p, P_i64, P_i64, P_i64, P_i32, P_f64]),
    "cup2d_poisson_explicit_info": (C.c_int, [C.c_void_p, P_i64, P_i64]),
    "cup2d_poisson_set_profiling": (C.c_int, [C.c_void_p, C.c_int32]),
    "cup2d_poisson_profile": (C.c_int, [C.c_void_p, P_f64, P_f64, C.c_int32]),
    "cup2d_batch_create": (C.c_int, [C.c_int32, C.POINTER(Forest), C.POINTER(SolveOpts),
                                     C.POINTER(C.c_void_p)]),
    "cup2d_batch_set_opts": (C.c_int, [C.c_void_p, C.POINTER(SolveOpts)]),
    "cup2d_batch_set_team": (C.c_int, [C.c_void_p, C.c_int32]),
    "cup2d_batch_size": (C.c_int32, [C.c_void_p]),
    "cup2d_batch_num_cells": (C.c_int64, [C.c_void_p, C.c_int32]),
    "cup2d_batch_solve_device": (C.c_int, [C.c_void_p, C.POINTER(C.c_void_p), C.POINTER(C.c_void_p),
                                           C.POINTER(SolveStats), C.c_void_p]),
    "cup2d_batch_tune": (C.c_int, [C.c_void_p, C.POINTER(C.c_void_p), C.POINTER(C.c_void_p), P_i32, C.c_int32,
                                   P_i32, C.c_int32, C.c_int32, P_f64, P_i32, P_i32]),
    "cup2d_batch_set_occupancy": (C.c_int, [C.c_void_p, C.c_int32]),
    "cup2d_poisson_rhs_fourier_device": (C.c_int, [C.c_void_p, C.c_int32, P_f64, C.c_void_p, C.c_void_p]),
    "cup2d_poisson_transfer": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "cup2d_batch_capture": (C.c_int, [C.c_void_p, C.POINTER(C.c_void_p), C.POINTER(C.c_void_p), C.c_int32]),
    "cup2d_batch_replay": (C.c_int, [C.c_void_p, C.c_void_p]),
    "cup2d_batch_replay_stats": (C.c_int, [C.c_void_p, C.c_void_p]),
    "cup2d_batch_solve": (C.c_int, [C.c_void_p, C.POINTER(P_f64), C.POINTER(P_f64), C.POINTER(SolveStats)]),
    "cup2d_batch_timeline": (C.c_int, [C.c_void_p, P_f64, P_f64, P_f64]),
    "cup2d_batch_set_profiling": (C.c_int, [C.c_void_p, C.c_int32]),
    "cup2d_batch_profile": (C.c_int, [C.c_void_p, P_f64, P_f64, C.c_int32]),
    "cup2d_batch_destroy": (C.c_int, [C.c_void_p]),
    "cup2d_server_default_opts": (None, [C.POINTER(ServerOpts)]),
    "cup2d_server_create": (C.c_int, [C.POINTER(ServerOpts), C.POINTER(C.c_void_p)]),
    "cup2d_server_add_mesh": (C.c_int, [C.c_void_p, C.POINTER(Forest), P_i64]),
    "cup2d_server_submit": (C.c_int, [C.c_void_p, C.c_int64, P_f64, P_f64, C.c_int32, P_i64]),
    "cup2d_server_poll": (C.c_int, [C.c_void_p, C.c_int64, C.POINTER(SolveStats), P_f64]),
    "cup2d_server_wait": (C.c_int, [C.c_void_p, C.c_int64, C.c_int32, C.POINTER(SolveStats), P_f64]),
    "cup2d_server_take_completed": (C.c_int, [C.c_void_p, P_i64, C.c_int32, C.c_int32, P_i32]),
    "cup2d_server_get_counters": (C.c_int, [C.c_void_p, C.POINTER(ServerCounters)]),
    "cup2d_server_destroy": (C.c_int, [C.c_void_p]),
    "cup2d_mesh_disks": (C.c_int, [C.c_int32, C.c_int32, C.c_int32, C.c_double, C.c_int32, C.c_int32,
                                   C.c_int32, P_f64, C.c_double, C.POINTER(C.c_void_p)]),
    "cup2d_mesh_uniform": (C.c_int, [C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_double,
                                     C.c_int32, C.c_int32, C.POINTER(C.c_void_p)]),
    "cup2d_mesh_forest": (C.c_int, [C.c_void_p, C.POINTER(Forest)]),
    "cup2d_mesh_destroy": (C.c_int, [C.c_void_p]),
    "cup2d_forest_validate": (C.c_int, [C.POINTER(Forest)]),
    "cup2d_forest_cell_h": (C.c_int, [C.POINTER(Forest), P_f64]),
    "cup2d_rhs_fourier": (C.c_int, [C.POINTER(Forest), C.c_uint64, C.c_int32, P_f64]),
    "cup2d_fourier_num_modes": (C.c_int32, [C.c_int32]),
    "cup2d_fourier_coefs": (C.c_int, [C.c_uint64, C.c_int32, P_f64]),
    "cup2d_fourier_advance": (C.c_int, [C.c_uint64, C.c_int32, C.c_double, C.c_int64, P_f64]),
    "cup2d_rhs_from_coefs": (C.c_int, [C.POINTER(Forest), C.c_int32, P_f64, P_f64]),
}

_lib = None


class Cup2dError(RuntimeError):
    def __init__(self, status: int, where: str):
        msg = f"{where}: status {status}"
        if _lib is not None:
            msg += f" ({_lib.cup2d_status_string(status).decode()})"
        super().__init__(msg)
        self.status = status


def lib() -> C.CDLL:
    """Loads the library once; raises if it has not been built."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise ImportError(f"{LIB_PATH} is missing: build it with `python -m cup2d_b200.build`")
        L = C.CDLL(str(LIB_PATH))
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def check(status: int, where: str, allow=(OK,)) -> int:
    if status not in allow:
        raise Cup2dError(status, where)
    return status
