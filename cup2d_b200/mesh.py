"""Block-AMR forests and synthetic right-hand sides.

A `Mesh` is the block list CUP2D's Cubism grid hands to ExpAMRSolver::getMat
(source/Poisson/ExpAMRSolver.cpp:180-313): per block its level and (i,j)
index at that level, over bpdx x bpdy root blocks of 8x8 cells.  Cell vectors
are block-major, v[block*64 + iy*8 + ix], in the mesh's block order.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from . import _lib as L


def _ptr(a: np.ndarray, ct):
    return a.ctypes.data_as(C.POINTER(ct))


@dataclass
class Mesh:
    bpdx: int
    bpdy: int
    level_max: int
    extent: float
    level: np.ndarray
    bx: np.ndarray
    by: np.ndarray
    periodic_x: bool = False
    periodic_y: bool = False
    _keep: list = field(default_factory=list, repr=False)

    def __post_init__(self):
        self.level = np.ascontiguousarray(self.level, dtype=np.int32)
        self.bx = np.ascontiguousarray(self.bx, dtype=np.int32)
        self.by = np.ascontiguousarray(self.by, dtype=np.int32)

    # ------------------------------------------------------------ build ---
    @classmethod
    def _from_handle(cls, h: C.c_void_p) -> "Mesh":
        f = L.Forest()
        L.check(L.lib().cup2d_mesh_forest(h, C.byref(f)), "cup2d_mesh_forest")
        n = f.nblocks
        lv = np.ctypeslib.as_array(f.level, shape=(n,)).copy()
        bx = np.ctypeslib.as_array(f.bx, shape=(n,)).copy()
        by = np.ctypeslib.as_array(f.by, shape=(n,)).copy()
        m = cls(f.bpdx, f.bpdy, f.level_max, f.extent, lv, bx, by, bool(f.periodic_x), bool(f.periodic_y))
        L.lib().cup2d_mesh_destroy(h)
        return m

    @classmethod
    def disks(cls, bpdx: int, bpdy: int, level_max: int, extent: float, disks, band: float,
              periodic_x: bool = False, periodic_y: bool = False) -> "Mesh":
        d = np.ascontiguousarray(np.asarray(disks, dtype=np.float64).reshape(-1, 3))
        h = C.c_void_p()
        L.check(L.lib().cup2d_mesh_disks(bpdx, bpdy, level_max, extent, int(periodic_x), int(periodic_y),
                                         d.shape[0], _ptr(d, C.c_double), band, C.byref(h)),
                "cup2d_mesh_disks")
        return cls._from_handle(h)

    @classmethod
    def uniform(cls, bpdx: int, bpdy: int, level_max: int, level: int, extent: float,
                periodic_x: bool = False, periodic_y: bool = False) -> "Mesh":
        h = C.c_void_p()
        L.check(L.lib().cup2d_mesh_uniform(bpdx, bpdy, level_max, level, extent, int(periodic_x),
                                           int(periodic_y), C.byref(h)), "cup2d_mesh_uniform")
        return cls._from_handle(h)

    # ------------------------------------------------------------ views ---
    @property
    def nblocks(self) -> int:
        return int(self.level.shape[0])

    @property
    def ncells(self) -> int:
        return 64 * self.nblocks

    def forest(self) -> L.Forest:
        """ctypes cup2d_forest viewing this mesh's arrays (kept alive by the mesh)."""
        f = L.Forest(self.bpdx, self.bpdy, self.level_max, int(self.periodic_x), int(self.periodic_y),
                     float(self.extent), self.nblocks, _ptr(self.level, C.c_int32), _ptr(self.bx, C.c_int32),
                     _ptr(self.by, C.c_int32))
        return f

    def validate(self) -> bool:
        f = self.forest()
        return L.lib().cup2d_forest_validate(C.byref(f)) == L.OK

    def cell_h(self) -> np.ndarray:
        out = np.empty(self.nblocks, dtype=np.float64)
        f = self.forest()
        L.check(L.lib().cup2d_forest_cell_h(C.byref(f), _ptr(out, C.c_double)), "cup2d_forest_cell_h")
        return out

    def cell_centres(self) -> tuple[np.ndarray, np.ndarray]:
        h = self.cell_h()[:, None]
        ix = np.tile(np.arange(8), 8)[None, :]
        iy = np.repeat(np.arange(8), 8)[None, :]
        x = (self.bx[:, None] * 8 + ix + 0.5) * h
        y = (self.by[:, None] * 8 + iy + 0.5) * h
        return x.reshape(-1), y.reshape(-1)

    def rhs_fourier(self, seed: int, kmax: int = 8) -> np.ndarray:
        b = np.empty(self.ncells, dtype=np.float64)
        f = self.forest()
        L.check(L.lib().cup2d_rhs_fourier(C.byref(f), seed, kmax, _ptr(b, C.c_double)), "cup2d_rhs_fourier")
        return b

    def rhs_from_coefs(self, coef: np.ndarray, kmax: int = 8) -> np.ndarray:
        coef = np.ascontiguousarray(coef, dtype=np.float64)
        b = np.empty(self.ncells, dtype=np.float64)
        f = self.forest()
        L.check(L.lib().cup2d_rhs_from_coefs(C.byref(f), kmax, _ptr(coef, C.c_double), _ptr(b, C.c_double)),
                "cup2d_rhs_from_coefs")
        return b


def fourier_coefs(seed: int, kmax: int = 8) -> np.ndarray:
    n = L.lib().cup2d_fourier_num_modes(kmax)
    c = np.empty(4 * n, dtype=np.float64)
    L.check(L.lib().cup2d_fourier_coefs(seed, kmax, _ptr(c, C.c_double)), "cup2d_fourier_coefs")
    return c


def fourier_advance(coef: np.ndarray, seed: int, step: int, rho: float = 0.95, kmax: int = 8) -> np.ndarray:
    c = np.ascontiguousarray(coef, dtype=np.float64).copy()
    L.check(L.lib().cup2d_fourier_advance(seed, kmax, rho, step, _ptr(c, C.c_double)), "cup2d_fourier_advance")
    return c
