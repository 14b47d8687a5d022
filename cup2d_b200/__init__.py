"""cup2d_b200 — B200-native pressure-Poisson solve of CUP2D.

BiCGSTAB with the 64x64 block-Jacobi preconditioner on the 8x8-cell
block-AMR forest, as hand-written sm_100a CUDA behind a C ABI
(include/cup2d_poisson.h).  The library libcup2d_poisson.so is built in
this directory by `python -m cup2d_b200.build`.
"""
from ._lib import Cup2dError, lib  # noqa: F401
from .mesh import Mesh, fourier_advance, fourier_coefs  # noqa: F401
from .poisson import (BatchSolver, ExpAMRSolver, PoissonSolver, ScalarGrid, Server, SimulationData, Solver,  # noqa: F401
                      device_pinv, make_opts, makePoissonSolver)

__version__ = "0.1.0"
