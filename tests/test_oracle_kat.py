"""Known-answer tests of the CPU oracle (no GPU).

The reference ships no tests, fixtures or golden vectors for its Poisson
path, so the oracle is pinned by properties that follow from the reference
source itself (source/Poisson/ExpAMRSolver.{h,cpp}):
  * P^-1 K = -I for the 64x64 block Laplacian K (ExpAMRSolver.cpp:25-99);
  * rows sum to zero (interpolation weights 2/3 - 1/5 + 8/15 = 1, the D1/D2
    weights sum to 0) and columns sum to zero (coarse- and fine-side fluxes
    are exact negatives), so 1^T A = 0 and A 1 = 0;
  * a uniform mesh gives the textbook Neumann 5-point matrix;
  * quadratic exactness: every row whose cell does not touch a wall gives
    (A p)_i = h_i^2 lap(p) for quadratic p, coarse/fine rows included (the
    ghost interpolation and the one-sided Taylor stencils are exact for
    quadratics, and the fluxes are conservative);
  * two coarse/fine rows computed by hand from makeFlux/interpolate
    (tests/golden/hand_rows.json);
  * second-order convergence to cos(pi x) cos(pi y);
  * the BiCGSTAB restatement converges to the solution of a direct solve.
"""
import json
from fractions import Fraction
from pathlib import Path

import numpy as np
import pytest

import scipy.sparse.linalg as spla

import oracle
from cup2d_b200 import Mesh
from cup2d_b200.problems import sized_mesh, small_mesh

GOLDEN = Path(__file__).resolve().parent / "golden"


def block_K():
    K = np.zeros((64, 64))
    for i in range(64):
        for j in range(64):
            yi, xi = divmod(i, 8)
            yj, xj = divmod(j, 8)
            K[i, j] = 4 if i == j else (-1 if abs(xi - xj) + abs(yi - yj) == 1 else 0)
    return K


def test_pinv_inverts_block_laplacian():
    P = oracle.pinv()
    assert np.max(np.abs(P @ block_K() + np.eye(64))) < 1e-13
    assert np.array_equal(P, P.T)
    assert np.all(np.linalg.eigvalsh(P) < 0)


MESHES = {
    "small": lambda: small_mesh(),
    "periodic_x": lambda: Mesh.disks(4, 2, 4, 2.0, [(1.0, 0.5, 0.12)], 0.1, periodic_x=True),
    "periodic_xy": lambda: Mesh.disks(2, 2, 4, 1.0, [(0.1, 0.9, 0.1)], 0.08, periodic_x=True, periodic_y=True),
    "sized": lambda: sized_mesh(np.random.default_rng(3), 800),
    "deep": lambda: Mesh.disks(2, 1, 7, 2.0, [(0.7, 0.4, 0.05)], 0.02),
}


@pytest.mark.parametrize("name", list(MESHES))
def test_rows_and_columns_sum_to_zero(name):
    m = MESHES[name]()
    S = oracle.Matrix(m).scipy()
    one = np.ones(S.shape[0])
    scale = np.abs(S).sum(axis=1).max()
    assert np.max(np.abs(S @ one)) < 1e-13 * scale
    assert np.max(np.abs(one @ S)) < 1e-13 * scale


def _cell_grid_index(m: Mesh):
    """(gx, gy) of every cell of a uniform mesh."""
    ix = np.tile(np.arange(8), 8)
    iy = np.repeat(np.arange(8), 8)
    gx = (m.bx[:, None] * 8 + ix[None, :]).reshape(-1)
    gy = (m.by[:, None] * 8 + iy[None, :]).reshape(-1)
    return gx, gy


@pytest.mark.parametrize("periodic", [False, True])
def test_uniform_mesh_is_textbook_laplacian(periodic):
    m = Mesh.uniform(3, 2, 2, 1, 3.0, periodic_x=periodic, periodic_y=periodic)
    S = oracle.Matrix(m).scipy().toarray()
    gx, gy = _cell_grid_index(m)
    NX, NY = 3 * 2 * 8, 2 * 2 * 8
    lut = {(x, y): i for i, (x, y) in enumerate(zip(gx, gy))}
    T = np.zeros_like(S)
    for i, (x, y) in enumerate(zip(gx, gy)):
        for dx, dy in ((1, 0), (-1, 0), (0, 1), (0, -1)):
            nx_, ny_ = x + dx, y + dy
            if periodic:
                nx_, ny_ = nx_ % NX, ny_ % NY
            elif not (0 <= nx_ < NX and 0 <= ny_ < NY):
                continue  # homogeneous Neumann wall: no flux
            T[i, lut[(nx_, ny_)]] += 1
            T[i, i] -= 1
    assert np.array_equal(S, T)


@pytest.mark.parametrize("name", ["small", "sized", "deep"])
def test_quadratic_exactness(name):
    m = MESHES[name]()
    A = oracle.Matrix(m)
    x, y = m.cell_centres()
    h = np.repeat(m.cell_h(), 64)
    # p = a x^2 + b xy + c y^2 + linear: lap p = 2a + 2c
    a, bq, c = 0.7, -0.3, 0.4
    p = a * x * x + bq * x * y + c * y * y + 0.2 * x - 0.1 * y
    Ap = A.spmv(p)
    Lx = m.bpdx * 8 * m.cell_h()[0] * 2 ** m.level[0]
    Ly = m.bpdy * 8 * m.cell_h()[0] * 2 ** m.level[0]
    away = (x - h > 1e-12) & (x + h < Lx - 1e-12) & (y - h > 1e-12) & (y + h < Ly - 1e-12)
    assert away.sum() > 0.5 * m.ncells
    expect = h * h * (2 * a + 2 * c)
    err = np.abs(Ap - expect)[away]
    assert err.max() < 1e-11 * max(1.0, np.abs(p).max())
    # coarse/fine rows are among the checked ones
    S = A.scipy()
    levels = np.repeat(m.level, 64)
    mixed = np.array([np.unique(levels[S.indices[S.indptr[i]:S.indptr[i + 1]]]).size > 1 for i in range(m.ncells)])
    assert (mixed & away).sum() > 0


def test_hand_derived_coarse_fine_rows():
    g = json.loads((GOLDEN / "hand_rows.json").read_text())
    f = g["forest"]
    m = Mesh(f["bpdx"], f["bpdy"], f["level_max"], f["extent"], np.array(f["level"]), np.array(f["bx"]),
             np.array(f["by"]))
    assert m.validate()
    S = oracle.Matrix(m).scipy()
    for row, cols in g["rows"].items():
        r = int(row)
        got = dict(zip(S.indices[S.indptr[r]:S.indptr[r + 1]].tolist(), S.data[S.indptr[r]:S.indptr[r + 1]].tolist()))
        got = {c: v for c, v in got.items() if v != 0.0}
        want = {int(c): float(Fraction(n, d)) for c, (n, d) in cols.items()}
        assert set(got) == set(want), (r, sorted(got), sorted(want))
        for c in want:
            assert abs(got[c] - want[c]) < 4e-16, (r, c, got[c], want[c])


def test_manufactured_solution_second_order():
    errs = []
    for lvl in (1, 2, 3):
        m = Mesh.uniform(2, 1, 4, lvl, 2.0)
        x, y = m.cell_centres()
        h = np.repeat(m.cell_h(), 64)
        exact = np.cos(np.pi * x) * np.cos(np.pi * y)
        b = -2 * np.pi ** 2 * h * h * exact
        b -= b.mean()
        sol, st = oracle.solve(m, b, tol_rel=1e-12, max_iter=20000, subtract_mean_=False)
        e = sol - sol.mean() - (exact - exact.mean())
        errs.append(np.abs(e).max())
    rates = np.log2(np.array(errs[:-1]) / np.array(errs[1:]))
    assert np.all(rates > 1.8), (errs, rates)


def test_manufactured_solution_amr():
    m = Mesh.disks(2, 1, 4, 2.0, [(0.9, 0.5, 0.15)], 0.1)
    x, y = m.cell_centres()
    h = np.repeat(m.cell_h(), 64)
    exact = np.cos(np.pi * x) * np.cos(np.pi * y)
    b = -2 * np.pi ** 2 * h * h * exact
    b -= b.mean()
    sol, st = oracle.solve(m, b, tol_rel=1e-12, max_iter=20000, subtract_mean_=False)
    assert st["converged"] == 1
    e = sol - sol.mean() - (exact - exact.mean())
    hmax = m.cell_h().max()
    assert np.abs(e).max() < 2.0 * hmax


def test_bicgstab_matches_direct_solve():
    m = small_mesh()
    A = oracle.Matrix(m)
    S = A.scipy().tocsc()
    b = m.rhs_fourier(5)
    n = S.shape[0]
    # direct solve of the singular system with the constant mode pinned:
    # drop the last equation and unknown (x_last = 0); b has zero sum, so the
    # dropped equation holds automatically
    xd = np.zeros(n)
    xd[:-1] = spla.spsolve(S[:-1, :-1], b[:-1])
    xd -= xd.mean()
    x, st = A.bicgstab(b, tol_rel=1e-10, max_iter=5000)
    assert st["converged"] == 1
    x -= x.mean()
    assert np.linalg.norm(x - xd) / np.linalg.norm(xd) < 1e-7


def test_bicgstab_reference_rules():
    """Restart cap, iteration cap and the best-iterate rule of BiCGSTAB.cu."""
    m = small_mesh()
    A = oracle.Matrix(m)
    b = m.rhs_fourier(2)
    x, st = A.bicgstab(b, tol_rel=0.0, max_iter=5)
    assert st["iterations"] == 5 and st["converged"] == 0 and st["hit_max_iter"] == 1
    # zero RHS: the breakdown test rho^2 < 1e-16 |r|^2 |rhat|^2 reads 0 < 0
    # and the improvement test error < error_opt reads 0 < 0, so the
    # reference neither restarts nor converges: it runs to the iteration cap
    # and returns x0
    x, st = A.bicgstab(np.zeros(m.ncells), tol_rel=1e-8, max_restarts=1, max_iter=7)
    assert st["restarts"] == 0 and st["iterations"] == 7 and st["hit_max_iter"] == 1 and np.all(x == 0)
    # the returned iterate is the best one by L-inf residual
    x, st = A.bicgstab(b, tol_rel=0.0, max_iter=40)
    r = b - A.spmv(x)
    assert abs(np.abs(r).max() - st["err_opt"]) < 1e-10 * st["err_init"]


def test_subtract_mean_is_volume_weighted():
    m = small_mesh()
    rng = np.random.default_rng(0)
    x = rng.standard_normal(m.ncells)
    y = oracle.subtract_mean(m.cell_h(), x)
    h2 = np.repeat(m.cell_h() ** 2, 64)
    assert abs(np.sum(h2 * y)) < 1e-12 * np.sum(h2 * np.abs(y))
    assert np.allclose(x - y, (x - y)[0])
