"""bMeanConstraint pinned to CUP2D's own code (CPU).

With sim.bMeanConstraint set, ExpAMRSolver::getMat records the row of cell
(0,0) of the block whose index is (0,0) (ExpAMRSolver.cpp:251-256), getVec
writes 0 into that row of b (:340-346), and every SpMV of the solver replaces
that row of its result by sum_i h_i^2 v_i over the operand (BiCGSTAB.cu:
393-410): the singular Neumann system becomes regular, with sum h^2 x = 0.

* the reference's own getMat/getVec (the checker's CPU build) pick the row the
  oracle and the library pick, on forests whose blocks come in any order;
* tests/golden/ref_solve_mean_*.npz hold the reference's GPU solve with the
  constraint (tests/golden/make_ref_fixtures.py mean); the oracle's
  constrained BiCGSTAB reaches the same solution, also for right-hand sides
  the plain Neumann problem cannot solve (a constant added).
"""
from pathlib import Path

import numpy as np
import pytest

import oracle
from cup2d_b200 import Mesh
from cup2d_b200.problems import sized_mesh
from tests.golden import make_ref_fixtures as F
from tests.test_ref_pin import load_solve_fixture, rel_l2_sampled

GOLDEN = Path(__file__).resolve().parent / "golden"


def _reversed(m):
    return Mesh(m.bpdx, m.bpdy, m.level_max, m.extent, m.level[::-1], m.bx[::-1], m.by[::-1], m.periodic_x,
                m.periodic_y)


def _meshes():
    rng = np.random.default_rng(17)
    out = {name: F.mesh_by_name(name) for name in ("small", "periodic_xy_rev", "sized_1500_rev")}
    for k in range(4):
        m = sized_mesh(rng, int(rng.integers(60, 600)))
        out[f"random_{k}_rev"] = _reversed(m)
        perm = rng.permutation(m.nblocks)
        out[f"random_{k}_perm"] = Mesh(m.bpdx, m.bpdy, m.level_max, m.extent, m.level[perm], m.bx[perm], m.by[perm],
                                       m.periodic_x, m.periodic_y)
    return out


def _ref_cpu():
    import oracle.ref as R
    if not R.available("cpu"):
        pytest.skip("reference checker not built (the reference tree is needed to build it)")
    return R


@pytest.mark.parametrize("name,mesh", list(_meshes().items()))
def test_reference_picks_the_same_mean_row(name, mesh):
    R = _ref_cpu()
    b = np.random.default_rng(3).standard_normal(mesh.ncells) + 1.0
    r = R.assemble(mesh, b, mean_constraint=1)
    row = oracle.mean_row(mesh)
    assert r["mean_row"] == row
    changed = np.flatnonzero(r["b"] != b)
    assert changed.tolist() == [row] and r["b"][row] == 0.0     # getVec zeroes that row only
    assert R.assemble(mesh, b)["mean_row"] == -1                 # off by default


def mean_cases():
    return [c for c in F.MEAN_CASES if (GOLDEN / f"ref_solve_{c}.npz").exists()]


def test_mean_fixtures_present():
    assert mean_cases() == list(F.MEAN_CASES)


def converged_mean_cases():
    return [c for c in mean_cases() if bool(load_solve_fixture(c)["converged"])]


def capped_mean_cases():
    return [c for c in mean_cases() if not bool(load_solve_fixture(c)["converged"])]


@pytest.mark.parametrize("case", converged_mean_cases())
def test_oracle_mean_solve_matches_reference(case):
    fx = load_solve_fixture(case)
    m, b = F.mean_case_rhs(case)
    assert F.array_digest(b) == str(fx["rhs_sha256"])
    _, _, tol_abs, tol_rel, _ = F.MEAN_CASES[case]
    x, st = oracle.solve(m, b, tol_abs=tol_abs, tol_rel=tol_rel, max_iter=1000, mean_constraint=True)
    assert st["converged"]
    assert st["err_init"] == pytest.approx(float(fx["err_init"]), rel=1e-5)
    assert rel_l2_sampled(x, fx) <= 1e-6
    assert np.linalg.norm(x) == pytest.approx(float(fx["x_norm2"]), rel=1e-6)


def test_capped_mean_case():
    """With the constraint the 1,500-block forest needs more than the
    reference's 1000 iterations (and restarts often: the constraint row makes
    the system far from symmetric)."""
    assert capped_mean_cases() == ["mean_sized_1500_rev"]


@pytest.mark.parametrize("case", capped_mean_cases())
def test_oracle_mean_iteration_cap_like_reference(case):
    """Both stop at the 1000-iteration cap, restarting along the way, with a
    best residual far from the tolerance (the printed figure is relative)."""
    fx = load_solve_fixture(case)
    m, b = F.mean_case_rhs(case)
    # two OpenMP threads: a reduction adds its per-thread partials in the
    # order the threads arrive, so with three or more the oracle's sums, and
    # where this chaotic solve stops, differ from run to run; two partials
    # sum the same either way
    threads = oracle.num_threads()
    oracle.set_threads(2)
    try:
        x, st = oracle.solve(m, b, tol_rel=1e-8, max_iter=1000, mean_constraint=True)
    finally:
        oracle.set_threads(threads)
    assert int(fx["iterations"]) == 1000 and st["iterations"] == 1000 and not st["converged"]
    assert st["err_init"] == pytest.approx(float(fx["err_init"]), rel=1e-5)
    assert int(fx["restarts"]) >= 5 and st["restarts"] >= 5
    # where it stops is chaotic (the oracle's best residual at the cap moves
    # from 1e-7 to 9e-3 with the summation order, i.e. the OpenMP threads)
    for rel in (float(fx["err_opt"]), st["err_opt"] / st["err_init"]):
        assert 1e-8 < rel < 0.1


def _on_coarse_fine_face(m, row):
    """Whether the row couples cells of another level (an explicit row of
    the device assembly, computed by whichever CTA holds it in the row
    partition, not necessarily the owner of its block)."""
    rp, col, _ = oracle.Matrix(m).csr()
    cols = col[rp[row]:rp[row + 1]]
    return bool(np.any(m.level[cols // 64] != m.level[row // 64]))


def test_mean_row_cases_cover_explicit_and_stencil_rows():
    """The constrained reference cases include a mean row on a coarse/fine
    face (the corner cell across a periodic edge of periodic_xy_rev) and
    mean rows inside the stencil, so the GPU tests of those cases cover
    both ways the solver records the mean row's own product."""
    kinds = {}
    for case in F.MEAN_CASES:
        m, _ = F.mean_case_rhs(case)
        kinds[case] = _on_coarse_fine_face(m, oracle.mean_row(m))
    assert kinds["mean_periodic_xy_rev"]
    assert not kinds["mean_small"] and not kinds["mean_sized_1500_rev"]

