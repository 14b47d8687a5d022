"""The pressure step around the solve (cup2d_poisson_pressure_step) against a
host restatement of PressureSingle::operator() (source/Operators/
PressureSingle.cpp:831-879) built on the oracle:

  pold = pres; tmp -= L(pold); pres = 0; solve; pres += pold - mean(pres)

with the volume-weighted mean of :853-868.  The device's L(pold) is
updatePressureRHS1's flux-corrected 5-point stencil, which equals the
assembled operator (the oracle's, which is the reference's) to rounding; it
is compared with the assembled operator's product here and bit for bit with
the oracle's restatement of updatePressureRHS1 in test_gpu_projection.py.
"""
import numpy as np
import pytest

import oracle
from cup2d_b200 import Mesh, Solver
from cup2d_b200 import _lib as L
from cup2d_b200.problems import sized_mesh, small_mesh

pytestmark = pytest.mark.gpu


def _host_step(m, tmp, pres, tol_rel):
    A = oracle.Matrix(m)
    pold = pres.copy()
    rhs = tmp - A.spmv(pold)
    x, st = oracle.solve(m, rhs, tol_rel=tol_rel, max_iter=20000)
    w = np.repeat(m.cell_h() ** 2, 64)
    x = x + pold - np.dot(w, x) / np.sum(w)
    return x, rhs, pold


@pytest.mark.parametrize("mesh_fn", [small_mesh, lambda: sized_mesh(np.random.default_rng(8), 900),
                                     lambda: Mesh.disks(4, 2, 4, 2.0, [(1.0, 0.5, 0.12)], 0.1, periodic_x=True)])
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_pressure_step_matches_host(cuda, mesh_fn, precision):
    import torch
    m = mesh_fn()
    tmp = m.rhs_fourier(41)
    # a previous pressure: the solution of another right-hand side
    pres0, _ = oracle.solve(m, m.rhs_fourier(42), tol_rel=1e-10, max_iter=5000)
    x_h, rhs_h, pold_h = _host_step(m, tmp, pres0, 1e-10)
    t = torch.from_numpy(tmp).to(cuda)
    p = torch.from_numpy(pres0).to(cuda)
    po = torch.empty_like(p)
    with Solver(m, tol_rel=1e-9, max_iter=8000, precision=precision) as s:
        st = s.pressure_step(t, p, po)
    torch.cuda.synchronize()
    assert st["status"] == L.OK, st
    assert np.array_equal(po.cpu().numpy(), pold_h)            # pold = pres, exactly
    scale = np.abs(oracle.Matrix(m).scipy()).dot(np.abs(pres0)) + np.abs(tmp)
    assert np.all(np.abs(t.cpu().numpy() - rhs_h) <= 1e-13 * (scale + 1e-300))   # tmp - L(pold)
    x = p.cpu().numpy()
    assert np.linalg.norm(x - x_h) / np.linalg.norm(x_h) <= 1e-6
    # the volume-weighted mean of the new pressure is the old one's
    w = np.repeat(m.cell_h() ** 2, 64)
    assert abs(np.dot(w, x - pres0)) / np.sum(w) <= 1e-12 * np.abs(x).max()


def test_pressure_step_arguments(cuda):
    import torch
    m = small_mesh()
    a = torch.zeros(m.ncells, dtype=torch.float64, device=cuda)
    b = torch.zeros_like(a)
    with Solver(m) as s:
        from cup2d_b200 import Cup2dError
        with pytest.raises(Cup2dError) as e:
            s.pressure_step(a, a, b)      # tmp and pres must be distinct
        assert e.value.status == L.INVALID_ARGUMENT
