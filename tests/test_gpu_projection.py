"""The pressure projection's field kernels on the device
(cup2d_poisson_pressure_rhs / _correction / _projection) against the
oracle's lab-based restatement of PressureSingle's kernels
(oracle/projection.cpp): bit for bit, on AMR forests with coarse/fine faces,
walls and periodic edges; plus the size-independent properties (exact
divergence and gradient of linear fields away from walls, conservation) at a
large size, and the whole projection against the host composition.
"""
import numpy as np
import pytest

import oracle
from cup2d_b200 import Cup2dError, Mesh, Solver
from cup2d_b200 import _lib as L
from cup2d_b200.problems import seeded_disks, sized_mesh, small_mesh

pytestmark = pytest.mark.gpu


def _meshes():
    return {
        "small": small_mesh,
        "periodic_x": lambda: Mesh.disks(4, 2, 4, 2.0, [(1.9, 0.5, 0.12)], 0.1, periodic_x=True),
        "periodic_xy": lambda: Mesh.disks(2, 2, 5, 1.0, [(0.03, 0.95, 0.1)], 0.06, periodic_x=True,
                                          periodic_y=True),
        "three_disks": lambda: Mesh.disks(8, 4, 5, 2.0, seeded_disks(np.random.default_rng(5), 3), 0.08),
        "sized_900": lambda: sized_mesh(np.random.default_rng(8), 900),
        "uniform": lambda: Mesh.uniform(4, 2, 3, 2, 2.0),
    }


MESHES = _meshes()


def _fields(m, seed):
    rng = np.random.default_rng(seed)
    n = m.ncells
    return rng.standard_normal((n, 2)), rng.standard_normal((n, 2)), rng.uniform(0, 1, n), rng.standard_normal(n)


def _dev(a, cuda):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).to(cuda)


@pytest.mark.parametrize("name", list(MESHES))
def test_pressure_rhs_bit_exact(cuda, name):
    import torch
    m = MESHES[name]()
    vel, udef, chi, pres = _fields(m, 11)
    dt = 0.0137
    tmp_o, pold_o = oracle.pressure_rhs(m, dt, vel, udef, chi, pres)
    V, U, X, P = (_dev(a, cuda) for a in (vel, udef, chi, pres))
    T = torch.empty(m.ncells, dtype=torch.float64, device=cuda)
    PO = torch.empty_like(T)
    with Solver(m) as s:
        s.pressure_rhs(dt, V, U, X, P, PO, T)
    torch.cuda.synchronize()
    assert np.array_equal(T.cpu().numpy(), tmp_o)
    assert np.array_equal(PO.cpu().numpy(), pold_o)
    assert not P.any()                                       # PRES = 0 before the solve
    assert np.array_equal(V.cpu().numpy(), vel)              # inputs untouched


@pytest.mark.parametrize("name", ["small", "periodic_xy", "sized_900"])
def test_pressure_rhs_parts(cuda, name):
    """Velocity part alone, and the Laplacian part alone on a given tmp."""
    import torch
    m = MESHES[name]()
    vel, udef, chi, pres = _fields(m, 12)
    dt = 0.02
    tmp_v, _ = oracle.pressure_rhs(m, dt, vel, udef, chi)
    tmp0 = np.random.default_rng(13).standard_normal(m.ncells)
    tmp_p, pold_o = oracle.pressure_rhs(m, dt, pres=pres, tmp=tmp0)
    T = torch.empty(m.ncells, dtype=torch.float64, device=cuda)
    with Solver(m) as s:
        s.pressure_rhs(dt, _dev(vel, cuda), _dev(udef, cuda), _dev(chi, cuda), tmp=T)
        torch.cuda.synchronize()
        assert np.array_equal(T.cpu().numpy(), tmp_v)
        T2, P, PO = _dev(tmp0, cuda), _dev(pres, cuda), torch.empty_like(T)
        s.pressure_rhs(dt, pres=P, pold=PO, tmp=T2)
        torch.cuda.synchronize()
    assert np.array_equal(T2.cpu().numpy(), tmp_p)
    assert np.array_equal(PO.cpu().numpy(), pold_o)


@pytest.mark.parametrize("name", list(MESHES))
def test_pressure_correction_bit_exact(cuda, name):
    import torch
    m = MESHES[name]()
    vel, _, _, pres = _fields(m, 21)
    dt = 0.0071
    want = oracle.pressure_correction(m, dt, pres, vel)
    V, P = _dev(vel, cuda), _dev(pres, cuda)
    with Solver(m) as s:
        s.pressure_correction(dt, P, V)
    torch.cuda.synchronize()
    assert np.array_equal(V.cpu().numpy(), want)
    assert np.array_equal(P.cpu().numpy(), pres)


def test_linear_fields_exact_at_size(cuda):
    """At ~6,000 blocks: linear velocity -> divergence h^2 (a + d) / dt and
    linear pressure -> velocity change -dt grad p on every cell off the walls
    (coarse/fine faces included); the chi-free divergence sums to zero."""
    import torch
    m = sized_mesh(np.random.default_rng(31), 6000, level_max=6)
    x, y = m.cell_centres()
    a, b, c, d = 0.7, -1.3, 0.4, 2.1
    vel = np.stack([a * x + b * y, c * x + d * y], axis=1)
    h = np.repeat(m.cell_h(), 64)
    h0 = m.extent / (max(m.bpdx, m.bpdy) * 8)
    ok = (x > h) & (x < m.bpdx * 8 * h0 - h) & (y > h) & (y < m.bpdy * 8 * h0 - h)
    dt = 0.02
    T = torch.empty(m.ncells, dtype=torch.float64, device=cuda)
    V = _dev(vel, cuda)
    zero2 = torch.zeros_like(V)
    zero = torch.zeros(m.ncells, dtype=torch.float64, device=cuda)
    with Solver(m) as s:
        s.pressure_rhs(dt, V, zero2, zero, tmp=T)
        torch.cuda.synchronize()
        tmp = T.cpu().numpy()
        want = h * h * (a + d) / dt
        assert np.allclose(tmp[ok], want[ok], rtol=1e-10, atol=1e-12 * np.abs(want).max())
        rnd = _dev(np.random.default_rng(32).standard_normal((m.ncells, 2)), cuda)
        s.pressure_rhs(dt, rnd, zero2, zero, tmp=T)
        torch.cuda.synchronize()
        t2 = T.cpu().numpy()
        assert abs(t2.sum()) <= 1e-12 * np.abs(t2).sum()
        P = _dev(0.3 * x - 0.9 * y, cuda)
        s.pressure_correction(dt, P, zero2)
        torch.cuda.synchronize()
    dv = zero2.cpu().numpy()
    assert np.allclose(dv[ok, 0], -dt * 0.3, rtol=1e-10)
    assert np.allclose(dv[ok, 1], dt * 0.9, rtol=1e-10)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_projection_matches_host(cuda, precision):
    """RHS -> solve -> pres += pold - mean -> velocity correction, against the
    same chain on the host (oracle kernels, oracle BiCGSTAB)."""
    import torch
    m = Mesh.disks(8, 4, 5, 2.0, seeded_disks(np.random.default_rng(5), 3), 0.08)
    # smooth fields (a solve to rel. residual 1e-9 bounds the error of the
    # smooth part of the solution, not of grid-scale noise); a constant chi
    # keeps the right-hand side a flux difference (zero sum), as the Neumann
    # problem needs
    x, y = m.cell_centres()
    vel = np.stack([np.sin(np.pi * x) * np.cos(np.pi * y) + 0.3 * np.cos(2 * np.pi * x),
                    np.cos(1.5 * np.pi * x) * np.sin(2 * np.pi * y) - 0.2 * x], axis=1)
    udef = np.stack([np.cos(np.pi * y), np.sin(np.pi * x)], axis=1)
    chi = np.full(m.ncells, 0.3)
    pres0, _ = oracle.solve(m, m.rhs_fourier(42), tol_rel=1e-10, max_iter=5000)
    dt = 0.01
    tmp_h, pold_h = oracle.pressure_rhs(m, dt, vel, udef, chi, pres0)
    x_h, st_h = oracle.solve(m, tmp_h, tol_rel=1e-10, max_iter=20000)
    assert st_h["converged"], st_h
    w = np.repeat(m.cell_h() ** 2, 64)
    pres_h = x_h + pold_h - np.dot(w, x_h) / np.sum(w)
    vel_h = oracle.pressure_correction(m, dt, pres_h, vel)
    V, U, X, P = (_dev(a, cuda) for a in (vel, udef, chi, pres0))
    T = torch.empty(m.ncells, dtype=torch.float64, device=cuda)
    PO = torch.empty_like(T)
    with Solver(m, tol_rel=1e-9, max_iter=8000, precision=precision) as s:
        st = s.pressure_projection(dt, V, U, X, P, PO, T)
    torch.cuda.synchronize()
    assert st["status"] == L.OK, st
    assert np.array_equal(T.cpu().numpy(), tmp_h)
    assert np.array_equal(PO.cpu().numpy(), pold_h)
    p = P.cpu().numpy()
    assert np.linalg.norm(p - pres_h) / np.linalg.norm(pres_h) <= 1e-6
    v = V.cpu().numpy()
    assert np.linalg.norm(v - vel_h) / np.linalg.norm(vel_h - vel) <= 1e-5


def test_projection_arguments(cuda):
    import torch
    m = small_mesh()
    n = m.ncells
    a = torch.zeros(n, dtype=torch.float64, device=cuda)
    b = torch.zeros_like(a)
    c = torch.zeros_like(a)
    v = torch.zeros(2 * n, dtype=torch.float64, device=cuda)
    u = torch.zeros_like(v)
    with Solver(m) as s:
        for call in (lambda: s.pressure_rhs(0.1, pres=a, pold=a, tmp=b),          # pold overlaps pres
                     lambda: s.pressure_rhs(0.1, tmp=b),                          # nothing to do
                     lambda: s.pressure_rhs(0.0, v, u, c, tmp=b),                 # dt <= 0
                     lambda: s.pressure_rhs(0.1, v, v, c, tmp=b),                 # vel overlaps udef
                     lambda: s.pressure_correction(0.1, v[:n], v),                # pres inside vel
                     lambda: s.pressure_correction(-1.0, a, v)):
            with pytest.raises(Cup2dError) as e:
                call()
            assert e.value.status == L.INVALID_ARGUMENT
        with pytest.raises(ValueError):
            s.pressure_correction(0.1, a, a)                                       # vel needs 2 per cell
