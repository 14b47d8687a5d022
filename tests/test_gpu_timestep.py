"""GPU tests of the time-stepping steps around the solve: the device RHS,
the transfer of the pressure across a mesh adaptation, and a warm-started
sequence of solves with remeshing (the time-stepping configuration: moving
disk, remesh + device re-assembly every 10 steps, AR(1) Fourier
coefficients), checked against the CPU oracle."""
import numpy as np
import pytest

import oracle
from cup2d_b200 import Cup2dError, Mesh, Solver
from cup2d_b200 import _lib as L
from cup2d_b200.mesh import fourier_advance, fourier_coefs
from cup2d_b200.problems import EXTENT, sized_mesh, small_mesh
from tests.transfer_rule import disk_mesh as _disk_mesh, transfer_restated as _transfer_restated

pytestmark = pytest.mark.gpu


def _meshes():
    rng = np.random.default_rng(5)
    return {"small": small_mesh(), "periodic": Mesh.disks(4, 2, 4, 2.0, [(1.0, 0.5, 0.12)], 0.1, periodic_x=True),
            "sized_800": sized_mesh(rng, 800), "two_disks": _disk_mesh(0.0)}


MESHES = _meshes()


@pytest.mark.parametrize("name", list(MESHES))
def test_rhs_device_matches_host(cuda, name):
    import torch
    m = MESHES[name]
    coef = fourier_advance(fourier_coefs(17), 17, 3)
    b_host = m.rhs_from_coefs(coef)
    b = torch.empty(m.ncells, dtype=torch.float64, device=cuda)
    with Solver(m) as s:
        s.rhs_fourier_device(coef, b)
    bd = b.cpu().numpy()
    scale = np.max(np.abs(b_host))
    assert np.max(np.abs(bd - b_host)) <= 1e-12 * scale
    assert abs(float(np.sum(bd))) <= 1e-12 * float(np.sum(np.abs(bd)))
    assert np.array_equal(m.rhs_fourier(17), m.rhs_from_coefs(fourier_coefs(17)))


@pytest.mark.parametrize("shift,lmax", [(0.0, 5), (0.05, 5), (0.12, 5), (0.05, 4), (0.05, 6)])
def test_transfer_matches_restatement(cuda, shift, lmax):
    """Bit-identical to the restated rule: copies and one 4-term mean."""
    import torch
    src, dst = _disk_mesh(0.0), _disk_mesh(shift, level_max=lmax)
    xs = np.random.default_rng(3).standard_normal(src.ncells)
    with Solver(src) as hs, Solver(dst) as hd:
        xd = torch.empty(dst.ncells, dtype=torch.float64, device=cuda)
        hs.transfer_to(hd, torch.from_numpy(xs).to(cuda), xd)
        got = xd.cpu().numpy()
    want = _transfer_restated(src, xs, dst)
    assert np.array_equal(got, want)
    if shift == 0.0 and lmax == 5:
        assert np.array_equal(got, xs)  # same forest: an exact copy


def test_transfer_preserves_smooth_field(cuda):
    """A smooth field carried to a shifted forest stays within the
    interpolation error of the cell sizes."""
    import torch
    src, dst = _disk_mesh(0.0), _disk_mesh(0.08)

    def field(m):
        x, y = m.cell_centres()
        return np.cos(np.pi * x) * np.sin(2 * np.pi * y)

    with Solver(src) as hs, Solver(dst) as hd:
        xd = torch.empty(dst.ncells, dtype=torch.float64, device=cuda)
        hs.transfer_to(hd, torch.from_numpy(field(src)).to(cuda), xd)
    err = np.max(np.abs(xd.cpu().numpy() - field(dst)))
    # |grad f| <= pi sqrt(5); a sample point lies within h/sqrt(2) of the
    # dst centre, h at most the level-0 cell size
    h_max = EXTENT / (8 * 8)
    assert err <= np.pi * np.sqrt(5) * h_max / np.sqrt(2)


def test_transfer_errors(cuda):
    import torch
    a, b = _disk_mesh(0.0), Mesh.disks(4, 2, 5, EXTENT, [(0.6, 0.5, 0.1)], 0.1)
    with Solver(a) as ha, Solver(b) as hb:
        xa = torch.zeros(a.ncells, dtype=torch.float64, device=cuda)
        xb = torch.zeros(b.ncells, dtype=torch.float64, device=cuda)
        with pytest.raises(Cup2dError):
            ha.transfer_to(hb, xa, xb)  # different root grids
        with pytest.raises(Cup2dError):
            ha.transfer_to(ha, xa, xa)  # aliasing
        with pytest.raises(Cup2dError):
            ha.rhs_fourier_device(fourier_coefs(1, kmax=30), xa, kmax=30)


def _sequence(cuda, steps, remesh_every, precision, tol_b):
    """Time-stepping: disk moves 0.002 per step, remesh (host forest, device
    re-assembly) every `remesh_every` steps with the pressure carried over,
    AR(1) coefficients, device RHS, warm-started solves to |b - Ax|_inf <=
    tol_b |b|_inf (an absolute tolerance per step: relative to a warm start's
    initial residual the target would move with the start).  Yields the
    mesh, b and x of every step."""
    import torch
    seed = 41
    coef = fourier_coefs(seed)
    mesh = _disk_mesh(0.0, level_max=4)
    opts = dict(tol_rel=0.0, max_iter=8000, precision=precision)
    cur, spare = Solver(mesh, **opts), None
    x = torch.zeros(mesh.ncells, dtype=torch.float64, device=cuda)
    try:
        for step in range(steps):
            if step > 0 and step % remesh_every == 0:
                mesh = _disk_mesh(0.002 * step, level_max=4)
                if spare is None:
                    spare = Solver(mesh, **opts)
                else:
                    spare.update_mesh(mesh)
                x_new = torch.empty(mesh.ncells, dtype=torch.float64, device=cuda)
                cur.transfer_to(spare, x, x_new)
                cur, spare, x = spare, cur, x_new
            coef = fourier_advance(coef, seed, step)
            b = torch.empty(mesh.ncells, dtype=torch.float64, device=cuda)
            cur.rhs_fourier_device(coef, b)
            cur.set_opts(tol_abs=tol_b * float(b.abs().max()), **opts)
            st = cur.solve_device(b, x)
            yield step, mesh, b, x, st
    finally:
        cur.close()
        if spare is not None:
            spare.close()


def test_sequence_matches_oracle(cuda):
    """FP64 steps to residual 1e-8 |b| across two remeshes: every step's
    pressure matches the oracle's solve of the same (host) RHS to rel. L2
    1e-6, and warm starts need fewer iterations than cold ones."""
    its = []
    for step, mesh, b, x, st in _sequence(cuda, 22, 10, "fp64", 1e-8):
        assert st["status"] == L.OK
        its.append(st["iterations"])
        if step in (0, 9, 10, 11, 20, 21):
            bh = b.cpu().numpy()
            x_o, st_o = oracle.solve(mesh, bh, tol_rel=1e-9, max_iter=8000)
            assert st_o["converged"]
            xd = x.cpu().numpy()
            xd, xo = xd - xd.mean(), x_o - x_o.mean()
            assert np.linalg.norm(xd - xo) <= 1e-6 * np.linalg.norm(xo), step
    assert np.mean(its[1:10]) < its[0]


def test_sequence_mixed(cuda):
    """Mixed-precision steps to 1e-6 |b|: each reaches the true residual
    target, checked with the FP64 operator, in fewer iterations than the
    first (cold) step on average."""
    import torch
    its = []
    for step, mesh, b, x, st in _sequence(cuda, 12, 5, "mixed", 1e-6):
        assert st["status"] == L.OK
        its.append(st["iterations"])
        with Solver(mesh) as h:
            r = torch.empty_like(b)
            h.apply(x, r)
            r = b - r
        assert float(r.abs().max()) <= 1e-6 * float(b.abs().max()) * 1.0001
    assert np.mean(its[1:]) < its[0]
