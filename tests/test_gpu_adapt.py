"""Forest adaptation on the device (cup2d_poisson_adapt_disks) against the
host forest generator.

The device builds the forest from the disk geometry (tag level by level,
2:1 balance to a fixpoint, Morton order) and re-assembles the operator; the
result must be the forest Mesh.disks builds on the host for the same
geometry, block for block in the same order, with the same assembled
operator (hence the oracle's, hence the reference's), and a time-stepping
remesh through it must give the same bits as the host-forest path.
"""
import numpy as np
import pytest

import oracle
from cup2d_b200 import Cup2dError, Mesh, Solver
from cup2d_b200 import _lib as L
from cup2d_b200.problems import seeded_disks

pytestmark = pytest.mark.gpu


def _cases():
    rng = np.random.default_rng(12)
    large = seeded_disks(np.random.default_rng(1), 3)
    return {
        # (bpdx, bpdy, levelMax, extent, periodic_x, periodic_y, disks, band)
        "small": (4, 2, 4, 2.0, False, False, [(0.6, 0.5, 0.1)], 0.15),
        "large_moved": (8, 4, 7, 2.0, False, False, [(cx + 0.02, cy, r) for cx, cy, r in large], 0.12),
        "periodic_x_edge": (4, 2, 5, 2.0, True, False, [(1.95, 0.5, 0.12)], 0.1),
        "periodic_xy_corner": (2, 2, 5, 1.0, True, True, [(0.02, 0.97, 0.1)], 0.06),
        "ten_disks": (8, 4, 5, 2.0, False, False, seeded_disks(rng, 10), 0.05),
        "no_disks": (4, 2, 4, 2.0, False, False, [], 0.1),
        "deep_thin": (2, 1, 8, 2.0, False, False, [(1.0, 0.5, 0.2)], 0.005),
    }


CASES = _cases()


@pytest.mark.parametrize("name", list(CASES))
def test_device_forest_equals_host(cuda, name):
    bpdx, bpdy, L_, ext, px, py, disks, band = CASES[name]
    host = Mesh.disks(bpdx, bpdy, L_, ext, disks, band, periodic_x=px, periodic_y=py)
    start = Mesh.uniform(bpdx, bpdy, L_, min(1, L_ - 1), ext, periodic_x=px, periodic_y=py)
    with Solver(start) as s:
        dev = s.adapt_disks(disks, band)
        assert s.ncells == host.ncells
        assert np.array_equal(dev.level, host.level)
        assert np.array_equal(dev.bx, host.bx)
        assert np.array_equal(dev.by, host.by)
        # the operator assembled from it is the oracle's, bit for bit
        rp, col, val = s.export_csr()
    rp_o, col_o, val_o = oracle.Matrix(host).csr()
    assert np.array_equal(rp, rp_o) and np.array_equal(col, col_o) and np.array_equal(val, val_o)


def test_adapt_remesh_step_equals_host_path(cuda):
    """One remesh of a time-stepping run: disks moved, forest adapted on the
    device, pressure carried over, warm-started solve -- the same bits as
    the host-forest path (update_mesh with the host generator's forest)."""
    import torch
    disks0 = seeded_disks(np.random.default_rng(1), 3)
    m0 = Mesh.disks(8, 4, 6, 2.0, disks0, 0.12)
    disks1 = [(cx + 0.05, cy, r) for cx, cy, r in disks0]
    m1 = Mesh.disks(8, 4, 6, 2.0, disks1, 0.12)
    assert m1.nblocks != m0.nblocks or not np.array_equal(m1.bx, m0.bx)
    with Solver(m0, tol_rel=1e-8, max_iter=5000) as cur, Solver(m0, tol_rel=1e-8, max_iter=5000) as dev, \
            Solver(m0, tol_rel=1e-8, max_iter=5000) as ref:
        b0 = torch.from_numpy(m0.rhs_fourier(3)).cuda()
        x0 = torch.zeros_like(b0)
        assert cur.solve_device(b0, x0)["status"] == L.OK
        dev.adapt_disks(disks1, 0.12)
        ref.update_mesh(m1)
        xd = torch.empty(m1.ncells, dtype=torch.float64, device=cuda)
        xr = torch.empty_like(xd)
        cur.transfer_to(dev, x0, xd)
        cur.transfer_to(ref, x0, xr)
        torch.cuda.synchronize()
        assert torch.equal(xd, xr)
        b1 = torch.from_numpy(m1.rhs_fourier(4)).cuda()
        sd = dev.solve_device(b1, xd)
        sr = ref.solve_device(b1, xr)
        assert sd["status"] == sr["status"] == L.OK
        assert sd["iterations"] == sr["iterations"]
        assert torch.equal(xd, xr)


def test_adapt_arguments(cuda):
    m = Mesh.uniform(2, 1, 3, 1, 2.0)
    with Solver(m) as s:
        with pytest.raises(Cup2dError) as e:
            s.adapt_disks([(0.5, 0.5, 0.1)] * 65, 0.1)
        assert e.value.status == L.INVALID_ARGUMENT
        with pytest.raises(Cup2dError) as e:
            s.adapt_disks([(0.5, 0.5, 0.1)], -1.0)
        assert e.value.status == L.INVALID_ARGUMENT
        # the handle is unchanged and still solves
        assert s.ncells == m.ncells
        x = s.solve(m.rhs_fourier(1))
        assert s.last_stats["status"] == L.OK and x.shape == (m.ncells,)
