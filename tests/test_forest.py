"""Host-side forests and synthetic right-hand sides (no GPU)."""
import numpy as np
import pytest

from cup2d_b200 import Mesh, fourier_advance, fourier_coefs
from cup2d_b200.problems import large_mesh, loguniform_sizes, sized_mesh, small_mesh


def _morton(m: Mesh):
    top = m.level_max - 1
    fx = m.bx.astype(np.int64) << (top - m.level)
    fy = m.by.astype(np.int64) << (top - m.level)

    def spread(v):
        out = np.zeros_like(v)
        for bit in range(31):
            out |= ((v >> bit) & 1) << (2 * bit)
        return out
    return spread(fx) | (spread(fy) << 1)


def test_small_config():
    m = small_mesh()
    assert m.validate()
    assert m.nblocks == 128 and m.ncells == 8192
    assert set(m.level.tolist()) == {0, 1, 2, 3}
    # finest-level blocks are children of parents that met the band
    # |dist - r| <= 0.15, so they lie within one parent diagonal of it
    h = m.cell_h()
    fine = m.level == 3
    cx = (m.bx[fine] + 0.5) * 8 * h[fine]
    cy = (m.by[fine] + 0.5) * 8 * h[fine]
    d = np.hypot(cx - 0.6, cy - 0.5)
    parent_diag = 16 * h[fine] * np.sqrt(2)
    assert np.all(np.abs(d - 0.1) <= 0.15 + parent_diag)
    # and the blocks nearest the disk edge are at the finest level
    cxa = (m.bx + 0.5) * 8 * h
    cya = (m.by + 0.5) * 8 * h
    near = np.abs(np.hypot(cxa - 0.6, cya - 0.5) - 0.1) < 0.05
    assert np.all(m.level[near] == 3)


def test_large_config_size():
    m = large_mesh()
    assert m.validate()
    assert 19000 <= m.nblocks <= 22000
    assert 1.2e6 <= m.ncells <= 1.45e6
    assert m.level.max() == 6


def test_morton_order_and_determinism():
    m1 = sized_mesh(np.random.default_rng(11), 900)
    m2 = sized_mesh(np.random.default_rng(11), 900)
    assert np.array_equal(m1.level, m2.level) and np.array_equal(m1.bx, m2.bx) and np.array_equal(m1.by, m2.by)
    k = _morton(m1)
    assert np.all(np.diff(k) > 0)


@pytest.mark.parametrize("periodic", [(False, False), (True, False), (True, True)])
def test_balance_faces_and_corners(periodic):
    m = Mesh.disks(3, 2, 6, 3.0, [(0.4, 0.3, 0.05), (2.5, 1.7, 0.08)], 0.03, *periodic)
    assert m.validate()
    # explicit 2:1 check over faces and corners
    leaves = {(l, i, j) for l, i, j in zip(m.level.tolist(), m.bx.tolist(), m.by.tolist())}
    for l, i, j in leaves:
        nx, ny = m.bpdx << l, m.bpdy << l
        for di in (-1, 0, 1):
            for dj in (-1, 0, 1):
                if di == dj == 0:
                    continue
                ni, nj = i + di, j + dj
                if periodic[0]:
                    ni %= nx
                if periodic[1]:
                    nj %= ny
                if not (0 <= ni < nx and 0 <= nj < ny):
                    continue
                for q in range(l, -1, -1):
                    if (q, ni >> (l - q), nj >> (l - q)) in leaves:
                        assert q >= l - 1
                        break


def test_invalid_forests_rejected():
    # overlap: a block and its parent
    m = Mesh(1, 1, 2, 1.0, np.array([0, 1, 1, 1, 1]), np.array([0, 0, 1, 0, 1]), np.array([0, 0, 0, 1, 1]))
    assert not m.validate()
    # hole: one child missing
    m = Mesh(1, 1, 2, 1.0, np.array([1, 1, 1]), np.array([0, 1, 0]), np.array([0, 0, 1]))
    assert not m.validate()
    # out of range
    m = Mesh(1, 1, 2, 1.0, np.array([1, 1, 1, 1]), np.array([0, 1, 0, 2]), np.array([0, 0, 1, 1]))
    assert not m.validate()


def test_rhs_zero_sum_and_seeded():
    m = small_mesh()
    b1 = m.rhs_fourier(7)
    b2 = m.rhs_fourier(7)
    b3 = m.rhs_fourier(8)
    assert np.array_equal(b1, b2)
    assert not np.allclose(b1, b3)
    assert abs(b1.sum()) < 1e-14 * np.abs(b1).sum()
    assert np.abs(b1).max() > 0


def test_rhs_is_divergence_of_fourier_field():
    # on a uniform periodic mesh the central-difference divergence of a
    # single mode is known in closed form; check the magnitude scaling with h
    m1 = Mesh.uniform(2, 1, 3, 1, 2.0)
    m2 = Mesh.uniform(2, 1, 3, 2, 2.0)
    r1 = np.abs(m1.rhs_fourier(3)).max() / m1.cell_h()[0] ** 2
    r2 = np.abs(m2.rhs_fourier(3)).max() / m2.cell_h()[0] ** 2
    # b = h^2 div(u) + O(h^4): the scaled maxima agree to O(h^2)
    assert abs(r1 - r2) / r2 < 0.2


def test_ar1_coefficients():
    c0 = fourier_coefs(5)
    c1 = fourier_advance(c0, 5, 1, rho=0.95)
    assert c0.shape == c1.shape
    corr = np.corrcoef(c0, c1)[0, 1]
    assert 0.85 < corr < 0.999
    assert np.array_equal(c1, fourier_advance(c0, 5, 1, rho=0.95))


def test_loguniform_sizes():
    s = loguniform_sizes(np.random.default_rng(0), 4000, 50, 6000)
    assert s.min() >= 50 and s.max() <= 6000
    med = np.median(np.log(s))
    assert abs(med - 0.5 * (np.log(50) + np.log(6000))) < 0.1


def test_sized_mesh_hits_target():
    rng = np.random.default_rng(2)
    for target in (60, 500, 3000):
        m = sized_mesh(rng, target)
        assert m.validate()
        assert 0.5 * target <= m.nblocks <= 2.0 * target
