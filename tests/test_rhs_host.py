"""Host generator of the time-stepping RHS: Fourier coefficients, their
AR(1) evolution and the RHS built from them (the reference the device RHS
kernel is checked against)."""
import numpy as np

from cup2d_b200.mesh import fourier_advance, fourier_coefs
from cup2d_b200.problems import small_mesh


def test_coefs_deterministic_and_ar1():
    c0 = fourier_coefs(5)
    assert np.array_equal(c0, fourier_coefs(5)) and not np.array_equal(c0, fourier_coefs(6))
    assert np.array_equal(fourier_advance(c0, 5, 3, rho=1.0), c0)         # rho = 1: frozen
    c1 = fourier_advance(c0, 5, 3)
    assert np.array_equal(c1, fourier_advance(c0, 5, 3))                   # seeded per step
    assert not np.array_equal(c1, fourier_advance(c0, 5, 4))
    assert 0.9 < np.corrcoef(c0, c1)[0, 1] < 0.99                          # rho = 0.95
    c = c0.copy()
    for k in range(200):
        c = fourier_advance(c, 5, k)
    assert 0.7 < np.std(c) < 1.3                                           # stationary N(0, 1)


def test_rhs_from_coefs():
    m = small_mesh()
    c = fourier_coefs(17)
    b = m.rhs_from_coefs(c)
    assert np.array_equal(b, m.rhs_fourier(17))
    assert abs(b.sum()) <= 1e-12 * np.abs(b).sum()                         # Neumann compatible
    assert not np.array_equal(b, m.rhs_from_coefs(fourier_advance(c, 17, 0)))
