"""Properties of the restated transfer rule (what the device kernel is
compared with), on the CPU: identity on the same forest, constants
preserved, every value a copy or a convex mean of source values."""
import numpy as np

from tests.transfer_rule import disk_mesh, transfer_restated


def test_identity_and_constants():
    a = disk_mesh(0.0, level_max=4)
    xs = np.random.default_rng(0).standard_normal(a.ncells)
    assert np.array_equal(transfer_restated(a, xs, a), xs)
    b = disk_mesh(0.03, level_max=4)
    assert np.all(transfer_restated(a, np.full(a.ncells, 2.5), b) == 2.5)


def test_values_within_source_range():
    a, b = disk_mesh(0.0, level_max=4), disk_mesh(0.05, level_max=4)
    assert set(zip(a.level, a.bx, a.by)) != set(zip(b.level, b.bx, b.by))  # refined and coarsened
    xs = np.random.default_rng(1).uniform(-1.0, 3.0, a.ncells)
    xd = transfer_restated(a, xs, b)
    assert xd.shape == (b.ncells,)
    assert xd.min() >= xs.min() and xd.max() <= xs.max()
    back = transfer_restated(b, xd, a)
    assert back.min() >= xs.min() and back.max() <= xs.max()
