"""The allocation-free FP64 solve against the allocating one.

cup2d_poisson_solve_device_noalloc serves callers that must not allocate
device memory at solve time (device memory owned by their own pool, or a loop
that cannot afford an allocation's synchronisation).  Its scratch is one
static device array shared by every call, so this file checks two calls in
a row (the second sees the first one's leftovers), that the device's free
memory does not change across a call, the size limit, and that the results
match the allocating entry point.  It is collected last so that a
run stopping at the first failure has already run every other test.
"""
import ctypes as C

import numpy as np
import pytest

from cup2d_b200 import Cup2dError, Solver
from cup2d_b200 import _lib as L
from cup2d_b200.problems import sized_mesh, small_mesh

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.mark.parametrize("mesh_fn", [small_mesh, lambda: sized_mesh(np.random.default_rng(21), 2500)])
def test_noalloc_matches_allocating_solve(cuda, mesh_fn):
    import torch
    m = mesh_fn()
    assert m.nblocks <= 4096
    rhs = [torch.from_numpy(m.rhs_fourier(s)).to(cuda) for s in (31, 32)]
    with Solver(m, tol_rel=1e-8, max_iter=5000) as s:
        ref = []
        for b in rhs:
            x = torch.zeros_like(b)
            st = s.solve_device(b, x)
            assert st["status"] == L.OK
            ref.append((x.cpu().numpy(), st))
        # two calls in a row through the C ABI; the second reuses the static
        # scratch the first one left behind.  The device's free memory is
        # the same before and after each call: the static array was
        # committed when the handle was created, and the call allocates
        # nothing (no pool growth, no module load).
        for (x_ref, st_ref), b in zip(ref, rhs):
            x = torch.zeros_like(b)
            torch.cuda.synchronize()
            free_before = torch.cuda.mem_get_info()[0]
            st = s.solve_device_noalloc(b, x)
            torch.cuda.synchronize()
            assert torch.cuda.mem_get_info()[0] == free_before
            assert st["status"] == L.OK, st
            assert st["rel_res_inf"] <= 1e-8
            # same kernel, grid and block ranges: the result matches the
            # allocating path within the solver tests' FP64 tolerance
            assert _rel(x.cpu().numpy(), x_ref) <= 1e-12
            assert st["iterations"] == st_ref["iterations"]


def test_noalloc_rejects_too_large(cuda):
    import torch
    from cup2d_b200.problems import large_mesh
    m = large_mesh()
    assert m.nblocks > 4096
    with Solver(m) as s:
        b = torch.zeros(m.ncells, dtype=torch.float64, device=cuda)
        x = torch.zeros_like(b)
        with pytest.raises(Cup2dError) as e:
            s.solve_device_noalloc(b, x)
        assert e.value.status == L.INVALID_ARGUMENT
        # the handle and the allocating path are unaffected
        st = s.solve_device(b, x)
        assert st["status"] in (L.OK, L.NOT_CONVERGED)
