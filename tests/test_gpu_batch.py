"""GPU tests of batched solves: many uneven problems in one persistent launch.

Each problem of a batch is solved by a group of `team` CTAs with the same
code as a single solve on a grid of `team` CTAs (same block ranges, same
reduction order), so a batch result is bit-identical to that single solve,
and to the same problem alone in a batch of one: a problem's result does
not depend on what else is in the batch.
"""
import numpy as np
import pytest

import oracle
from cup2d_b200 import BatchSolver, Cup2dError, Mesh, Solver
from cup2d_b200 import _lib as L
from cup2d_b200.problems import loguniform_sizes, sized_mesh, small_mesh

pytestmark = pytest.mark.gpu


def _meshes():
    rng = np.random.default_rng(11)
    ms = [small_mesh(), Mesh.uniform(1, 1, 1, 0, 1.0),
          Mesh.disks(4, 2, 4, 2.0, [(1.0, 0.5, 0.12)], 0.1, periodic_x=True)]
    for n in loguniform_sizes(rng, 7, 50, 1500):
        ms.append(sized_mesh(rng, int(n)))
    return ms


MESHES = _meshes()


def _device_rhs(torch, cuda, meshes, seed0=100):
    bs = [torch.from_numpy(m.rhs_fourier(seed0 + i)).to(cuda) for i, m in enumerate(meshes)]
    xs = [torch.zeros_like(b) for b in bs]
    return bs, xs


def _rel_l2(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("team", [1, 4])
def test_batch_bit_identical_to_single(cuda, precision, team):
    import torch
    bs, xs = _device_rhs(torch, cuda, MESHES)
    with BatchSolver(MESHES, tol_rel=1e-8, max_iter=5000, precision=precision, team=team) as B:
        stats = B.solve_device(bs, xs)
    for i, m in enumerate(MESHES):
        x1 = torch.zeros_like(bs[i])
        with Solver(m, tol_rel=1e-8, max_iter=5000, precision=precision) as s:
            s.set_grid(team)
            st = s.solve_device(bs[i], x1)
        assert stats[i]["status"] == L.OK == st["status"], (i, stats[i], st)
        assert stats[i]["iterations"] == st["iterations"]
        assert stats[i]["refinements"] == st["refinements"]
        assert torch.equal(xs[i], x1), (i, (xs[i] - x1).abs().max().item())


def test_batch_alone_equals_in_mix(cuda):
    import torch
    k = 5
    bs, xs = _device_rhs(torch, cuda, MESHES)
    with BatchSolver(MESHES, tol_rel=1e-6, precision="mixed", team=4) as B:
        B.solve_device(bs, xs)
    b1 = [bs[k].clone()]
    x1 = [torch.zeros_like(bs[k])]
    with BatchSolver([MESHES[k]], tol_rel=1e-6, precision="mixed", team=4) as B1:
        B1.solve_device(b1, x1)
    assert torch.equal(xs[k], x1[0])


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_batch_matches_oracle(cuda, precision):
    import torch
    meshes = MESHES[:6]
    bs, xs = _device_rhs(torch, cuda, meshes)
    with BatchSolver(meshes, tol_rel=1e-8, max_iter=8000, precision=precision, team=8) as B:
        stats = B.solve_device(bs, xs)
    for i, m in enumerate(meshes):
        b = bs[i].cpu().numpy()
        x = xs[i].cpu().numpy()
        x_o, st_o = oracle.solve(m, b, tol_rel=1e-10, max_iter=8000)
        assert stats[i]["status"] == L.OK, (i, stats[i])
        # FP64 true residual of the returned solution (x0 = 0, so r0 = b)
        r = b - oracle.Matrix(m).spmv(x)
        assert np.max(np.abs(r)) <= 1.5e-8 * np.max(np.abs(b)), i
        assert _rel_l2(x, x_o) <= 1e-6, (i, _rel_l2(x, x_o))


def test_batch_warm_start_and_repeat(cuda):
    """Solving again from the converged solutions starts from a residual
    near the first tolerance and takes a few iterations (the true residual
    of the returned solution can sit above the recursive one that stopped
    the first solve), and the launch can be repeated on the same batch."""
    import torch
    meshes = MESHES[:4]
    bs, xs = _device_rhs(torch, cuda, meshes)
    with BatchSolver(meshes, tol_rel=1e-8, precision="fp64", team=2) as B:
        first = B.solve_device(bs, xs)
        # every first solve ended at |r|_inf <= 1e-8 |b|_inf; an absolute
        # tolerance just above the largest of those is already met
        tol = 2e-8 * max(float(b.abs().max()) for b in bs)
        assert all(s["err_final"] <= tol for s in first)
        B.set_opts(tol_rel=0.0, tol_abs=tol, precision="fp64")
        st = B.solve_device(bs, xs)
    for s0, s in zip(first, st):
        assert s["status"] == L.OK
        assert s["err_init"] <= 1e-6 * s0["err_init"]
        assert s["iterations"] <= max(3, s0["iterations"] // 4)


def test_batch_arguments(cuda):
    import torch
    meshes = MESHES[:3]
    bs, xs = _device_rhs(torch, cuda, meshes)
    with BatchSolver(meshes) as B:
        assert len(B) == 3
        assert [B.ncells(i) for i in range(3)] == [m.ncells for m in meshes]
        with pytest.raises(Cup2dError):
            B.set_team(0)
        with pytest.raises(ValueError):
            B.solve_device(bs[:2], xs[:2])
        with pytest.raises(ValueError):
            B.solve_device(bs, [xs[1], xs[0], xs[2]])  # sizes differ
    with pytest.raises(Cup2dError):
        BatchSolver([])


def test_batch_autotune(cuda, tmp_path):
    """The autotuner keeps the fastest candidate launch shape, the batch then
    solves with it, and a second call with the same cache reuses the choice
    without timing."""
    import torch
    bs, xs = _device_rhs(torch, cuda, MESHES)
    cache = str(tmp_path / "tune.json")
    with BatchSolver(MESHES, tol_rel=1e-6, precision="mixed") as B:
        best = B.autotune(bs, xs, teams=(1, 2, 4, 8), ctas_per_sm=(0, 1), iters=10, cache=cache)
        rates = B.tune_rates
        assert best in rates and rates[best] == max(rates.values()) and rates[best] > 0
        assert len(rates) == 8
        # the chosen team is in use: results equal a single solve on that grid
        for x in xs:
            x.zero_()
        st = B.solve_device(bs, xs)
    assert all(s["status"] == L.OK for s in st)
    with Solver(MESHES[2], tol_rel=1e-6, precision="mixed") as s1:
        s1.set_grid(best[0])
        x1 = torch.zeros_like(bs[2])
        s1.solve_device(bs[2], x1)
    assert torch.equal(x1, xs[2])
    with BatchSolver(MESHES, tol_rel=1e-6, precision="mixed") as B2:
        assert B2.autotune(bs, xs, teams=(1, 2, 4, 8), ctas_per_sm=(0, 1), iters=10, cache=cache) == best
        assert not hasattr(B2, "tune_rates")


def test_batch_occupancy_cap(cuda):
    """An occupancy cap changes how many problems run at once, never a
    problem's result."""
    import torch
    bs, xs = _device_rhs(torch, cuda, MESHES)
    with BatchSolver(MESHES, tol_rel=1e-8, max_iter=5000, team=4) as B:
        B.solve_device(bs, xs)
        ys = [torch.zeros_like(b) for b in bs]
        B.set_occupancy(1)
        B.solve_device(bs, ys)
        with pytest.raises(Cup2dError):
            B.set_occupancy(-1)
    assert all(torch.equal(x, y) for x, y in zip(xs, ys))


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_batch_graph_replay(cuda, precision):
    """A captured batch replays to the same results as solve_device: cold
    (x zeroed inside the graph) with the captured b, and after b is
    overwritten in place, warm from the previous replay's x."""
    import torch
    bs, xs = _device_rhs(torch, cuda, MESHES)
    tol = dict(tol_rel=1e-8, max_iter=5000, precision=precision, team=4)
    with BatchSolver(MESHES, **tol) as B:
        ref = B.solve_device(bs, [torch.zeros_like(b) for b in bs])
        xref = [torch.zeros_like(b) for b in bs]
        B.solve_device(bs, xref)
        B.capture(bs, xs, zero_x=True)
        for x in xs:
            x.fill_(1.0)  # zeroed by the graph
        for _ in range(2):
            B.replay()
            st = B.replay_stats()
            assert [s["iterations"] for s in st] == [s["iterations"] for s in ref]
            assert all(torch.equal(x, y) for x, y in zip(xs, xref))
        # time stepping: new b in place, warm start from the last solution
        B.capture(bs, xs)
        warm = [x.clone() for x in xs]
        for b, m, i in zip(bs, MESHES, range(len(bs))):
            b.copy_(torch.from_numpy(m.rhs_fourier(900 + i)))
        B.replay()
        st = B.replay_stats()
        assert all(s["status"] == L.OK for s in st)
        B.solve_device(bs, warm)
        assert all(torch.equal(x, y) for x, y in zip(xs, warm))
    with pytest.raises(Cup2dError):
        with BatchSolver(MESHES[:2], **tol) as B2:
            B2.replay()
