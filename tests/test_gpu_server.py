"""GPU tests of the request server: continuous admission of solves of
different sizes, resident meshes, warm starts, admission by memory budget.

A request runs the same persistent solve as a single solve with grid = team
(same block ranges, same reduction order), so its result is bit-identical
to that solve run alone, whatever else is on the device meanwhile.
"""
import threading

import numpy as np
import pytest

from cup2d_b200 import Cup2dError, Server, Solver
from cup2d_b200 import _lib as L
from cup2d_b200.problems import loguniform_sizes, sized_mesh, small_mesh

pytestmark = pytest.mark.gpu

TEAM = 4


def _meshes():
    rng = np.random.default_rng(21)
    ms = [small_mesh()]
    for n in loguniform_sizes(rng, 5, 60, 1500):
        ms.append(sized_mesh(rng, int(n)))
    return ms


MESHES = _meshes()


def _solo(mesh, b, precision="fp64"):
    with Solver(mesh, tol_rel=1e-8, max_iter=5000, precision=precision) as s:
        s.set_grid(TEAM)
        x = s.solve(b)
        return x, s.last_stats


def _requests(n_per_mesh=3, seed0=300):
    out = []
    for i, m in enumerate(MESHES):
        for k in range(n_per_mesh):
            out.append((i, m.rhs_fourier(seed0 + 10 * i + k)))
    return out


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_server_results_equal_alone(cuda, precision):
    reqs = _requests()
    with Server(max_inflight=8, team=TEAM, tol_rel=1e-8, max_iter=5000, precision=precision) as S:
        ids = [S.add_mesh(m) for m in MESHES]
        xs = [np.zeros_like(b) for _, b in reqs]
        rids = [S.submit(ids[i], b, x) for (i, b), x in zip(reqs, xs)]
        stats = [S.wait(r) for r in rids]
        c = S.counters()
    assert all(s is not None and s["status"] == L.OK for s in stats), stats
    assert c["completed"] == len(reqs) and c["failed"] == 0 and c["queued"] == 0 and c["inflight"] == 0
    assert c["assemblies"] == len(MESHES)  # every mesh assembled once, then resident
    for (i, b), x, st in zip(reqs, xs, stats):
        x_solo, st_solo = _solo(MESHES[i], b, precision)
        assert st["iterations"] == st_solo["iterations"]
        assert np.array_equal(x, x_solo), (i, np.max(np.abs(x - x_solo)))
        assert st["latency_ms"] > 0.0


def test_server_small_budget_evicts(cuda):
    """A budget that holds about two of the meshes: every request still runs
    (idle meshes are evicted and re-assembled), with the same results."""
    reqs = _requests(n_per_mesh=2, seed0=500)
    big = max(m.nblocks for m in MESHES)
    budget = int(1.5 * big * 9216) + (2 << 20)
    with Server(max_inflight=4, team=TEAM, hbm_budget_bytes=budget, tol_rel=1e-8, max_iter=5000) as S:
        ids = [S.add_mesh(m) for m in MESHES]
        order = list(range(len(reqs)))
        np.random.default_rng(0).shuffle(order)
        xs = {k: np.zeros_like(reqs[k][1]) for k in order}
        rids = {k: S.submit(ids[reqs[k][0]], reqs[k][1], xs[k]) for k in order}
        stats = {k: S.wait(rids[k]) for k in order}
        c = S.counters()
    assert all(s["status"] == L.OK for s in stats.values())
    assert c["evictions"] > 0 and c["assemblies"] > len(MESHES)
    assert c["resident_bytes"] <= budget
    for k in order:
        i, b = reqs[k]
        x_solo, _ = _solo(MESHES[i], b)
        assert np.array_equal(xs[k], x_solo)


def test_server_warm_start(cuda):
    m = MESHES[3]
    b = m.rhs_fourier(7)
    # an absolute tolerance: relative to a warm start's tiny initial residual
    # the same relative target would be out of reach
    tol = 1e-8 * float(np.max(np.abs(b)))
    with Server(max_inflight=2, team=TEAM, tol_rel=0.0, tol_abs=tol, max_iter=5000) as S:
        mid = S.add_mesh(m)
        x1 = np.zeros_like(b)
        s1 = S.wait(S.submit(mid, b, x1))
        x2 = np.zeros_like(b)
        s2 = S.wait(S.submit(mid, b, x2, warm_start=True))
    assert s1["status"] == L.OK and s2["status"] == L.OK
    assert s2["err_init"] <= 1e-6 * s1["err_init"]
    assert s2["iterations"] <= max(3, s1["iterations"] // 4)
    assert np.max(np.abs(x2 - x1)) <= 1e-6 * np.max(np.abs(x1))


def test_server_threads(cuda):
    """Submitters on several host threads at once."""
    with Server(max_inflight=6, team=TEAM, tol_rel=1e-6) as S:
        ids = [S.add_mesh(m) for m in MESHES]
        errors = []

        def client(t):
            try:
                rng = np.random.default_rng(t)
                for k in range(6):
                    i = int(rng.integers(len(MESHES)))
                    b = MESHES[i].rhs_fourier(1000 * t + k)
                    x = np.zeros_like(b)
                    st = S.wait(S.submit(ids[i], b, x))
                    if st is None or st["status"] != L.OK:
                        errors.append((t, k, st))
            except Exception as e:  # pragma: no cover - reported below
                errors.append((t, repr(e)))

        th = [threading.Thread(target=client, args=(t,)) for t in range(4)]
        for t in th:
            t.start()
        for t in th:
            t.join()
        c = S.counters()
    assert not errors, errors
    assert c["completed"] == 24


def test_server_take_completed(cuda):
    """The completion queue reports each finished request once, and no
    request that was already collected with wait."""
    reqs = _requests(n_per_mesh=1, seed0=700)
    with Server(max_inflight=4, team=TEAM, tol_rel=1e-6) as S:
        ids = [S.add_mesh(m) for m in MESHES]
        xs = [np.zeros_like(b) for _, b in reqs]
        rids = [S.submit(ids[i], b, x) for (i, b), x in zip(reqs, xs)]
        first = S.wait(rids[0])
        seen = []
        while len(seen) < len(rids) - 1:
            got = S.take_completed(timeout_ms=5000)
            assert got, "no completion within 5 s"
            seen += got
        stats = [S.poll(r) for r in seen]
        assert S.take_completed(timeout_ms=0) == []
    assert first["status"] == L.OK
    assert sorted(seen) == sorted(rids[1:])
    assert all(s["status"] == L.OK for s in stats)


def test_server_errors(cuda):
    m = MESHES[0]
    b = m.rhs_fourier(1)
    x = np.zeros_like(b)
    with Server(max_inflight=2, team=TEAM, hbm_budget_bytes=1 << 20) as S:
        with pytest.raises(Cup2dError):
            S.submit(12345, b, x)
        mid = S.add_mesh(MESHES[-1])   # larger than the 1 MiB budget
        bb = MESHES[-1].rhs_fourier(1)
        st = S.wait(S.submit(mid, bb, np.zeros_like(bb)))
        assert st["status"] == L.OOM
        with pytest.raises(Cup2dError):
            S.poll(987654)
