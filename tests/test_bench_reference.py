"""bench.py's timing of the reference's own GPU path (`--impl reference
--ref-gpu`) on CPU, with the reference checker stubbed: the line it prints
(same workload string as the GPU arm, the fixed part of a call reported
beside the solves/s), and the `unavailable` line when the checker's GPU build
is missing."""
import argparse
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent.parent
sys.path.insert(0, str(ROOT))


def _args(**kw):
    base = dict(impl="reference", workload="batch", ref_gpu=True, batch=128, warmup=3, steps=2)
    base.update(kw)
    return argparse.Namespace(**base)


def test_ref_gpu_unavailable_without_checker(monkeypatch):
    import bench
    import oracle.ref as R
    monkeypatch.setattr(R, "available", lambda kind="cpu": False)
    line = bench.run_reference(_args(), 1, 0)
    assert line["impl"] == "reference" and "unavailable" in line


def test_ref_gpu_line(monkeypatch):
    import bench
    import oracle.ref as R
    from cup2d_b200.problems import batch_problems
    calls = []

    def fake_solve(mesh, b, tol_rel=1e-8, **kw):
        calls.append((mesh.nblocks, tol_rel))
        big = mesh.nblocks > 3000
        return np.zeros_like(b), {"converged": tol_rel >= 1.0 or not big,
                                  "iterations": 1 if tol_rel >= 1.0 else (1000 if big else 200)}

    monkeypatch.setattr(R, "available", lambda kind="cpu": True)
    monkeypatch.setattr(R, "solve", fake_solve)
    line = bench.run_reference(_args(), 1, 0)
    meshes = batch_problems(128, seed=3)
    assert line["config"]["workload"] == bench.batch_label(meshes, 0)
    assert line["impl"] == "reference" and line["cpu_baseline"]["kind"] == "reference"
    assert line["value"] > 0 and line["solve_only"]["value"] >= line["value"]
    assert line["per_call_fixed_ms"] >= 0
    # every problem of the 5 slices is solved twice: to 1e-6, then at tol_rel = 1
    parts = bench.cpu_slices(meshes)
    n = sum(len(parts[k]) for k in range(5))
    assert len(calls) == 2 * n
    assert sorted(t for _, t in calls) == [bench.TOL] * n + [1.0] * n
    timed = sum(len(parts[k]) for k in range(3, 5))
    big = sum(1 for k in range(3, 5) for i in parts[k] if meshes[i].nblocks > 3000)
    assert line["capped"] == big
    assert f"{timed} solves in " in line["cpu_baseline"]["sample"]
