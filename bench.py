"""Benchmark: Poisson solves/s and p50/p99 latency on one B200 (or N replicas).

Workload (default "large"): the block-AMR pressure-Poisson problem of
bpdx=8, bpdy=4, levelMax=7 refined near 3 seeded disks (20,834 blocks,
1,333,376 cells), divergence-of-random-Fourier-velocity right-hand sides
(one seed per step), x0 = 0, solved to relative true L-inf residual 1e-6.
A step is one solve.  The headline `value` is the mixed-precision solver
(FP32 Krylov vectors, FP64 solution and true residual); the plain FP64
solver (the reference's algorithm) is timed on the same right-hand sides
and reported under "plain_fp64".

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

--impl reference times the reference's algorithm on the host CPU: the C++
restatement of ExpAMRSolver + BiCGSTABSolver::main (CUP2D's own CPU build
needs its un-vendored Cubism submodule, MPI, HDF5 and GSL).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "Poisson solves/s at rel-res 1e-6 (batched-mixed vs plain FP64)"
UNIT = "solves/s"
TOL = 1e-6


def _peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clock/throttle samples during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *a):
        self.out = ""
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.out, _ = self.proc.communicate(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
                self.out = ""

    def summary(self) -> dict:
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in (self.out or "").splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = max(mx, float(f[2]))
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx or None,
                "reasons": sorted(reasons), "samples": len(sm)}


def _dist():
    import torch
    import torch.distributed as dist
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1 and not dist.is_initialized():
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300), device_id=torch.device("cuda", local))
    return world, rank, local


def _max_over_ranks(v: float, world: int) -> float:
    if world == 1:
        return v
    import torch
    import torch.distributed as dist
    t = torch.tensor([v], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def _barrier(world: int):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def algorithmic_bytes(n: int, nb: int, R: int, nnz: int, iters: int, updates: int, precision: str) -> float:
    """Bytes one solve must move: the fused five-pass schedule per BiCGSTAB
    iteration (vector streams) plus the explicit coarse/fine rows and the
    per-block neighbour table read by each of its two SpMVs.

    FP64: 25 vector streams x 8 B per cell.  Mixed: FP32 r, rhat, p, nu, t, z
    and the FP64 solution x read+written in passes C and E = 116 B per cell;
    each true-residual refresh reads x, b (FP64) and rhat, writes r (FP32).
    Matrix: 12 B per stored non-zero (FP64) or 8 B (FP32) + 4 B per stored
    row, and 28 B per block of structure (neighbours, row mask, row base)."""
    meta = 28.0 * nb
    if precision == "fp64":
        mat = 12.0 * nnz + 4.0 * R + meta
        per_iter = 25 * 8.0 * n + 2 * mat
        setup = (8 + 8 + 8 + 8) * n + mat   # r = b - A x0, rhat: R x,b W r,rhat
        final = 16.0 * n                     # mean removal: R x, W x
        return setup + iters * per_iter + final
    mat32 = 8.0 * nnz + 4.0 * R + meta
    mat64 = 12.0 * nnz + 4.0 * R + meta
    per_iter = 116.0 * n + 2 * mat32
    per_update = (8 + 8 + 4 + 4) * n + mat64
    setup = 8.0 * n + (8 + 8 + 4 + 4) * n + mat64   # sum b; true residual, rhat
    final = 16.0 * n
    return setup + iters * per_iter + updates * per_update + final


def run_ours(args, world, rank, local) -> dict | None:
    import numpy as np
    import torch

    from cup2d_b200 import Solver
    from cup2d_b200.problems import large_mesh, small_mesh

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    mesh = large_mesh() if args.workload == "large" else small_mesh()
    n = mesh.ncells
    seeds = [1000 * rank + 17 + s for s in range(args.warmup + args.steps)]
    bs = [torch.from_numpy(mesh.rhs_fourier(s)).to(dev) for s in seeds]
    x = torch.zeros(n, dtype=torch.float64, device=dev)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)  # 256 MiB > L2
    solver = Solver(mesh, tol_rel=TOL, max_iter=20000, max_restarts=100)
    R, nnz = solver.explicit_info()
    stream = torch.cuda.current_stream(dev)

    def timed(precision: str):
        """Device time of each solve (CUDA events on the launching stream);
        x0 = 0 is written inside the timed region, the L2 flush outside."""
        solver.set_opts(tol_rel=TOL, max_iter=20000, max_restarts=100, precision=precision)
        ms = []
        for i, b in enumerate(bs):
            flush.fill_(float(i))
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            x.zero_()
            solver.solve_device(b, x, stream=stream, stats=False)
            e1.record(stream)
            torch.cuda.synchronize(dev)
            if i >= args.warmup:
                ms.append(e0.elapsed_time(e1))
        return ms

    # stats pass (untimed): iterations / updates per right-hand side
    def stats_pass(precision: str):
        solver.set_opts(tol_rel=TOL, max_iter=20000, max_restarts=100, precision=precision)
        out = []
        for b in bs[args.warmup:]:
            x.zero_()
            out.append(solver.solve_device(b, x, stream=stream, stats=True))
        return out

    _barrier(world)
    with ClockSampler(local) as clk:
        ms_mixed = timed("mixed")
        ms_fp64 = timed("fp64")
    st_mixed = stats_pass("mixed")
    st_fp64 = stats_pass("fp64")
    tot_mixed = _max_over_ranks(sum(ms_mixed), world)
    tot_fp64 = _max_over_ranks(sum(ms_fp64), world)

    # end to end through the public host-buffer API (pinned host memory)
    solver.set_opts(tol_rel=TOL, max_iter=20000, max_restarts=100, precision="mixed")
    hb = [torch.from_numpy(mesh.rhs_fourier(s)).pin_memory() for s in seeds[args.warmup:]]
    hx = torch.zeros(n, dtype=torch.float64).pin_memory()
    _barrier(world)
    torch.cuda.synchronize(dev)
    t0 = time.perf_counter()
    for b in hb:
        hx.zero_()
        solver.solve(b.numpy(), out=hx.numpy())
    e2e_s = _max_over_ranks(time.perf_counter() - t0, world)

    if rank != 0:
        return None
    peak, peak_kind = _peaks()
    K = args.steps
    it_m = [s["iterations"] for s in st_mixed]
    up_m = [s["refinements"] for s in st_mixed]
    it_d = [s["iterations"] for s in st_fp64]
    bytes_m = [algorithmic_bytes(n, mesh.nblocks, R, nnz, i, u, "mixed") for i, u in zip(it_m, up_m)]
    bytes_d = [algorithmic_bytes(n, mesh.nblocks, R, nnz, i, 0, "fp64") for i in it_d]
    ach_m = sum(bytes_m) / (sum(ms_mixed) * 1e-3) / 1e9
    ach_d = sum(bytes_d) / (sum(ms_fp64) * 1e-3) / 1e9
    lat = sorted(ms_mixed)
    latd = sorted(ms_fp64)

    def pct(v, q):
        return v[min(len(v) - 1, int(round(q * (len(v) - 1))))]

    # DRAM bytes per launch: the per-iteration traffic of one ncu capture of
    # this workload (profiles/traffic.json) times this run's iterations
    traffic = traffic_d = None
    tp = ROOT / "profiles" / "traffic.json"
    if tp.exists():
        tj = json.loads(tp.read_text()).get(args.workload, {})
        if "dram_bytes_per_iteration_mixed" in tj:
            traffic = tj["dram_bytes_per_iteration_mixed"] * (sum(it_m) / K)
        if "dram_bytes_per_iteration_fp64" in tj:
            traffic_d = tj["dram_bytes_per_iteration_fp64"] * (sum(it_d) / K)
    value = world * K / (tot_mixed * 1e-3)
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": K, "warmup": args.warmup,
        "ms_per_step": tot_mixed / K, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32+f64", "data": "synthetic (seeded Fourier-velocity divergence RHS on disk-refined AMR forests)",
        "config": {"workload": f"{args.workload}: bpdx={mesh.bpdx} bpdy={mesh.bpdy} levelMax={mesh.level_max}, "
                               f"{mesh.nblocks} blocks, {n} cells, explicit coarse/fine rows {R} ({nnz} nnz)",
                   "tol": "true |b-Ax|_inf / |b|_inf <= 1e-6, x0 = 0", "solver": "mixed (FP32 Krylov, FP64 x)",
                   "l2": "256 MiB written between steps (flush)", "parallelism": f"replicas x{world}"},
        "latency_ms": {"p50": pct(lat, 0.5), "p99": pct(lat, 0.99), "mean": statistics.mean(lat)},
        "iterations_mean": statistics.mean(it_m), "true_res_updates_mean": statistics.mean(up_m),
        "plain_fp64": {"value": world * K / (tot_fp64 * 1e-3), "unit": UNIT, "ms_per_step": tot_fp64 / K,
                       "latency_ms": {"p50": pct(latd, 0.5), "p99": pct(latd, 0.99)},
                       "iterations_mean": statistics.mean(it_d),
                       "roofline": {"bound": "hbm", "achieved": ach_d, "peak": peak, "unit": "GB/s",
                                    "frac": ach_d / peak, "traffic": traffic_d,
                                    "kernel": "k_bicgstab64 (one persistent launch per solve)"}},
        "speedup_mixed_vs_fp64": tot_fp64 / tot_mixed,
        "roofline": {"bound": "hbm", "achieved": ach_m, "peak": peak, "unit": "GB/s", "frac": ach_m / peak,
                     "traffic": traffic, "kernel": "k_bicgstab_mixed (one persistent launch per solve)",
                     "peak_kind": peak_kind},
        "e2e": {"value": world * K / e2e_s, "unit": UNIT, "h2d_bytes_per_step": 2 * 8 * n,
                "d2h_bytes_per_step": 8 * n},
        "gpu_launches": 2 * K,
        "clocks": clk.summary(),
        "status_ok": all(s["status"] == 0 for s in st_mixed + st_fp64),
    }
    if not args.no_cpu:
        line["cpu_baseline"] = cpu_baseline(mesh, bs[args.warmup].cpu().numpy(), statistics.mean(it_d))
    return line


def cpu_baseline(mesh, b, fp64_iters: float, sample_iters: int = 60) -> dict:
    """The oracle (C++/OpenMP restatement of the reference solve) on the host
    cores: a bounded sample of `sample_iters` BiCGSTAB iterations of the same
    solve, scaled to solves/s by the FP64 iteration count of the GPU run
    (same algorithm, same matrix and right-hand side)."""
    import oracle
    cores = oracle.num_threads()
    A = oracle.Matrix(mesh)
    t0 = time.perf_counter()
    A.bicgstab(b, tol_rel=0.0, max_iter=sample_iters, max_restarts=100)
    dt = time.perf_counter() - t0
    per_iter = dt / sample_iters
    return {"value": 1.0 / (per_iter * fp64_iters), "unit": UNIT, "cores": cores, "kind": "port",
            "sample": f"{sample_iters} BiCGSTAB iterations of the same FP64 solve in {dt:.2f} s "
                      f"(OpenMP, {cores} threads), scaled by {fp64_iters:.0f} iterations/solve"}


def run_reference(args, world, rank) -> dict | None:
    if rank != 0:
        return None
    import oracle
    from cup2d_b200.problems import large_mesh, small_mesh
    mesh = large_mesh() if args.workload == "large" else small_mesh()
    n = mesh.ncells
    cores = oracle.num_threads()
    A = oracle.Matrix(mesh)
    sample = 30
    seeds = [17 + s for s in range(args.warmup + args.steps)]
    # iterations the reference algorithm needs at this tolerance (one full
    # solve, untimed), then K bounded samples of `sample` iterations each
    b0 = mesh.rhs_fourier(seeds[args.warmup])
    _, st = A.bicgstab(b0, tol_rel=TOL, max_iter=20000, max_restarts=100)
    full_iters = st["iterations"]
    times = []
    for i, s in enumerate(seeds):
        b = mesh.rhs_fourier(s)
        t0 = time.perf_counter()
        A.bicgstab(b, tol_rel=0.0, max_iter=sample, max_restarts=100)
        dt = time.perf_counter() - t0
        if i >= args.warmup:
            times.append(dt)
    per_solve = statistics.mean(times) / sample * full_iters
    v = 1.0 / per_solve
    return {"metric": METRIC, "value": v, "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": per_solve * 1e3, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic", "impl": "reference",
            "config": {"workload": f"{args.workload}: {mesh.nblocks} blocks, {n} cells", "tol": "rel 1e-6"},
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": cores, "kind": "port",
                             "sample": f"per step {sample} BiCGSTAB iterations (OpenMP, {cores} threads), "
                                       f"scaled by {full_iters} iterations/solve at rel 1e-6"},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def profile_case(args) -> int:
    """Short solves for profilers: two FP64 and two mixed solves of the
    workload, each capped at `--profile-iters` iterations, one kernel launch
    each.  Prints the solve statistics; no timing is reported."""
    import torch

    from cup2d_b200 import Solver
    from cup2d_b200.problems import large_mesh, small_mesh
    dev = torch.device("cuda", 0)
    mesh = large_mesh() if args.workload == "large" else small_mesh()
    b = torch.from_numpy(mesh.rhs_fourier(17)).to(dev)
    it = args.profile_iters
    with Solver(mesh, tol_rel=0.0, max_iter=it) as s:
        for prec in ("fp64", "mixed"):
            s.set_opts(tol_rel=0.0, max_iter=it, precision=prec)
            for _ in range(2):
                x = torch.zeros(mesh.ncells, dtype=torch.float64, device=dev)
                print(prec, s.solve_device(b, x), flush=True)
            if args.phases:
                # one more solve with the device phase timers on
                s.set_profiling(True)
                x = torch.zeros(mesh.ncells, dtype=torch.float64, device=dev)
                st = s.solve_device(b, x)
                n = max(1, st["iterations"])
                print(f"{prec}: {st['solve_ms'] * 1e3 / n:.2f} us/iteration over {n} iterations", flush=True)
                for name, (c, w) in s.profile().items():
                    print(f"  {name:22s} compute {c * 1e3 / n:7.2f} us/it   barrier wait {w * 1e3 / n:7.2f} us/it")
                s.set_profiling(False)
    return 0


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=["large", "small"], default="large")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline sample")
    ap.add_argument("--profile-iters", type=int, default=0,
                    help="profiling case: capped solves only (see profile_case)")
    ap.add_argument("--phases", action="store_true", help="with --profile-iters: print device phase timers")
    args = ap.parse_args(argv)
    if args.profile_iters > 0:
        return profile_case(args)
    if args.warmup < 3:
        ap.error("--warmup must be >= 3")
    if args.impl == "reference":
        world = int(os.environ.get("WORLD_SIZE", "1"))
        rank = int(os.environ.get("RANK", "0"))
        line = run_reference(args, world, rank)
    else:
        world, rank, local = _dist()
        line = run_ours(args, world, rank, local)
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
    if line is not None:
        print(json.dumps(line), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
