"""Benchmark: Poisson solves/s and p50/p99 latency on one B200 (or N replicas).

Workload "batch" (default): 512 block-AMR pressure-Poisson problems, each a
forest refined near 1-3 seeded disks with levelMax 3..6 and a size drawn
log-uniform in 50..6000 blocks (38.3M cells in total), divergence-of-random-
Fourier-velocity right-hand sides, x0 = 0, each solved to relative true
L-inf residual 1e-6.  A step is one batched launch solving all of them.  The
headline `value` is batched mixed precision (FP32 Krylov vectors, FP64
solution and true residual); beside it the plain FP64 solver (the
reference's algorithm, one launch per problem) under "plain_fp64" and
batched FP64 under "batched_fp64".

Workload "large": one 20,834-block (1,333,376-cell) problem of bpdx=8,
bpdy=4, levelMax=7 refined near 3 seeded disks; a step is one solve.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                  [--workload batch|large|small]

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

# Hardware work queues per context.  CUDA's default of 8 maps the serving
# workload's 24 solve streams and 8 assembly streams onto 8 queues, where an
# assembly kernel can wait behind an unrelated persistent solve that shares
# its queue; 32 (the maximum) gives every stream its own.  Read when the
# CUDA context is created, so it is set before anything touches CUDA.
os.environ.setdefault("CUDA_DEVICE_MAX_CONNECTIONS", "32")

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
    """The largest of the ranks' values (times are max over ranks): one
    scalar all-reduce, on the device for NCCL, on the host for gloo."""
    if world == 1:
        return v
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([v], dtype=torch.float64, device=dev)
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

    FP64: 23 vector streams x 8 B per cell (A: R r,p,nu W p,z; B: R z,rhat
    W nu; C: R r,nu W s,z2; D: R z2,s W t; E: R x,z,z2,s,t,rhat W x,r).
    Mixed: the same streams with FP32 Krylov vectors and the FP64 solution x
    (read and written in pass E) = 100 B per cell; each true-residual refresh
    reads x, b (FP64) and rhat, writes r (FP32).  Matrix: 12 B per stored
    non-zero (FP64) or 8 B (FP32) + 4 B per stored row, and 28 B per block of
    structure (neighbours, row mask, row base)."""
    meta = 28.0 * nb
    if precision == "fp64":
        mat = 12.0 * nnz + 4.0 * R + meta
        per_iter = 23 * 8.0 * n + 2 * mat
        setup = (8 + 8 + 8 + 8) * n + mat   # r = b - A x0, rhat: R x,b W r,rhat
        final = 16.0 * n                     # mean removal: R x, W x
        return setup + iters * per_iter + final
    mat32 = 8.0 * nnz + 4.0 * R + meta
    mat64 = 12.0 * nnz + 4.0 * R + meta
    per_iter = 100.0 * n + 2 * mat32
    per_update = (8 + 8 + 4 + 4) * n + mat64
    setup = 8.0 * n + (8 + 8 + 4 + 4) * n + mat64   # sum b; true residual, rhat
    final = 16.0 * n
    return setup + iters * per_iter + updates * per_update + final


def spmv_leg(dev, stream, steps: int = 20, warmup: int = 5, forest: str = "full") -> dict:
    """The operator apply y = A x alone (the library's standalone SpMV, FP64
    and FP32) on one forest far above L2: bpdx=64, bpdy=32, levelMax=6, 3
    seeded disks, band 0.35 (1.15 M blocks, 73 M cells: 1.2 GB of x and y in
    FP64, so that launch and ramp-up are small against the transfer).  With
    forest="small" (profiling captures): bpdx=32, bpdy=16, the same disks and
    levels, band 0.15 (0.1 M blocks, 6.6 M cells: every kernel's traffic
    still twice L2 or more).
    Algorithmic bytes per launch:
    read x, write y, the explicit coarse/fine rows (values + column indices +
    row pointers) and 28 B of block structure per block."""
    import numpy as np
    import torch

    from cup2d_b200 import Mesh, Solver
    from cup2d_b200.problems import EXTENT, seeded_disks
    bpd, band = ((64, 32), 0.35) if forest == "full" else ((32, 16), 0.15)
    mesh = Mesh.disks(bpd[0], bpd[1], 6, EXTENT, seeded_disks(np.random.default_rng(5), 3), band)
    n = mesh.ncells
    out = {"mesh": f"bpdx={bpd[0]} bpdy={bpd[1]} levelMax=6, 3 disks, band {band}: {mesh.nblocks} blocks, {n} cells"}
    peak, kind = _peaks()
    with Solver(mesh) as h:
        R, nnz = h.explicit_info()
        for name, dt, vb, ab in (("fp64", torch.float64, 8, 12.0), ("fp32", torch.float32, 4, 8.0)):
            g = torch.Generator(device=dev).manual_seed(1)
            x = torch.randn(n, dtype=dt, device=dev, generator=g)
            y = torch.empty_like(x)
            ms = []
            for i in range(warmup + steps):
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                h.apply(x, y, stream=stream)
                e1.record(stream)
                torch.cuda.synchronize(dev)
                if i >= warmup:
                    ms.append(e0.elapsed_time(e1))
            by = 2.0 * vb * n + ab * nnz + 4.0 * R + 28.0 * mesh.nblocks
            t = statistics.median(ms)
            out[name] = {"kernel": "k_apply", "ms": t, "bytes": by, "achieved": by / (t * 1e-3) / 1e9, "peak": peak,
                         "unit": "GB/s", "frac": by / (t * 1e-3) / 1e9 / peak, "peak_kind": kind,
                         "l2": "x and y larger than L2" if 2 * vb * n > 126e6 else "x and y fit in L2"}
        # the mixed form's P^-1 apply alone, mma.sync (the solver's) and
        # tcgen05 (TMEM accumulators), on the same 73 M-cell vector: 8 B/cell
        g = torch.Generator(device=dev).manual_seed(2)
        p32 = torch.randn(n, dtype=torch.float32, device=dev, generator=g)
        z32 = torch.empty_like(p32)
        for name, tc in (("precond32_mma_sync", False), ("precond32_tcgen05", True)):
            ms = []
            for i in range(warmup + steps):
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                h.precond(p32, z32, stream=stream, tcgen05=tc)
                e1.record(stream)
                torch.cuda.synchronize(dev)
                if i >= warmup:
                    ms.append(e0.elapsed_time(e1))
            t = statistics.median(ms)
            by = 8.0 * n
            out[name] = {"kernel": "k_precond32_tc" if tc else "k_precond32", "ms": t, "bytes": by,
                         "achieved": by / (t * 1e-3) / 1e9, "peak": peak, "unit": "GB/s",
                         "frac": by / (t * 1e-3) / 1e9 / peak, "peak_kind": kind,
                         "flops_tensor_tflops": 3 * 2 * 64 * n / (t * 1e-3) / 1e12}
        del p32, z32, x, y
        # the pressure projection's field kernels on the same forest:
        # updatePressureRHS + updatePressureRHS1 (read vel, udef 16 B, chi,
        # pres 8 B; write tmp, pold 8 B; pres = 0 8 B) and pressureCorrection
        # (read pres 8 B, vel 16 B; write vel 16 B)
        g = torch.Generator(device=dev).manual_seed(3)
        vel = torch.randn(2 * n, dtype=torch.float64, device=dev, generator=g)
        udef = torch.randn(2 * n, dtype=torch.float64, device=dev, generator=g)
        chi = torch.rand(n, dtype=torch.float64, device=dev, generator=g)
        pres = torch.randn(n, dtype=torch.float64, device=dev, generator=g)
        pres0 = pres.clone()
        tmp = torch.empty_like(pres)
        pold = torch.empty_like(pres)
        for name, by in (("pressure_rhs", 64.0 * n), ("pressure_correction", 40.0 * n)):
            ms = []
            for i in range(warmup + steps):
                if name == "pressure_rhs":
                    pres.copy_(pres0)
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                if name == "pressure_rhs":
                    h.pressure_rhs(0.01, vel, udef, chi, pres, pold, tmp, stream=stream)
                else:
                    h.pressure_correction(0.01, pres0, vel, stream=stream)
                e1.record(stream)
                torch.cuda.synchronize(dev)
                if i >= warmup:
                    ms.append(e0.elapsed_time(e1))
            t = statistics.median(ms)
            out[name] = {"kernel": "k_" + name + (" + memset(pres)" if name == "pressure_rhs" else ""), "ms": t,
                         "bytes": by, "achieved": by / (t * 1e-3) / 1e9, "peak": peak, "unit": "GB/s",
                         "frac": by / (t * 1e-3) / 1e9 / peak, "peak_kind": kind}
    return out


def run_ours(args, world, rank, local) -> dict | None:
    """Single-problem workloads (large, small): a step is one solve."""
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
    if not args.no_cpu and world == 1:  # the host baseline: rank 0 at N=1 only
        line["cpu_baseline"] = cpu_baseline(mesh, seeds[args.warmup:args.warmup + 3])
    return line


def _pct(v, q):
    v = sorted(v)
    return v[min(len(v) - 1, int(round(q * (len(v) - 1))))]


CPU_SLICES = 64
CPU_SLICE_STRIDE = 41  # coprime with CPU_SLICES: consecutive slices sit far apart within the strata


def cpu_slices(meshes, parts: int = CPU_SLICES) -> list[list[int]]:
    """The batch cut into `parts` size-stratified slices: problems in size
    order, the j-th slice takes every parts-th one from position j, so every
    slice holds one problem of each stratum of `parts` consecutive sizes.
    Slices are returned in the order j = k * 41 mod parts, so that the first
    few (the ones a short run times) do not all hold the largest problem of
    each stratum; all parts slices together are the whole batch."""
    order = sorted(range(len(meshes)), key=lambda i: (-meshes[i].nblocks, i))
    return [order[(k * CPU_SLICE_STRIDE) % parts::parts] for k in range(parts)]


def time_cpu_solves(meshes, seeds, idx) -> tuple[float, list[dict]]:
    """Full solves on the host cores, timed: the oracle (C++/OpenMP
    restatement of ExpAMRSolver::solve with BiCGSTABSolver::main) solves each
    problem of `idx` from x0 = 0 to the batched workload's tolerance
    (|r|_inf <= 1e-6 |b|_inf; the iteration cap lifted so that every solve
    reaches it, as on the GPU) and removes the mean.  Operators are
    assembled before the clock starts, as the GPU arm's are."""
    import numpy as np

    import oracle
    mats = [oracle.Matrix(meshes[i]) for i in idx]
    bs = [meshes[i].rhs_fourier(seeds[i]) for i in idx]
    hs = [np.ascontiguousarray(meshes[i].cell_h()) for i in idx]
    P = oracle.pinv()
    sts = []
    t0 = time.perf_counter()
    for A, b, h in zip(mats, bs, hs):
        x, st = A.bicgstab(b, tol_rel=TOL, max_iter=20000, max_restarts=100, P=P)
        oracle.subtract_mean(h, x)
        sts.append(st)
    return time.perf_counter() - t0, sts


def batch_label(meshes, rank: int) -> str:
    """The batched workload's name, printed identically by both arms."""
    cells = sum(m.ncells for m in meshes)
    return (f"batch: {len(meshes)} problems, sizes log-uniform 50..6000 blocks "
            f"({min(m.nblocks for m in meshes)}..{max(m.nblocks for m in meshes)}), levelMax 3..6, 1-3 disks, "
            f"{cells} cells in total, mesh seed {3 + 1000 * rank}")


def batch_cpu_baseline(meshes, seeds, slices: int) -> dict:
    """The host baseline beside the GPU arm: full solves of `slices`
    size-stratified slices of the batch (about 15 s of CPU work)."""
    import oracle
    parts = cpu_slices(meshes)
    tot, solves, cit = 0.0, 0, 0
    for j in range(slices):
        dt, sts = time_cpu_solves(meshes, seeds, parts[j])
        tot += dt
        solves += len(sts)
        cit += sum(s["iterations"] * meshes[i].ncells for s, i in zip(sts, parts[j]))
    cores = oracle.num_threads()
    return {"value": solves / tot, "unit": UNIT, "cores": cores, "kind": "port",
            "sample": f"full solves of {solves} of the {len(meshes)} problems ({slices} size-stratified slices of "
                      f"1/{CPU_SLICES} of the batch), x0 = 0 to rel. 1e-6, OpenMP over {cores} threads, "
                      f"{tot:.1f} s timed ({tot / cit * 1e9:.2f} ns per cell-iteration)"}


def run_batch(args, world, rank, local) -> dict | None:
    """Batched workload: `--batch` uneven problems (sizes log-uniform in
    50..6000 blocks), each step one batched solve of all of them from x0 = 0.
    Headline: batched mixed precision.  Beside it: the plain FP64 solver one
    problem per launch (the reference's algorithm, the 3x target's base) and
    batched FP64."""
    import numpy as np
    import torch

    from cup2d_b200 import BatchSolver, Solver
    from cup2d_b200.problems import batch_problems

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    stream = torch.cuda.current_stream(dev)
    meshes = batch_problems(args.batch, seed=3 + 1000 * rank)
    n = len(meshes)
    seeds = [1000 * rank + 100 + i for i in range(n)]
    hb = [torch.from_numpy(m.rhs_fourier(s)).pin_memory() for m, s in zip(meshes, seeds)]
    bs = [b.to(dev) for b in hb]
    xs = [torch.zeros_like(b) for b in bs]
    cells = [m.ncells for m in meshes]
    opts = dict(tol_rel=TOL, max_iter=20000, max_restarts=100, timeout_ms=120000)
    B = BatchSolver(meshes, precision="mixed", team=args.team_mixed, **opts)

    def zero_x():
        for x in xs:
            x.zero_()

    def timed_batch(precision: str, team: int):
        """The launch shape is picked by the autotuner (unless --no-tune);
        each step replays a CUDA graph of one whole batched solve (x0 = 0
        written inside it) unless --no-graph.  CUDA events around each step
        on the launching stream; the working set is far above L2."""
        B.set_opts(precision=precision, **opts)
        B.set_team(team)
        B.set_occupancy(0)
        shape = {"team": team, "ctas_per_sm": 0, "tuned": False}
        if not args.no_tune:
            teams = [int(t) for t in args.tune_teams.split(",")]
            cps = [int(c) for c in args.tune_cps.split(",")]
            zero_x()
            t, c = B.autotune(bs, xs, teams=teams, ctas_per_sm=cps, iters=args.tune_iters)
            shape = {"team": t, "ctas_per_sm": c, "tuned": True, "tune_iters": args.tune_iters,
                     "rates_cell_it_per_s": {f"{k[0]}/{k[1]}": r for k, r in B.tune_rates.items()}}
        graph = not args.no_graph
        if graph:
            B.capture(bs, xs, zero_x=True)
        ms = []
        for i in range(args.warmup + args.steps):
            if not graph:
                zero_x()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            if graph:
                B.replay(stream)
            else:
                B.solve_device(bs, xs, stream=stream, stats=False)
            e1.record(stream)
            torch.cuda.synchronize(dev)
            if i >= args.warmup:
                ms.append(e0.elapsed_time(e1))
        if graph:
            B.replay(stream)
            st = B.replay_stats()
        else:
            zero_x()
            st = B.solve_device(bs, xs, stream=stream)
        begin, end, _ = B.timeline()
        shape["graph"] = graph
        return ms, st, end - begin, shape

    _barrier(world)
    with ClockSampler(local) as clk:
        ms_mx, st_mx, span_mx, shape_mx = timed_batch("mixed", args.team_mixed)
    if args.headline_only:
        # profiling runs: the headline leg alone (one batched launch per step)
        B.close()
        tot = _max_over_ranks(sum(ms_mx), world)
        if rank != 0:
            return None
        return {"metric": METRIC, "value": world * n * args.steps / (tot * 1e-3), "unit": UNIT, "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": tot / args.steps,
                "note": "headline leg only (profiling run)", "launch_shape": shape_mx,
                "cell_iterations_per_step": sum(s["iterations"] * c for s, c in zip(st_mx, cells))}
    ms_b64, st_b64, _, shape_64 = timed_batch("fp64", args.team_fp64)

    # plain FP64: one handle per problem, one persistent launch per solve
    hs = [Solver(m, precision="fp64", **opts) for m in meshes]
    ms_plain = []
    plain_steps = args.plain_steps if args.plain_steps > 0 else args.steps
    for i in range(args.warmup + plain_steps):
        zero_x()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for h, b, x in zip(hs, bs, xs):
            h.solve_device(b, x, stream=stream, stats=False)
        e1.record(stream)
        torch.cuda.synchronize(dev)
        if i >= args.warmup:
            ms_plain.append(e0.elapsed_time(e1))
    R_nnz = [h.explicit_info() for h in hs]
    # plain FP64 per-solve latency (one solve at a time, CUDA events)
    lat_plain = []
    for h, b, x in zip(hs, bs, xs):
        x.zero_()
        lat_plain.append(h.solve_device(b, x, stream=stream)["solve_ms"])
    for h in hs:
        h.close()

    # end to end through the public host-buffer API (pinned host memory)
    B.set_opts(precision="mixed", **opts)
    B.set_team(shape_mx["team"])
    B.set_occupancy(shape_mx["ctas_per_sm"])
    hx = [torch.zeros(c, dtype=torch.float64).pin_memory() for c in cells]
    hbn = [b.numpy() for b in hb]
    hxn = [x.numpy() for x in hx]
    _barrier(world)
    torch.cuda.synchronize(dev)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        for x in hxn:
            x[...] = 0.0
        B.solve(hbn, hxn)
    e2e_s = _max_over_ranks(time.perf_counter() - t0, world)
    B.close()
    spmv = spmv_leg(dev, stream) if not args.no_spmv else None

    K = args.steps
    tot_mx = _max_over_ranks(sum(ms_mx), world)
    tot_b64 = _max_over_ranks(sum(ms_b64), world)
    tot_plain = _max_over_ranks(sum(ms_plain), world)
    if rank != 0:
        return None
    peak, peak_kind = _peaks()
    by_mx = sum(algorithmic_bytes(m.ncells, m.nblocks, R, nnz, s["iterations"], s["refinements"], "mixed")
                for m, (R, nnz), s in zip(meshes, R_nnz, st_mx))
    by_64 = sum(algorithmic_bytes(m.ncells, m.nblocks, R, nnz, s["iterations"], 0, "fp64")
                for m, (R, nnz), s in zip(meshes, R_nnz, st_b64))
    ach_mx = by_mx / (statistics.mean(ms_mx) * 1e-3) / 1e9
    ach_64 = by_64 / (statistics.mean(ms_b64) * 1e-3) / 1e9
    cit_mx = sum(s["iterations"] * c for s, c in zip(st_mx, cells))
    cit_64 = sum(s["iterations"] * c for s, c in zip(st_b64, cells))
    traffic = None
    tp = ROOT / "profiles" / "traffic.json"
    if tp.exists():
        tj = json.loads(tp.read_text()).get("batch", {})
        if "dram_bytes_per_cell_iteration_mixed" in tj:
            traffic = tj["dram_bytes_per_cell_iteration_mixed"] * cit_mx
    plain_per_s = world * n * len(ms_plain) / (tot_plain * 1e-3)
    value = world * n * K / (tot_mx * 1e-3)
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": K, "warmup": args.warmup,
        "ms_per_step": tot_mx / K, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32+f64", "data": "synthetic (seeded Fourier-velocity divergence RHS on disk-refined AMR forests)",
        "config": {"workload": batch_label(meshes, rank),
                   "tol": "true |b-Ax|_inf / |b|_inf <= 1e-6, x0 = 0 (every problem)",
                   "solver": f"batched mixed (FP32 Krylov, FP64 x), team {shape_mx['team']} CTAs per problem, "
                             f"occupancy cap {shape_mx['ctas_per_sm'] or 'none'}",
                   "step": f"one launch solving all {n} problems" + (", replayed from a CUDA graph"
                                                                     if shape_mx["graph"] else ""),
                   "launch_shape": shape_mx,
                   "l2": "inputs larger than L2 (working set ~4 GB)", "parallelism": f"replicas x{world}"},
        "latency_ms": {"step_p50": _pct(ms_mx, 0.5), "step_p99": _pct(ms_mx, 0.99),
                       "problem_span_p50": float(np.percentile(span_mx, 50)),
                       "problem_span_p99": float(np.percentile(span_mx, 99))},
        "iterations_mean": statistics.mean(s["iterations"] for s in st_mx),
        "true_res_updates_mean": statistics.mean(s["refinements"] for s in st_mx),
        "plain_fp64": {"value": plain_per_s, "unit": UNIT, "ms_per_step": tot_plain / len(ms_plain),
                       "how": "one handle and one persistent launch per problem, problems back to back",
                       "latency_ms": {"p50": _pct(lat_plain, 0.5), "p99": _pct(lat_plain, 0.99)},
                       "iterations_mean": None},
        "batched_fp64": {"value": world * n * K / (tot_b64 * 1e-3), "unit": UNIT, "ms_per_step": tot_b64 / K,
                         "launch_shape": shape_64,
                         "iterations_mean": statistics.mean(s["iterations"] for s in st_b64),
                         "roofline": {"bound": "hbm", "achieved": ach_64, "peak": peak, "unit": "GB/s",
                                      "frac": ach_64 / peak, "kernel": "k_bicgstab_batch64"}},
        "speedup_batched_mixed_vs_plain_fp64": value / plain_per_s,
        "cell_iterations_per_step": {"mixed": cit_mx, "fp64": cit_64},
        "roofline": {"bound": "hbm", "achieved": ach_mx, "peak": peak, "unit": "GB/s", "frac": ach_mx / peak,
                     "traffic": traffic, "kernel": "k_bicgstab_batch_mixed (one launch per step)",
                     "peak_kind": peak_kind},
        "e2e": {"value": world * n * K / e2e_s, "unit": UNIT, "h2d_bytes_per_step": 2 * 8 * sum(cells),
                "d2h_bytes_per_step": 8 * sum(cells)},
        "spmv": spmv,
        "gpu_launches": K,
        "clocks": clk.summary(),
        "status_ok": all(s["status"] == 0 for s in st_mx + st_b64),
    }
    if not args.no_serve:
        line["serving"] = run_serve_sweep(args)
    if world == 1 and not args.no_configs:
        # the other configurations of the benchmark, measured in the same run
        line["large"] = large_leg(dev, stream)
        line["timestep"] = run_timestep(args)
    if not args.no_cpu and world == 1:  # the host baseline: rank 0 at N=1 only
        line["cpu_baseline"] = batch_cpu_baseline(meshes, seeds, args.cpu_slices)
    return line


def large_leg(dev, stream, solves: int = 2) -> dict:
    """The large configuration (bpdx=8, bpdy=4, levelMax=7, 3 seeded disks;
    20,834 blocks) solved from x0 = 0 to true |b-Ax|_inf <= tol |b|_inf, tol
    1e-6 (the served/batched tolerance) and 1e-8 (the configuration's), plain
    FP64 and mixed, without the reference's 1000-iteration cap: device time
    per solve (CUDA events, 256 MiB L2 flush between solves)."""
    import torch

    from cup2d_b200 import Solver
    from cup2d_b200.problems import large_mesh
    mesh = large_mesh()
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    bs = [torch.from_numpy(mesh.rhs_fourier(17 + k)).to(dev) for k in range(solves + 1)]
    x = torch.zeros(mesh.ncells, dtype=torch.float64, device=dev)
    out = {"mesh": f"{mesh.nblocks} blocks, {mesh.ncells} cells"}
    with Solver(mesh) as s:
        for tol in (1e-6, 1e-8):
            for prec in ("fp64", "mixed"):
                s.set_opts(tol_rel=tol, max_iter=20000, max_restarts=100, precision=prec)
                ms, its = [], []
                for k, b in enumerate(bs):
                    flush.fill_(float(k))
                    x.zero_()
                    # device time of the solve launch: the library's CUDA
                    # events around it on the launching stream
                    st = s.solve_device(b, x, stream=stream)
                    if k == 0:
                        continue  # warm-up
                    ms.append(st["solve_ms"])
                    its.append(st["iterations"])
                    if st["status"] != 0:
                        raise RuntimeError(f"large {prec} {tol}: status {st['status']}")
                out[f"{prec}_{tol:g}"] = {"solves_per_s": 1e3 / statistics.mean(ms), "ms": statistics.mean(ms),
                                          "iterations_mean": statistics.mean(its)}
    return out


def run_timestep(args) -> dict:
    """Time-stepping sequence: `--ts-steps` consecutive solves on the large
    forest (bpdx=8, bpdy=4, levelMax=7, 3 seeded disks) whose disks move
    0.002 per step along x; every 10 steps the forest is re-adapted on the
    device to the moved disks (tag, 2:1 balance, Morton order), re-assembled
    on the device and the pressure carried over by the device transfer.  The
    RHS comes from AR(1) Fourier coefficients (rho 0.95) through the device
    RHS kernel; each solve is warm-started from the previous pressure, to
    |b - Ax|_inf <= 1e-6 |b|_inf.  Run for the mixed and the plain FP64
    solver; wall-clock over the whole sequence (remeshes included) and
    CUDA-event solve times per step."""
    import numpy as np
    import torch

    from cup2d_b200 import Solver
    from cup2d_b200.mesh import fourier_advance, fourier_coefs
    from cup2d_b200.problems import large_mesh, seeded_disks

    dev = torch.device("cuda", 0)
    stream = torch.cuda.current_stream(dev)
    seed, every = 11, 10
    out = {}

    disks0 = seeded_disks(np.random.default_rng(1), 3)  # the disks of large_mesh(1)

    def sequence(precision: str, steps: int, warm: bool):
        opts = dict(tol_rel=0.0, max_iter=20000, max_restarts=100, timeout_ms=120000, precision=precision)
        mesh = large_mesh(1)
        cur, spare = Solver(mesh, **opts), Solver(mesh, **opts)
        coef = fourier_coefs(seed)
        x = torch.zeros(mesh.ncells, dtype=torch.float64, device=dev)
        b = torch.empty_like(x)
        its, solve_ms, remesh_ms, nblocks = [], [], [], []
        torch.cuda.synchronize(dev)
        t0 = time.perf_counter()
        for step in range(steps):
            if step > 0 and step % every == 0:
                tr = time.perf_counter()
                mesh = spare.adapt_disks([(cx + 0.002 * step, cy, r) for cx, cy, r in disks0], 0.12)
                x_new = torch.empty(mesh.ncells, dtype=torch.float64, device=dev)
                cur.transfer_to(spare, x, x_new, stream=stream)
                cur, spare, x = spare, cur, x_new
                b = torch.empty_like(x)
                torch.cuda.synchronize(dev)
                remesh_ms.append((time.perf_counter() - tr) * 1e3)
            coef = fourier_advance(coef, seed, step)
            cur.rhs_fourier_device(coef, b, stream=stream)
            cur.set_opts(tol_abs=TOL * float(b.abs().max()), **opts)
            if not warm:
                x.zero_()
            st = cur.solve_device(b, x, stream=stream)
            if st["status"] != 0:
                raise RuntimeError(f"step {step}: status {st['status']}")
            its.append(st["iterations"])
            solve_ms.append(st["solve_ms"])
            nblocks.append(mesh.nblocks)
        wall = time.perf_counter() - t0
        cur.close()
        spare.close()
        return {"solves_per_s": steps / wall, "steps": steps, "wall_s": wall,
                "solve_ms": {"p50": _pct(solve_ms, 0.5), "p99": _pct(solve_ms, 0.99),
                             "mean": statistics.mean(solve_ms)},
                "iterations_mean": statistics.mean(its),
                "remesh_ms_mean": statistics.mean(remesh_ms) if remesh_ms else None,
                "remeshes": len(remesh_ms), "blocks": [min(nblocks), max(nblocks)]}

    sequence("mixed", min(args.warmup, 5), True)  # warm-up: library, allocator, clocks
    with ClockSampler(0) as clk:
        for prec in ("mixed", "fp64"):
            out[prec] = sequence(prec, args.ts_steps, True)
        out["mixed_cold"] = sequence("mixed", min(args.ts_steps, 50), False)
    return {"metric": "time-stepping Poisson solves/s (warm start, remesh every 10 steps)",
            "value": out["mixed"]["solves_per_s"], "unit": UNIT, "n_gpus": 1, "steps": args.ts_steps,
            "warmup": min(args.warmup, 5), "higher_is_better": True, "dtype": "f32+f64",
            "config": {"workload": "timestep: large forest (bpdx=8 bpdy=4 levelMax=7, 3 seeded disks), disks "
                                   "move 0.002/step, every 10 steps forest adaptation + re-assembly + pressure "
                                   "transfer on the device, AR(1) rho=0.95 Fourier RHS on the device, warm start",
                       "tol": "|b - Ax|_inf <= 1e-6 |b|_inf per step"},
            "legs": out, "clocks": clk.summary(), "data": "synthetic"}


def run_serve_sweep(args) -> dict:
    """The serving workload at each offered rate of --serve-rates: served
    solves/s, p50/p99 latency per rate, and the saturation point (the
    highest served rate)."""
    rates = [float(r) for r in args.serve_rates.split(",") if r.strip()]
    legs = []
    for rate in rates:
        args.serve_rate = rate
        legs.append(run_serve(args))
    best = max(legs, key=lambda d: d["value"])
    return {"metric": "served Poisson solves/s (open-loop arrivals), offered-rate sweep", "unit": UNIT,
            "sweep": [{"offered_rate": d["offered_rate"], "served": d["value"], "latency_ms": d["latency_ms"],
                       "status_ok": d["status_ok"], "device_busy": d["device_busy"],
                       "assemblies": d["server"]["assemblies"], "assembly_ms_mean": d["assembly_ms_mean"]}
                      for d in legs],
            "saturation": {"served": best["value"], "at_offered_rate": best["offered_rate"]},
            "config": legs[0]["config"], "requests_per_rate": args.serve_requests}


def run_serve(args) -> dict:
    """Serving workload: open-loop Poisson arrivals at --serve-rate requests/s,
    mesh sizes log-uniform in 64..20000 blocks; 30% of the requests reuse a
    recently used (resident) mesh with a new right-hand side, the others
    bring a mesh the server has not seen (a new mesh id: assembled on
    admission).  Each request: x0 = 0, mixed precision to rel. 1e-6, team by
    mesh size.  Latency = submission to completion (the server's clock)."""
    import numpy as np
    import torch

    from cup2d_b200 import Server
    from cup2d_b200.problems import loguniform_sizes, sized_mesh
    rng = np.random.default_rng(7)
    pool = [sized_mesh(rng, int(n)) for n in loguniform_sizes(rng, args.serve_pool, 64, 20000)]
    rhs = [[torch.from_numpy(m.rhs_fourier(900 + k)).pin_memory().numpy() for k in range(3)] for m in pool]
    # pinned solution buffers, allocated before the clock starts (a
    # page-locked allocation serialises the device's streams)
    free_x: dict[int, list] = {i: [torch.zeros(m.ncells, dtype=torch.float64).pin_memory().numpy()
                                   for _ in range(args.serve_xbufs)] for i, m in enumerate(pool)}

    def take_x(i):
        if free_x[i]:
            x = free_x[i].pop()
            x[...] = 0.0
            return x
        return np.zeros(pool[i].ncells)  # pageable fallback when all are in use

    n = args.serve_requests
    gaps = rng.exponential(1.0 / args.serve_rate, size=n)
    kinds = rng.random(n) < 0.3          # True: reuse a resident mesh
    picks = rng.integers(len(pool), size=n)
    S = Server(max_inflight=args.serve_inflight, team=0, blocks_per_cta=args.serve_bpc,
               solve_share=args.serve_share, tol_rel=TOL,
               max_iter=20000, precision="mixed", timeout_ms=120000)
    recent: list[tuple[int, int]] = []   # (mesh id, pool index) of recently used meshes
    busy: dict[int, tuple] = {}          # request -> (pool index, x)
    lat, iters, statuses, solve_ms, blocks = [], [], [], [], []
    t0 = time.perf_counter()
    t_next = t0
    k = 0
    done_t = t0
    while k < n or busy:
        now = time.perf_counter()
        while k < n and now >= t_next:
            if kinds[k] and recent:
                mid, i = recent[int(rng.integers(len(recent)))]
            else:
                i = int(picks[k])
                mid = S.add_mesh(pool[i])
                recent.append((mid, i))
                recent[:] = recent[-16:]
            x = take_x(i)
            rid = S.submit(mid, rhs[i][k % 3], x)
            busy[rid] = (i, x)
            k += 1
            t_next += gaps[k - 1]
        wait_ms = 0 if k < n else 2
        for rid in S.take_completed(timeout_ms=wait_ms):
            st = S.poll(rid)
            i, x = busy.pop(rid)
            if isinstance(x, np.ndarray) and x.size == pool[i].ncells and len(free_x[i]) < args.serve_xbufs:
                free_x[i].append(x)
            solve_ms.append(st["solve_ms"])
            blocks.append(pool[i].nblocks)
            lat.append(st["latency_ms"])
            iters.append(st["iterations"])
            statuses.append(st["status"])
            done_t = time.perf_counter()
        if k < n:
            time.sleep(max(0.0, min(0.0005, t_next - time.perf_counter())))
    c = S.counters()
    S.close()
    span = done_t - t0
    return {"metric": "served Poisson solves/s (open-loop arrivals)", "value": n / span, "unit": UNIT,
            "offered_rate": args.serve_rate, "requests": n,
            "latency_ms": {"p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99)),
                           "mean": float(np.mean(lat))},
            "iterations_mean": float(np.mean(iters)), "status_ok": all(v == 0 for v in statuses),
            "device_busy": float(np.sum(solve_ms) / (span * 1e3)),  # mean solves running at once
            "solve_ms": {"p50": float(np.percentile(solve_ms, 50)), "max": float(np.max(solve_ms))},
            "blocks_mean": float(np.mean(blocks)),
            "config": f"sizes log-uniform 64..20000 blocks (pool of {len(pool)} forests), 30% reuse a resident "
                      f"mesh with a new RHS, 70% a new mesh id (assembled on admission); mixed, rel. 1e-6, "
                      f"x0 = 0; {args.serve_inflight} solve slots, team = blocks/{args.serve_bpc} (2..128)",
            "server": {k2: c[k2] for k2 in ("admitted", "completed", "failed", "assemblies", "evictions",
                                            "resident_meshes")},
            "assembly_ms_mean": c["assembly_us"] / 1e3 / max(1, c["assemblies"])}


def cpu_baseline(mesh, seeds) -> dict:
    """The oracle on the host cores for a one-problem workload: full solves of
    the same problem (x0 = 0 to rel. 1e-6, cap lifted), timed end to end."""
    import oracle
    A = oracle.Matrix(mesh)
    P = oracle.pinv()
    tot, its = 0.0, []
    for s_ in seeds:
        b = mesh.rhs_fourier(s_)
        t0 = time.perf_counter()
        x, st = A.bicgstab(b, tol_rel=TOL, max_iter=20000, max_restarts=100, P=P)
        oracle.subtract_mean(mesh.cell_h(), x)
        tot += time.perf_counter() - t0
        its.append(st["iterations"])
    cores = oracle.num_threads()
    return {"value": len(seeds) / tot, "unit": UNIT, "cores": cores, "kind": "port",
            "sample": f"{len(seeds)} full solves (x0 = 0 to rel. 1e-6, {statistics.mean(its):.0f} iterations on "
                      f"average), OpenMP over {cores} threads, {tot:.1f} s timed"}


def run_reference_batch(args) -> dict:
    """The reference algorithm on the host cores for the batched workload,
    timed in full: step k solves slice k mod 64 of the batch (one problem of
    each size stratum: the batch's size mix) with the oracle, every solve to
    the tolerance, inside the timed region; operators are assembled before
    the clock starts (as the GPU arm's are).  value = solves / time."""
    import oracle
    from cup2d_b200.problems import batch_problems
    meshes = batch_problems(args.batch, seed=3)
    seeds = [100 + i for i in range(len(meshes))]
    parts = cpu_slices(meshes)
    cores = oracle.num_threads()
    times, solves, cit = [], 0, 0
    for k in range(args.warmup + args.steps):
        idx = parts[k % len(parts)]
        dt, sts = time_cpu_solves(meshes, seeds, idx)
        if k >= args.warmup:
            times.append(dt)
            solves += len(sts)
            cit += sum(s["iterations"] * meshes[i].ncells for s, i in zip(sts, idx))
    tot = sum(times)
    v = solves / tot
    sample = (f"step k: full solves of slice k mod {len(parts)} of the batch ({len(parts[0])} problems, one of each "
              f"size stratum), x0 = 0 to rel. 1e-6, iteration cap lifted, OpenMP over {cores} threads; "
              f"{solves} solves in {tot:.1f} s timed ({tot / cit * 1e9:.2f} ns per cell-iteration)")
    return {"metric": METRIC, "value": v, "unit": UNIT, "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": tot / len(times) * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded Fourier-velocity divergence RHS on "
                                                         "disk-refined AMR forests)", "impl": "reference",
            "config": {"workload": batch_label(meshes, 0),
                       "tol": "true |b-Ax|_inf / |b|_inf <= 1e-6, x0 = 0 (every problem)"},
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": cores, "kind": "port", "sample": sample},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def run_reference_gpu_batch(args) -> dict:
    """The reference's own GPU path on the batched workload, for comparison
    (`--impl reference --ref-gpu`; the reference arm's line stays the CPU
    one): CUP2D's ExpAMRSolver::solve with its cuBLAS/cuSPARSE BiCGSTAB
    (source/Poisson/BiCGSTAB.cu:412-620), its Poisson sources compiled
    unchanged against one-rank stand-ins (oracle/_ref), one problem per call
    as CUP2D runs it, on the slices the CPU arm solves.  A call constructs
    the solver (P^-1, library handles, device buffers), assembles on the
    host (getMat), copies b and x in, solves with the reference's hard-coded
    1000-iteration cap and copies x back; wall clock per step.  The same
    calls with tol_rel = 1 (one iteration) measure the fixed part of a call,
    reported beside it ("per_call_fixed_ms", "solve_only")."""
    import oracle.ref as R
    from cup2d_b200.problems import batch_problems
    if not R.available("gpu"):
        return {"impl": "reference", "unavailable": "the reference GPU checker (oracle/_ref) is not built"}
    meshes = batch_problems(args.batch, seed=3)
    seeds = [100 + i for i in range(len(meshes))]
    parts = cpu_slices(meshes)
    times, fixed, its = [], [], []
    solves = capped = cells = 0
    for k in range(args.warmup + args.steps):
        idx = parts[k % len(parts)]
        bs = [meshes[i].rhs_fourier(seeds[i]) for i in idx]
        t0 = time.perf_counter()
        sts = [R.solve(meshes[i], b, tol_rel=TOL)[1] for i, b in zip(idx, bs)]
        dt = time.perf_counter() - t0
        t0 = time.perf_counter()
        for i, b in zip(idx, bs):
            R.solve(meshes[i], b, tol_rel=1.0)
        df = time.perf_counter() - t0
        if k >= args.warmup:
            times.append(dt)
            fixed.append(df)
            solves += len(idx)
            cells += sum(meshes[i].ncells for i in idx)
            capped += sum(1 for s in sts if not s["converged"])
            its += [s["iterations"] for s in sts if s["iterations"] is not None]
    tot, tfix = sum(times), sum(fixed)
    v = solves / tot
    sample = (f"step k: slice k mod {len(parts)} of the batch ({len(parts[0])} problems, one of each size stratum), "
              f"x0 = 0 to rel. 1e-6, one ExpAMRSolver per call (construction, host getMat, GPU BiCGSTAB with the "
              f"reference's 1000-iteration cap: {capped} of {solves} capped), {solves} solves in {tot:.1f} s")
    steps = len(times)
    return {"metric": METRIC, "value": v, "unit": UNIT, "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": tot / steps * 1e3, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic (seeded Fourier-velocity divergence RHS on disk-refined AMR forests)",
            "impl": "reference", "path": "reference GPU: ExpAMRSolver::solve, cuBLAS/cuSPARSE BiCGSTAB (oracle/_ref)",
            "config": {"workload": batch_label(meshes, 0),
                       "tol": "true |b-Ax|_inf / |b|_inf <= 1e-6, x0 = 0 (every problem)"},
            "iterations_mean": statistics.mean(its) if its else None, "capped": capped,
            "per_call_fixed_ms": tfix / solves * 1e3,
            "solve_only": {"value": solves / max(tot - tfix, 1e-9), "unit": UNIT,
                           "how": "steps' time less the same calls at tol_rel = 1"},
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": 1, "kind": "reference", "sample": sample},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": int(16 * cells / steps),
                    "d2h_bytes_per_step": int(8 * cells / steps)}}


def run_reference(args, world, rank) -> dict | None:
    if rank != 0:
        return None
    if args.workload == "batch" and getattr(args, "ref_gpu", False):
        return run_reference_gpu_batch(args)
    if args.workload == "batch":
        return run_reference_batch(args)
    import oracle
    from cup2d_b200.problems import large_mesh, small_mesh
    mesh = large_mesh() if args.workload == "large" else small_mesh()
    n = mesh.ncells
    cores = oracle.num_threads()
    A = oracle.Matrix(mesh)
    P = oracle.pinv()
    seeds = [17 + s for s in range(args.warmup + args.steps)]
    times, its = [], []
    for i, s_ in enumerate(seeds):
        b = mesh.rhs_fourier(s_)
        t0 = time.perf_counter()
        x, st = A.bicgstab(b, tol_rel=TOL, max_iter=20000, max_restarts=100, P=P)
        oracle.subtract_mean(mesh.cell_h(), x)
        dt = time.perf_counter() - t0
        if i >= args.warmup:
            times.append(dt)
            its.append(st["iterations"])
    v = len(times) / sum(times)
    return {"metric": METRIC, "value": v, "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": statistics.mean(times) * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic", "impl": "reference",
            "config": {"workload": f"{args.workload}: bpdx={mesh.bpdx} bpdy={mesh.bpdy} levelMax={mesh.level_max}, "
                                   f"{mesh.nblocks} blocks, {n} cells", "tol": "true |b-Ax|_inf / |b|_inf <= 1e-6, x0 = 0"},
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": cores, "kind": "port",
                             "sample": f"one full solve per step (x0 = 0 to rel. 1e-6, cap lifted, "
                                       f"{statistics.mean(its):.0f} iterations on average), OpenMP over {cores} threads"},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def profile_case(args) -> int:
    """Short solves for profilers: two FP64 and two mixed solves of the
    workload, each capped at `--profile-iters` iterations, one kernel launch
    each.  Prints the solve statistics; no timing is reported."""
    import torch
    if args.workload == "batch":
        return profile_batch(args)

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


def profile_batch(args) -> int:
    """Two FP64 and two mixed batched launches over the first `--batch`
    problems of the batched workload, each problem capped at
    `--profile-iters` iterations."""
    import torch

    from cup2d_b200 import BatchSolver
    from cup2d_b200.problems import batch_problems
    dev = torch.device("cuda", 0)
    meshes = batch_problems(args.batch, seed=3)
    bs = [torch.from_numpy(m.rhs_fourier(100 + i)).to(dev) for i, m in enumerate(meshes)]
    it = args.profile_iters
    with BatchSolver(meshes, tol_rel=0.0, max_iter=it) as B:
        for prec, team in (("fp64", args.team_fp64), ("mixed", args.team_mixed)):
            B.set_opts(tol_rel=0.0, max_iter=it, precision=prec)
            B.set_team(team)
            for _ in range(2):
                xs = [torch.zeros_like(b) for b in bs]
                st = B.solve_device(bs, xs)
                _, _, launch_ms = B.timeline()
                cit = sum(s["iterations"] * m.ncells for s, m in zip(st, meshes))
                print(f"{prec} team {team}: {launch_ms:.2f} ms, {cit} cell-iterations, "
                      f"{sum(m.ncells for m in meshes)} cells", flush=True)
        if args.phases:
            # one full batched solve per form (rel. 1e-6) with the device phase timers on
            for prec, team in (("fp64", args.team_fp64), ("mixed", args.team_mixed)):
                B.set_opts(tol_rel=TOL, max_iter=20000, precision=prec, timeout_ms=120000)
                B.set_team(team)
                B.set_profiling(True)
                xs = [torch.zeros_like(b) for b in bs]
                st = B.solve_device(bs, xs)
                _, _, launch_ms = B.timeline()
                prof = B.profile()
                B.set_profiling(False)
                cit = sum(s["iterations"] * m.ncells for s, m in zip(st, meshes))
                print(f"{prec} team {team}: launch {launch_ms:.1f} ms, {cit} cell-iterations; per CTA:", flush=True)
                for name, (c, w) in prof.items():
                    print(f"  {name:22s} compute {c:8.2f} ms   barrier wait {w:8.2f} ms", flush=True)
    return 0


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--ref-gpu", action="store_true",
                    help="with --impl reference, batch: time the reference's own GPU path (oracle/_ref) instead "
                         "of the CPU reference algorithm")
    ap.add_argument("--workload", choices=["batch", "large", "small", "serve", "timestep"], default="batch")
    ap.add_argument("--ts-steps", type=int, default=500, help="timestep workload: time steps per leg")
    ap.add_argument("--batch", type=int, default=512, help="batch workload: number of problems")
    ap.add_argument("--team-mixed", type=int, default=8, help="batch: CTAs per problem, mixed (with --no-tune)")
    ap.add_argument("--team-fp64", type=int, default=8, help="batch: CTAs per problem, FP64 (with --no-tune)")
    ap.add_argument("--no-tune", action="store_true", help="batch: fixed teams, no autotuner")
    ap.add_argument("--tune-iters", type=int, default=0,
                    help="batch autotuner: iterations per problem of a candidate (0 = full solves: a fixed "
                         "iteration count ignores the tail of the largest problems and favours small teams)")
    ap.add_argument("--tune-teams", default="5,6,8,12", help="batch autotuner: candidate teams")
    ap.add_argument("--tune-cps", default="0", help="batch autotuner: candidate CTAs per SM (0 = all)")
    ap.add_argument("--no-spmv", action="store_true", help="batch: skip the standalone SpMV leg")
    ap.add_argument("--spmv-only", action="store_true", help="the standalone SpMV leg alone (profiling runs)")
    ap.add_argument("--no-graph", action="store_true", help="batch: launch directly instead of graph replays")
    ap.add_argument("--spmv-forest", choices=["full", "small"], default="full",
                    help="with --spmv-only: the forest of the standalone kernel leg (small: for profiling)")
    ap.add_argument("--plain-steps", type=int, default=0,
                    help="batch: timed steps of the one-at-a-time FP64 leg (0 = --steps)")
    ap.add_argument("--cpu-slices", type=int, default=4,
                    help="batch CPU baseline: size-stratified slices (1/64 of the batch each) solved in full")
    ap.add_argument("--no-serve", action="store_true", help="batch: skip the serving leg")
    ap.add_argument("--no-configs", action="store_true",
                    help="batch: skip the large and time-stepping legs that follow the headline")
    ap.add_argument("--serve-rate", type=float, default=100.0, help="serving: offered requests/s (--workload serve)")
    ap.add_argument("--serve-rates", default="100,300,1000",
                    help="batch workload's serving leg: offered rates of the sweep (requests/s)")
    ap.add_argument("--serve-requests", type=int, default=300, help="serving: requests")
    ap.add_argument("--serve-pool", type=int, default=40, help="serving: distinct forests")
    ap.add_argument("--serve-inflight", type=int, default=24, help="serving: solve slots")
    ap.add_argument("--serve-share", type=float, default=0.9, help="serving: share of solve CTAs in use")
    ap.add_argument("--serve-bpc", type=int, default=320, help="serving: blocks per CTA of a solve's team")
    ap.add_argument("--serve-xbufs", type=int, default=12, help="serving: pinned solution buffers per forest")
    ap.add_argument("--headline-only", action="store_true",
                    help="batch: time the batched mixed leg only (for profilers; no comparison legs)")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline sample")
    ap.add_argument("--profile-iters", type=int, default=0,
                    help="profiling case: capped solves only (see profile_case)")
    ap.add_argument("--phases", action="store_true", help="with --profile-iters: print device phase timers")
    args = ap.parse_args(argv)
    if args.profile_iters > 0:
        return profile_case(args)
    if args.spmv_only:
        import torch
        dev = torch.device("cuda", 0)
        torch.cuda.set_device(dev)
        print(json.dumps(spmv_leg(dev, torch.cuda.current_stream(dev), steps=args.steps, warmup=args.warmup,
                                  forest=args.spmv_forest)))
        return 0
    if args.warmup < 3:
        ap.error("--warmup must be >= 3")
    if args.impl == "reference":
        world = int(os.environ.get("WORLD_SIZE", "1"))
        rank = int(os.environ.get("RANK", "0"))
        line = run_reference(args, world, rank)
    else:
        world, rank, local = _dist()
        if args.workload in ("serve", "timestep"):
            import torch
            torch.cuda.set_device(local)
            line = (run_serve if args.workload == "serve" else run_timestep)(args) if rank == 0 else None
        else:
            line = (run_batch if args.workload == "batch" else run_ours)(args, world, rank, local)
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
    if line is not None:
        print(json.dumps(line), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
