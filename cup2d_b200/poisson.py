"""Python mirror of CUP2D's Poisson-solver interface on the B200 C ABI.

Reference interface (paths in the CUP2D tree):
  class PoissonSolver { virtual void solve(const ScalarGrid* input,
                                           ScalarGrid* output) = 0; }   source/Poisson/Base.h:8-13
  makePoissonSolver(SimulationData&)                                    source/Poisson/Base.cpp:8-30
  libcubismup2d.poisson.Solver.solve(input, output)                     source/Bindings/Poisson.cpp:10-11
  ExpAMRSolver::solve (tolerances, re-assembly, mean removal)           source/Poisson/ExpAMRSolver.cpp:354-416

`ScalarGrid` here is a mesh plus one value per cell, (nblocks, 8, 8) in
block order (numpy on the host, or a CUDA tensor).  `Solver` is the handle
level API: solves on host arrays or device tensors, plus the building
blocks (operator apply, preconditioner, assembled CSR) used by the tests.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field
from typing import Optional

import numpy as np

from . import _lib as L
from .mesh import Mesh


def _pd(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def default_opts() -> L.SolveOpts:
    o = L.SolveOpts()
    L.lib().cup2d_default_opts(C.byref(o))
    return o


def make_opts(tol_abs=0.0, tol_rel=1e-8, max_restarts=100, max_iter=1000, precision="fp64",
              subtract_mean=True, reliable_delta=0.5, reliable_restart=True, timeout_ms=20000,
              mean_constraint=0) -> L.SolveOpts:
    o = default_opts()
    o.tol_abs = tol_abs
    o.tol_rel = tol_rel
    o.max_restarts = max_restarts
    o.max_iter = max_iter
    o.precision = {"fp64": L.PREC_FP64, "mixed": L.PREC_MIXED}[precision] if isinstance(precision, str) \
        else int(precision)
    o.subtract_mean = int(bool(subtract_mean))
    o.reliable_delta = reliable_delta
    o.reliable_restart = int(bool(reliable_restart))
    o.timeout_ms = timeout_ms
    o.mean_constraint = int(mean_constraint)
    return o


class Solver:
    """One solver handle: P^-1 and the assembled operator resident on the GPU."""

    def __init__(self, mesh: Mesh, opts: Optional[L.SolveOpts] = None, **kw):
        self.mesh = mesh
        self.opts = opts if opts is not None else make_opts(**kw)
        self._h = C.c_void_p()
        f = mesh.forest()
        L.check(L.lib().cup2d_poisson_create(C.byref(f), C.byref(self.opts), C.byref(self._h)),
                "cup2d_poisson_create")
        self.last_stats: Optional[dict] = None

    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            L.lib().cup2d_poisson_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    @property
    def ncells(self) -> int:
        return int(L.lib().cup2d_poisson_num_cells(self._h))

    def update_mesh(self, mesh: Mesh) -> None:
        self.mesh = mesh
        f = mesh.forest()
        L.check(L.lib().cup2d_poisson_update_mesh(self._h, C.byref(f)), "cup2d_poisson_update_mesh")

    def adapt_disks(self, disks, band: float) -> Mesh:
        """Re-adapts the forest on the device to the disk geometry (refined
        to the finest level within `band` of each disk, 2:1 balanced, Morton
        order: the forest Mesh.disks builds on the host for this handle's
        root grid, levels, extent and periodicity) and re-assembles the
        operator.  Returns the new forest (read back from the device)."""
        d = np.ascontiguousarray(np.asarray(disks, dtype=np.float64).reshape(-1, 3))
        nb = C.c_int64()
        L.check(L.lib().cup2d_poisson_adapt_disks(self._h, d.shape[0], _pd(d), float(band), C.byref(nb)),
                "cup2d_poisson_adapt_disks")
        self.mesh = self.device_forest()
        return self.mesh

    def device_forest(self) -> Mesh:
        """The handle's current forest, read back from the device."""
        nb = self.ncells // 64
        lv, bx, by = (np.empty(nb, dtype=np.int32) for _ in range(3))
        p = lambda a: a.ctypes.data_as(C.POINTER(C.c_int32))  # noqa: E731
        L.check(L.lib().cup2d_poisson_get_forest(self._h, p(lv), p(bx), p(by)), "cup2d_poisson_get_forest")
        m = self.mesh
        return Mesh(m.bpdx, m.bpdy, m.level_max, m.extent, lv, bx, by, m.periodic_x, m.periodic_y)

    def set_opts(self, opts: Optional[L.SolveOpts] = None, **kw) -> None:
        self.opts = opts if opts is not None else make_opts(**kw)
        L.check(L.lib().cup2d_poisson_set_opts(self._h, C.byref(self.opts)), "cup2d_poisson_set_opts")

    def set_grid(self, grid: int) -> None:
        L.check(L.lib().cup2d_poisson_set_grid(self._h, int(grid)), "cup2d_poisson_set_grid")

    # ------------------------------------------------------------ solve ---
    def solve(self, b: np.ndarray, x0: Optional[np.ndarray] = None, out: Optional[np.ndarray] = None) -> np.ndarray:
        """Host arrays in, host array out (the host<->device copies are part
        of the call).  With `out` (contiguous float64, e.g. pinned memory) the
        initial guess is read from and the solution written to that array."""
        b = np.ascontiguousarray(b, dtype=np.float64)
        if out is not None:
            if out.dtype != np.float64 or not out.flags.c_contiguous or out.shape != b.shape:
                raise ValueError("out must be a contiguous float64 array shaped like b")
            x = out
            if x0 is not None:
                x[...] = x0
        else:
            x = np.zeros_like(b) if x0 is None else np.array(x0, dtype=np.float64, copy=True)
        st = L.SolveStats()
        L.check(L.lib().cup2d_poisson_solve(self._h, _pd(b), _pd(x), C.byref(st)), "cup2d_poisson_solve")
        self.last_stats = st.as_dict()
        return x

    def solve_device(self, b, x, stream=None, stats: bool = True) -> Optional[dict]:
        """Device tensors (torch, float64, contiguous): x holds x0 and receives
        the solution.  With stats=False the call is asynchronous."""
        _check_dev(b, self.ncells, F64)
        _check_dev(x, self.ncells, F64)
        st = L.SolveStats()
        s = _stream_handle(stream)
        L.check(L.lib().cup2d_poisson_solve_device(self._h, C.c_void_p(b.data_ptr()), C.c_void_p(x.data_ptr()),
                                                   C.byref(st) if stats else None, s),
                "cup2d_poisson_solve_device")
        if stats:
            self.last_stats = st.as_dict()
            return self.last_stats
        return None

    def pressure_step(self, tmp, pres, pold, stream=None) -> dict:
        """PressureSingle's step around the solve on device tensors:
        pold = pres; tmp -= L(pold); pres = solve(tmp); pres += pold - mean.
        Returns the solve's statistics (the call synchronises)."""
        for t in (tmp, pres, pold):
            _check_dev(t, self.ncells, F64)
        st = L.SolveStats()
        L.check(L.lib().cup2d_poisson_pressure_step(self._h, C.c_void_p(tmp.data_ptr()), C.c_void_p(pres.data_ptr()),
                                                     C.c_void_p(pold.data_ptr()), C.byref(st),
                                                     _stream_handle(stream)),
                "cup2d_poisson_pressure_step")
        self.last_stats = st.as_dict()
        return self.last_stats

    def pressure_rhs(self, dt: float, vel=None, udef=None, chi=None, pres=None, pold=None, tmp=None,
                     stream=None) -> None:
        """What PressureSingle::operator() does before the solve, on device
        tensors (float64, block-major cells; vel and udef (ncells, 2)):
        with vel: tmp = updatePressureRHS(vel, udef, chi) at time step dt;
        with pres: pold = pres, tmp -= updatePressureRHS1(pold), pres = 0.
        Asynchronous on `stream`."""
        n = self.ncells
        if vel is not None:
            for t, k in ((vel, 2 * n), (udef, 2 * n), (chi, n)):
                _check_dev(t, k, F64)
        if pres is not None:
            _check_dev(pres, n, F64)
            _check_dev(pold, n, F64)
        _check_dev(tmp, n, F64)
        ptr = lambda t: None if t is None else C.c_void_p(t.data_ptr())  # noqa: E731
        L.check(L.lib().cup2d_poisson_pressure_rhs(self._h, float(dt), ptr(vel), ptr(udef), ptr(chi), ptr(pres),
                                                    ptr(pold), ptr(tmp), _stream_handle(stream)),
                "cup2d_poisson_pressure_rhs")

    def pressure_correction(self, dt: float, pres, vel, stream=None) -> None:
        """PressureSingle::pressureCorrection: vel += -0.5 dt h grad(pres) / h^2
        (central differences, flux-corrected), in place.  Asynchronous."""
        _check_dev(pres, self.ncells, F64)
        _check_dev(vel, 2 * self.ncells, F64)
        L.check(L.lib().cup2d_poisson_pressure_correction(self._h, float(dt), C.c_void_p(pres.data_ptr()),
                                                           C.c_void_p(vel.data_ptr()), _stream_handle(stream)),
                "cup2d_poisson_pressure_correction")

    def pressure_projection(self, dt: float, vel, udef, chi, pres, pold, tmp, stream=None) -> dict:
        """The pressure projection of PressureSingle::operator() without the
        obstacle terms: RHS, solve, pres += pold - mean, velocity correction.
        Returns the solve's statistics (the call synchronises)."""
        n = self.ncells
        for t, k in ((vel, 2 * n), (udef, 2 * n), (chi, n), (pres, n), (pold, n), (tmp, n)):
            _check_dev(t, k, F64)
        st = L.SolveStats()
        p = lambda t: C.c_void_p(t.data_ptr())  # noqa: E731
        L.check(L.lib().cup2d_poisson_pressure_projection(self._h, float(dt), p(vel), p(udef), p(chi), p(pres),
                                                           p(pold), p(tmp), C.byref(st), _stream_handle(stream)),
                "cup2d_poisson_pressure_projection")
        self.last_stats = st.as_dict()
        return self.last_stats

    def solve_device_noalloc(self, b, x, stream=None) -> dict:
        """The FP64 device solve without any device allocation, for callers
        that must not allocate at solve time (their device memory belongs to
        their own pool, or their loop cannot afford the synchronisation an
        allocation can cause).  Scratch lives in one static 16.2 MiB device
        array shared by all calls: at most CUP2D_NOALLOC_MAX_BLOCKS (4096)
        blocks, and calls that overlap on the GPU race."""
        _check_dev(b, self.ncells, F64)
        _check_dev(x, self.ncells, F64)
        st = L.SolveStats()
        L.check(L.lib().cup2d_poisson_solve_device_noalloc(self._h, C.c_void_p(b.data_ptr()),
                                                           C.c_void_p(x.data_ptr()), C.byref(st),
                                                           _stream_handle(stream)),
                "cup2d_poisson_solve_device_noalloc")
        self.last_stats = st.as_dict()
        return self.last_stats

    # ------------------------------------------------------ components ---
    def apply(self, x, y, stream=None) -> None:
        """y = A x on device tensors: float64, or float32 (the mixed form's SpMV)."""
        _check_dev(x, self.ncells)
        _check_dev(y, self.ncells, str(x.dtype))
        if str(x.dtype) not in ("torch.float32", F64):
            raise ValueError(f"expected float32 or float64 tensors, got {x.dtype}")
        s = _stream_handle(stream)
        fn = L.lib().cup2d_poisson_apply32 if str(x.dtype) == "torch.float32" else L.lib().cup2d_poisson_apply
        L.check(fn(self._h, C.c_void_p(x.data_ptr()), C.c_void_p(y.data_ptr()), s), "cup2d_poisson_apply")

    def rhs_fourier_device(self, coef: np.ndarray, b, kmax: int = 8, stream=None) -> None:
        """b (float64 CUDA tensor) = the zero-sum synthetic RHS of this
        forest for Fourier coefficients `coef` (Mesh.rhs_from_coefs on the
        device)."""
        coef = np.ascontiguousarray(coef, dtype=np.float64)
        _check_dev(b, self.ncells, F64)
        L.check(L.lib().cup2d_poisson_rhs_fourier_device(self._h, int(kmax), _pd(coef), C.c_void_p(b.data_ptr()),
                                                         _stream_handle(stream)), "cup2d_poisson_rhs_fourier_device")

    def transfer_to(self, dst: "Solver", x_src, x_dst, stream=None) -> None:
        """x_dst (on dst's forest) = x_src (on this forest), e.g. a warm
        start carried across a mesh adaptation."""
        _check_dev(x_src, self.ncells, F64)
        _check_dev(x_dst, dst.ncells, F64)
        L.check(L.lib().cup2d_poisson_transfer(self._h, C.c_void_p(x_src.data_ptr()), dst._h,
                                               C.c_void_p(x_dst.data_ptr()), _stream_handle(stream)),
                "cup2d_poisson_transfer")

    def precond(self, p, z, stream=None, tcgen05: bool = False) -> None:
        """z = P^-1 p per block: FP64, or FP32 (split TF32) on float32 tensors;
        tcgen05=True takes the FP32 apply on the tcgen05 tensor cores (TMEM
        accumulators) instead of mma.sync."""
        if tcgen05:
            fn = L.lib().cup2d_poisson_precond32_tc
        else:
            fn = L.lib().cup2d_poisson_precond32 if str(p.dtype) == "torch.float32" else L.lib().cup2d_poisson_precond
        s = _stream_handle(stream)
        L.check(fn(self._h, C.c_void_p(p.data_ptr()), C.c_void_p(z.data_ptr()), s), "cup2d_poisson_precond")

    def export_csr(self):
        n = C.c_int64()
        nnz = C.c_int64()
        L.check(L.lib().cup2d_poisson_export_csr(self._h, C.byref(n), C.byref(nnz), None, None, None),
                "cup2d_poisson_export_csr")
        rp = np.empty(n.value + 1, dtype=np.int64)
        col = np.empty(nnz.value, dtype=np.int32)
        val = np.empty(nnz.value, dtype=np.float64)
        L.check(L.lib().cup2d_poisson_export_csr(self._h, C.byref(n), C.byref(nnz),
                                                 rp.ctypes.data_as(C.POINTER(C.c_int64)),
                                                 col.ctypes.data_as(C.POINTER(C.c_int32)), _pd(val)),
                "cup2d_poisson_export_csr")
        return rp, col, val

    PHASES = ("residual/init", "A: p, P^-1", "B: SpMV (rhat,nu)", "C: s, P^-1", "D: SpMV (t,s),(t,t)",
              "E: x, r, norms", "true residual", "mean removal", "sum b", "next problem")

    def set_profiling(self, enable: bool = True) -> None:
        L.check(L.lib().cup2d_poisson_set_profiling(self._h, int(bool(enable))), "set_profiling")

    def profile(self) -> dict:
        """Per-phase (compute ms, barrier-wait ms), per-CTA averages since
        profiling was enabled."""
        c = np.zeros(10)
        w = np.zeros(10)
        L.check(L.lib().cup2d_poisson_profile(self._h, _pd(c), _pd(w), 10), "profile")
        return {name: (float(c[i]), float(w[i])) for i, name in enumerate(self.PHASES) if c[i] or w[i]}

    def explicit_info(self) -> tuple[int, int]:
        r = C.c_int64()
        z = C.c_int64()
        L.check(L.lib().cup2d_poisson_explicit_info(self._h, C.byref(r), C.byref(z)), "explicit_info")
        return r.value, z.value


def tune_key(device_name: str, precision: int, nblocks, teams, ctas_per_sm) -> str:
    """Cache key of an autotuner choice: the GPU, the precision, the batch
    size, its size quantiles (10/50/90/100 %) and the candidate lists."""
    sizes = np.sort(np.asarray(nblocks, dtype=np.int64))
    q = ",".join(str(int(sizes[int(f * (len(sizes) - 1))])) for f in (0.1, 0.5, 0.9, 1.0))
    return "|".join([device_name, "mixed" if precision == L.PREC_MIXED else "fp64", f"n={len(sizes)}", "q=" + q,
                     "teams=" + ",".join(map(str, teams)), "cps=" + ",".join(map(str, ctas_per_sm))])


class BatchSolver:
    """Many independent problems in one persistent launch (no counterpart in
    the reference, which solves one problem per PoissonSolver::solve call;
    each problem here gets exactly that solve)."""

    def __init__(self, meshes: list[Mesh], opts: Optional[L.SolveOpts] = None, team: Optional[int] = None, **kw):
        self.meshes = list(meshes)
        self.opts = opts if opts is not None else make_opts(**kw)
        n = len(self.meshes)
        forests = (L.Forest * n)(*[m.forest() for m in self.meshes])
        self._h = C.c_void_p()
        L.check(L.lib().cup2d_batch_create(n, forests, C.byref(self.opts), C.byref(self._h)), "cup2d_batch_create")
        if team is not None:
            self.set_team(team)
        self.last_stats: Optional[list[dict]] = None

    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            L.lib().cup2d_batch_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __len__(self) -> int:
        return int(L.lib().cup2d_batch_size(self._h))

    def ncells(self, i: int) -> int:
        return int(L.lib().cup2d_batch_num_cells(self._h, int(i)))

    def set_opts(self, opts: Optional[L.SolveOpts] = None, **kw) -> None:
        self.opts = opts if opts is not None else make_opts(**kw)
        L.check(L.lib().cup2d_batch_set_opts(self._h, C.byref(self.opts)), "cup2d_batch_set_opts")

    def set_team(self, team: int) -> None:
        L.check(L.lib().cup2d_batch_set_team(self._h, int(team)), "cup2d_batch_set_team")

    def solve_device(self, bs, xs, stream=None, stats: bool = True) -> Optional[list[dict]]:
        """bs[i], xs[i]: contiguous float64 CUDA tensors of problem i; xs hold
        the initial guesses and receive the solutions."""
        n = len(self)
        if len(bs) != n or len(xs) != n:
            raise ValueError(f"expected {n} right-hand sides and solutions")
        for i in range(n):
            _check_dev(bs[i], self.ncells(i), F64)
            _check_dev(xs[i], self.ncells(i), F64)
        pb = (C.c_void_p * n)(*[t.data_ptr() for t in bs])
        px = (C.c_void_p * n)(*[t.data_ptr() for t in xs])
        st = (L.SolveStats * n)()
        L.check(L.lib().cup2d_batch_solve_device(self._h, pb, px, st if stats else None, _stream_handle(stream)),
                "cup2d_batch_solve_device")
        if stats:
            self.last_stats = [s.as_dict() for s in st]
            return self.last_stats
        return None

    def set_occupancy(self, ctas_per_sm: int) -> None:
        """CTAs per SM of batched launches (0 = as many as fit)."""
        L.check(L.lib().cup2d_batch_set_occupancy(self._h, int(ctas_per_sm)), "cup2d_batch_set_occupancy")

    def autotune(self, bs, xs, teams=(5, 6, 8, 12), ctas_per_sm=(0,), iters: int = 0,
                 cache: Optional[str] = None) -> tuple[int, int]:
        """Picks the launch shape for this batch -- team size (CTAs per
        problem) and occupancy cap (CTAs per SM, 0 = all that fit): every
        candidate pair runs a batched launch -- full solves from xs with
        iters = 0 (the default: the schedule's tail, set by the largest
        problems, is part of the cost), or each problem capped at `iters`
        iterations -- and the fastest in cell-iterations/s is kept and
        returned as (team, ctas_per_sm).  With `cache` (a JSON file) a choice
        made before for the same GPU, precision and size distribution is
        reused without timing.  xs are overwritten when timing runs."""
        import json
        import os

        import torch
        key = tune_key(torch.cuda.get_device_name(), self.opts.precision,
                       [self.ncells(i) // 64 for i in range(len(self))], teams, ctas_per_sm)
        table = {}
        if cache and os.path.exists(cache):
            with open(cache) as f:
                table = json.load(f)
            if key in table:
                team, cps = int(table[key]["team"]), int(table[key]["ctas_per_sm"])
                self.set_team(team)
                self.set_occupancy(cps)
                return team, cps
        n = len(self)
        for i in range(n):
            _check_dev(bs[i], self.ncells(i), F64)
            _check_dev(xs[i], self.ncells(i), F64)
        pb = (C.c_void_p * n)(*[t.data_ptr() for t in bs])
        px = (C.c_void_p * n)(*[t.data_ptr() for t in xs])
        ct = (C.c_int32 * len(teams))(*teams)
        cc = (C.c_int32 * max(1, len(ctas_per_sm)))(*ctas_per_sm)
        rates = (C.c_double * (len(teams) * max(1, len(ctas_per_sm))))()
        best, best_cps = C.c_int32(), C.c_int32()
        L.check(L.lib().cup2d_batch_tune(self._h, pb, px, ct, len(teams), cc, len(ctas_per_sm), int(iters), rates,
                                         C.byref(best), C.byref(best_cps)), "cup2d_batch_tune")
        nc = max(1, len(ctas_per_sm))
        cps_list = list(ctas_per_sm) if ctas_per_sm else [0]
        self.tune_rates = {(t, cps_list[c]): rates[k * nc + c] for k, t in enumerate(teams) for c in range(nc)}
        if cache:
            table[key] = {"team": best.value, "ctas_per_sm": best_cps.value,
                          "rates": {f"{t}/{c}": r for (t, c), r in self.tune_rates.items()}}
            os.makedirs(os.path.dirname(os.path.abspath(cache)), exist_ok=True)
            with open(cache, "w") as f:
                json.dump(table, f, indent=1)
        return best.value, best_cps.value

    def capture(self, bs, xs, zero_x: bool = False) -> None:
        """Records one whole batched solve of these device tensors as a CUDA
        graph (options, team and occupancy as now); `replay` then re-runs it
        on whatever bs/xs hold, with xs warm from the previous replay unless
        zero_x.  The tensors are kept alive while the graph exists."""
        n = len(self)
        if len(bs) != n or len(xs) != n:
            raise ValueError(f"expected {n} right-hand sides and solutions")
        for i in range(n):
            _check_dev(bs[i], self.ncells(i), F64)
            _check_dev(xs[i], self.ncells(i), F64)
        pb = (C.c_void_p * n)(*[t.data_ptr() for t in bs])
        px = (C.c_void_p * n)(*[t.data_ptr() for t in xs])
        L.check(L.lib().cup2d_batch_capture(self._h, pb, px, L.GRAPH_ZERO_X if zero_x else 0), "cup2d_batch_capture")
        self._graph_io = (list(bs), list(xs))

    def replay(self, stream=None) -> None:
        L.check(L.lib().cup2d_batch_replay(self._h, _stream_handle(stream)), "cup2d_batch_replay")

    def replay_stats(self) -> list[dict]:
        st = (L.SolveStats * len(self))()
        L.check(L.lib().cup2d_batch_replay_stats(self._h, st), "cup2d_batch_replay_stats")
        self.last_stats = [s.as_dict() for s in st]
        return self.last_stats

    def solve(self, bs, xs) -> list[dict]:
        """Host arrays (contiguous float64, e.g. pinned): xs[i] holds the
        initial guess and receives the solution; the copies are part of the
        call."""
        n = len(self)
        if len(bs) != n or len(xs) != n:
            raise ValueError(f"expected {n} right-hand sides and solutions")
        for i in range(n):
            for a in (bs[i], xs[i]):
                if a.dtype != np.float64 or not a.flags.c_contiguous or a.size != self.ncells(i):
                    raise ValueError(f"problem {i}: expected contiguous float64 arrays of {self.ncells(i)} cells")
        pb = (L.P_f64 * n)(*[_pd(a) for a in bs])
        px = (L.P_f64 * n)(*[_pd(a) for a in xs])
        st = (L.SolveStats * n)()
        L.check(L.lib().cup2d_batch_solve(self._h, pb, px, st), "cup2d_batch_solve")
        self.last_stats = [s.as_dict() for s in st]
        return self.last_stats

    def set_profiling(self, enable: bool = True) -> None:
        L.check(L.lib().cup2d_batch_set_profiling(self._h, int(bool(enable))), "cup2d_batch_set_profiling")

    def profile(self) -> dict:
        """Per-phase (compute ms, barrier-wait ms), per-CTA averages over the
        launches since profiling was enabled (phases as Solver.PHASES)."""
        c = np.zeros(10)
        w = np.zeros(10)
        L.check(L.lib().cup2d_batch_profile(self._h, _pd(c), _pd(w), 10), "cup2d_batch_profile")
        return {name: (float(c[i]), float(w[i])) for i, name in enumerate(Solver.PHASES) if c[i] or w[i]}

    def timeline(self) -> tuple[np.ndarray, np.ndarray, float]:
        """(begin_ms, end_ms, launch_ms) of the last solve that returned stats."""
        n = len(self)
        b = np.empty(n)
        e = np.empty(n)
        t = C.c_double()
        L.check(L.lib().cup2d_batch_timeline(self._h, _pd(b), _pd(e), C.byref(t)), "cup2d_batch_timeline")
        return b, e, t.value


class Server:
    """Request server (no counterpart in the reference): register meshes,
    submit solves from any thread, poll or wait for them.  Every request runs
    as its own persistent solve of `team` CTAs; requests overlap on the
    device as slots and memory allow.  Host arrays passed to submit must stay
    alive (and unmodified) until the request completes; pinned memory makes
    the copies asynchronous."""

    WARM_START = 1

    def __init__(self, max_inflight: int = 24, team: int = 16, hbm_budget_bytes: int = 0,
                 opts: Optional[L.SolveOpts] = None, blocks_per_cta: int = 320, solve_share: float = 0.9,
                 **kw):
        o = L.ServerOpts()
        L.lib().cup2d_server_default_opts(C.byref(o))
        o.max_inflight = max_inflight
        o.team = team
        o.blocks_per_cta = blocks_per_cta
        o.solve_share = solve_share
        o.hbm_budget_bytes = hbm_budget_bytes
        o.solve = opts if opts is not None else make_opts(**kw)
        self._h = C.c_void_p()
        L.check(L.lib().cup2d_server_create(C.byref(o), C.byref(self._h)), "cup2d_server_create")
        self._keep: dict[int, tuple] = {}   # request -> (b, x) kept alive until completion
        self._meshes: list = []

    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            L.lib().cup2d_server_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def add_mesh(self, mesh: Mesh) -> int:
        f = mesh.forest()
        mid = C.c_int64()
        L.check(L.lib().cup2d_server_add_mesh(self._h, C.byref(f), C.byref(mid)), "cup2d_server_add_mesh")
        self._meshes.append(mesh)
        return mid.value

    def submit(self, mesh_id: int, b: np.ndarray, x: np.ndarray, warm_start: bool = False) -> int:
        for a in (b, x):
            if a.dtype != np.float64 or not a.flags.c_contiguous:
                raise ValueError("b and x must be contiguous float64 arrays")
        rid = C.c_int64()
        L.check(L.lib().cup2d_server_submit(self._h, int(mesh_id), _pd(b), _pd(x),
                                            self.WARM_START if warm_start else 0, C.byref(rid)),
                "cup2d_server_submit")
        self._keep[rid.value] = (b, x)
        return rid.value

    def _result(self, rid: int, st: int, stats: L.SolveStats, lat: C.c_double):
        if st == L.PENDING:
            return None
        self._keep.pop(rid, None)
        d = stats.as_dict()
        d["latency_ms"] = lat.value
        return d

    def poll(self, rid: int) -> Optional[dict]:
        """None while the request is pending, else its statistics (once)."""
        stats, lat = L.SolveStats(), C.c_double()
        st = L.lib().cup2d_server_poll(self._h, int(rid), C.byref(stats), C.byref(lat))
        if st == L.INVALID_ARGUMENT:
            raise L.Cup2dError(st, "cup2d_server_poll")
        return self._result(rid, st, stats, lat)

    def wait(self, rid: int, timeout_ms: int = 60000) -> Optional[dict]:
        stats, lat = L.SolveStats(), C.c_double()
        st = L.lib().cup2d_server_wait(self._h, int(rid), int(timeout_ms), C.byref(stats), C.byref(lat))
        if st == L.INVALID_ARGUMENT:
            raise L.Cup2dError(st, "cup2d_server_wait")
        return self._result(rid, st, stats, lat)

    def take_completed(self, max_ids: int = 256, timeout_ms: int = 0) -> list[int]:
        """Ids of requests that finished since the last call (then poll them)."""
        ids = (C.c_int64 * max_ids)()
        n = C.c_int32()
        L.check(L.lib().cup2d_server_take_completed(self._h, ids, int(max_ids), int(timeout_ms), C.byref(n)),
                "cup2d_server_take_completed")
        return list(ids[:n.value])

    def counters(self) -> dict:
        c = L.ServerCounters()
        L.check(L.lib().cup2d_server_get_counters(self._h, C.byref(c)), "cup2d_server_get_counters")
        return c.as_dict()


def _stream_handle(stream) -> C.c_void_p:
    """cudaStream_t of a torch stream; torch's current stream by default."""
    if stream is None:
        import torch
        stream = torch.cuda.current_stream()
    return C.c_void_p(stream.cuda_stream)


F64 = "torch.float64"


def _check_dev(t, n: int, dtype: str | None = None) -> None:
    if not (hasattr(t, "is_cuda") and t.is_cuda and t.is_contiguous() and t.numel() == n):
        raise ValueError(f"expected a contiguous CUDA tensor of {n} elements")
    if dtype is not None and str(t.dtype) != dtype:
        raise ValueError(f"expected a {dtype} tensor, got {t.dtype}")


def device_pinv() -> np.ndarray:
    P = np.empty(4096, dtype=np.float64)
    L.check(L.lib().cup2d_pinv(_pd(P)), "cup2d_pinv")
    return P.reshape(64, 64)


# ------------------------------------------------- reference interface ----

@dataclass
class ScalarGrid:
    """A scalar field on a mesh: data[block, iy, ix]."""
    mesh: Mesh
    data: object  # numpy (nblocks,8,8) float64, or a CUDA tensor of that shape

    @classmethod
    def zeros(cls, mesh: Mesh, device=None) -> "ScalarGrid":
        if device is None:
            return cls(mesh, np.zeros((mesh.nblocks, 8, 8)))
        import torch
        return cls(mesh, torch.zeros((mesh.nblocks, 8, 8), dtype=torch.float64, device=device))


@dataclass
class SimulationData:
    """The fields of CUP2D's SimulationData that the Poisson path reads
    (source/Simulation.cpp:239-245, ExpAMRSolver.cpp:366-372)."""
    mesh: Mesh
    poissonSolver: str = "cuda_iterative"
    PoissonTol: float = 1e-6
    PoissonTolRel: float = 0.0
    maxPoissonRestarts: int = 30
    maxPoissonIterations: int = 1000
    bMeanConstraint: int = 0
    step: int = 0
    precision: str = "fp64"
    UpdateFluxCorrection: bool = True  # set when the mesh changed


class PoissonSolver:
    """Base.h:8-13."""

    def solve(self, input: ScalarGrid, output: ScalarGrid) -> None:  # noqa: A002
        raise NotImplementedError


class ExpAMRSolver(PoissonSolver):
    """`cuda_iterative`: BiCGSTAB + 64x64 block-Jacobi on the GPU.

    Follows ExpAMRSolver::solve: tolerances are zero and restarts 100 for the
    first 10 steps (ExpAMRSolver.cpp:366-368), the operator is re-assembled
    when the mesh changed (UpdateFluxCorrection, :370-376), output holds the
    initial guess and receives the solution with its volume-weighted mean
    removed (:383-415)."""

    def __init__(self, sim: SimulationData):
        self.sim = sim
        self.solver = Solver(sim.mesh, self._opts())
        sim.UpdateFluxCorrection = False

    def _opts(self) -> L.SolveOpts:
        s = self.sim
        early = s.step < 10
        return make_opts(tol_abs=0.0 if early else s.PoissonTol, tol_rel=0.0 if early else s.PoissonTolRel,
                         max_restarts=100 if early else s.maxPoissonRestarts, max_iter=s.maxPoissonIterations,
                         precision=s.precision, mean_constraint=s.bMeanConstraint)

    def solve(self, input: ScalarGrid, output: ScalarGrid) -> None:  # noqa: A002
        s = self.sim
        if s.UpdateFluxCorrection:
            s.UpdateFluxCorrection = False
            self.solver.update_mesh(s.mesh)
        self.solver.set_opts(self._opts())
        if isinstance(input.data, np.ndarray):
            x = self.solver.solve(input.data.reshape(-1), np.asarray(output.data).reshape(-1))
            output.data[...] = x.reshape(-1, 8, 8)
        else:
            self.solver.solve_device(input.data.reshape(-1), output.data.view(-1))


def makePoissonSolver(sim: SimulationData) -> PoissonSolver:
    """Base.cpp:8-30."""
    if sim.poissonSolver == "cuda_iterative":
        return ExpAMRSolver(sim)
    if sim.poissonSolver == "iterative":
        raise NotImplementedError('Poisson solver "iterative" (the CPU AMRSolver) is not part of cup2d_b200; '
                                  'use "cuda_iterative"')
    raise ValueError(f'Poisson solver: "{sim.poissonSolver}" unrecognized!')
