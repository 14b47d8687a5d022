"""Generates the reference-produced fixtures under tests/golden/ with the
checker built from CUP2D's own Poisson sources (oracle/ref, oracle/_ref).

  python tests/golden/make_ref_fixtures.py assembly [--out DIR]
      CPU.  For every mesh of assembly_meshes(): the SHA-256 of the exact bytes
      of the reference's COO system (int32 rows, int32 columns, float64
      values, in the order LocalSpMatDnVec holds them) and of its P^-1, with
      sizes.  -> ref_assembly.json

  python tests/golden/make_ref_fixtures.py mean [--out DIR]
      GPU.  The same for the bMeanConstraint cases of MEAN_CASES (solved with
      sim.bMeanConstraint = 1).  -> ref_solve_<case>.npz

  python tests/golden/make_ref_fixtures.py solve [--out DIR]
      GPU.  For every case in SOLVE_CASES: ExpAMRSolver::solve with the
      reference's cuBLAS/cuSPARSE BiCGSTAB (x0 = 0, the case's tolerances),
      the mean-removed solution at every `stride`-th cell (at most 16,384
      cells, float64) with full-vector norms, and the statistics the
      reference's solver prints.  -> ref_solve_<case>.npz

Meshes and right-hand sides come from the library's own generators
(cup2d_b200.problems, Mesh.rhs_fourier); the fixtures record a SHA-256 of
each right-hand side so that a change of the generator shows up as such.
"""
from __future__ import annotations

import argparse
import hashlib
import json
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

HERE = Path(__file__).resolve().parent
MAX_SAMPLES = 16384


# batch problems (index into batch_problems(512, seed=3)) spanning the size
# range: the smallest, the quartiles and the largest
BATCH_PICKS = (320, 76, 440, 27, 156)


def assembly_meshes() -> dict:
    from cup2d_b200.problems import batch_problems
    out = {name: make() for name, make in assembly_meshes_light().items()}
    batch = batch_problems(512, seed=3)
    for k in BATCH_PICKS:
        out[f"batch_{k}"] = batch[k]
    return out


def mesh_by_name(name: str):
    """Rebuilds a fixture's mesh from its name (the tests use this); a
    "_rev" suffix lists the named mesh's blocks in reverse order."""
    if name.endswith("_rev"):
        from cup2d_b200.mesh import Mesh
        m = mesh_by_name(name[:-4])
        return Mesh(m.bpdx, m.bpdy, m.level_max, m.extent, m.level[::-1], m.bx[::-1], m.by[::-1], m.periodic_x,
                    m.periodic_y)
    if name.startswith("batch_"):
        from cup2d_b200.problems import batch_problems
        return batch_problems(512, seed=3)[int(name.split("_")[1])]
    return assembly_meshes_light()[name]()


def assembly_meshes_light() -> dict:
    """Name -> constructor, without building the 512-problem batch."""
    from cup2d_b200.mesh import Mesh
    from cup2d_b200.problems import large_mesh, quoted_small_mesh, sized_mesh, small_mesh
    return {
        "small": small_mesh,
        "small_quoted": quoted_small_mesh,
        "uniform": lambda: Mesh.uniform(2, 1, 3, 2, 2.0),
        "single_block": lambda: Mesh.uniform(1, 1, 1, 0, 1.0),
        "periodic_x": lambda: Mesh.disks(4, 2, 4, 2.0, [(1.0, 0.5, 0.12)], 0.1, periodic_x=True),
        "periodic_xy": lambda: Mesh.disks(2, 2, 4, 1.0, [(0.1, 0.9, 0.1)], 0.08, periodic_x=True,
                                          periodic_y=True),
        "sized_1500": lambda: sized_mesh(np.random.default_rng(5), 1500),
        "large": large_mesh,
    }


# case -> (mesh name, rhs seed, tol_abs, tol_rel)
SOLVE_CASES = {
    "small": ("small", 1, 1e-12, 1e-8),
    "small_quoted": ("small_quoted", 1, 1e-12, 1e-8),
    "sized_1500": ("sized_1500", 2, 0.0, 1e-8),
    "large": ("large", 1, 0.0, 1e-8),
    "large_rel1e6": ("large", 1, 0.0, 1e-6),
    "batch_320": ("batch_320", 100, 0.0, 1e-6),
    "batch_156": ("batch_156", 101, 0.0, 1e-6),
    "batch_320_1e8": ("batch_320", 100, 0.0, 1e-8),
    "batch_156_1e8": ("batch_156", 101, 0.0, 1e-8),
}


# bMeanConstraint cases: case -> (mesh name, rhs seed, tol_abs, tol_rel, constant
# added to the right-hand side).  A constant makes the Neumann problem
# incompatible; the constrained system is regular and solves it anyway.
MEAN_CASES = {
    "mean_small": ("small", 1, 0.0, 1e-8, 0.0),
    "mean_small_shift": ("small", 1, 0.0, 1e-8, 0.25),
    "mean_periodic_xy_rev": ("periodic_xy_rev", 3, 0.0, 1e-8, -0.1),
    "mean_sized_1500_rev": ("sized_1500_rev", 2, 0.0, 1e-8, 0.05),
}


def mean_case_rhs(case: str):
    mesh_name, seed, _, _, shift = MEAN_CASES[case]
    m = mesh_by_name(mesh_name)
    return m, m.rhs_fourier(seed) + shift


def coo_digest(row: np.ndarray, col: np.ndarray, val: np.ndarray) -> str:
    h = hashlib.sha256()
    h.update(np.ascontiguousarray(row, dtype="<i4").tobytes())
    h.update(np.ascontiguousarray(col, dtype="<i4").tobytes())
    h.update(np.ascontiguousarray(val, dtype="<f8").tobytes())
    return h.hexdigest()


def array_digest(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a, dtype="<f8").tobytes()).hexdigest()


def sample_stride(n: int) -> int:
    return max(1, -(-n // MAX_SAMPLES))


def make_assembly(out: Path) -> None:
    import oracle.ref as R
    rec = {}
    for name, m in assembly_meshes().items():
        r = R.assemble(m)
        rec[name] = {"nblocks": m.nblocks, "ncells": m.ncells, "nnz": int(r["val"].shape[0]),
                     "coo_sha256": coo_digest(r["row"], r["col"], r["val"]),
                     "h2_sha256": array_digest(r["h2"])}
        pinv = r["pinv"]
        print(f"{name}: {m.nblocks} blocks, {r['val'].shape[0]} nnz", flush=True)
    doc = {"what": "SHA-256 of the reference's assembled COO system (ExpAMRSolver::getMat + "
                   "LocalSpMatDnVec::make, int32 rows | int32 cols | float64 values, little-endian) "
                   "and of its P^-1 (ExpAMRSolver ctor, 64x64 row-major float64)",
           "generator": "tests/golden/make_ref_fixtures.py assembly",
           "pinv_sha256": array_digest(pinv), "meshes": rec}
    (out / "ref_assembly.json").write_text(json.dumps(doc, indent=1) + "\n")


def make_solve(out: Path, cases: list[str]) -> None:
    import oracle.ref as R
    for case in cases:
        mesh_name, seed, tol_abs, tol_rel = SOLVE_CASES[case]
        m = mesh_by_name(mesh_name)
        b = m.rhs_fourier(seed)
        t = time.time()
        x, st = R.solve(m, b, tol_abs=tol_abs, tol_rel=tol_rel)
        dt = time.time() - t
        s = sample_stride(m.ncells)
        h2 = np.repeat(m.cell_h() ** 2, 64)
        np.savez_compressed(
            out / f"ref_solve_{case}.npz", x_sample=x[::s], stride=np.int64(s), ncells=np.int64(m.ncells),
            x_norm2=np.float64(np.linalg.norm(x)), x_absmax=np.float64(np.abs(x).max()),
            x_h2_sum=np.float64(np.dot(h2, x)), rhs_sha256=np.array(array_digest(b)),
            mesh=np.array(mesh_name), seed=np.int64(seed), tol_abs=np.float64(tol_abs),
            tol_rel=np.float64(tol_rel), iterations=np.int64(st["iterations"] or -1),
            converged=np.bool_(st["converged"]), restarts=np.int64(st["restarts"]),
            err_init=np.float64(st["err_init"]), err_opt=np.float64(st["err_opt"]),
            norm_ax0=np.float64(st["norm_ax0"]), log=np.array(st["log"]))
        print(f"{case}: {m.nblocks} blocks, iterations {st['iterations']}, converged {st['converged']}, "
              f"restarts {st['restarts']}, err {st['err_init']:.3e} -> {st['err_opt']:.3e}, {dt:.1f} s",
              flush=True)


def make_mean(out: Path, cases: list[str]) -> None:
    import oracle.ref as R
    for case in cases:
        mesh_name, seed, tol_abs, tol_rel, shift = MEAN_CASES[case]
        m, b = mean_case_rhs(case)
        t = time.time()
        x, st = R.solve(m, b, tol_abs=tol_abs, tol_rel=tol_rel, mean_constraint=1)
        dt = time.time() - t
        s = sample_stride(m.ncells)
        h2 = np.repeat(m.cell_h() ** 2, 64)
        np.savez_compressed(
            out / f"ref_solve_{case}.npz", x_sample=x[::s], stride=np.int64(s), ncells=np.int64(m.ncells),
            x_norm2=np.float64(np.linalg.norm(x)), x_absmax=np.float64(np.abs(x).max()),
            x_h2_sum=np.float64(np.dot(h2, x)), rhs_sha256=np.array(array_digest(b)),
            mesh=np.array(mesh_name), seed=np.int64(seed), shift=np.float64(shift), mean_constraint=np.int64(1),
            tol_abs=np.float64(tol_abs), tol_rel=np.float64(tol_rel), iterations=np.int64(st["iterations"] or -1),
            converged=np.bool_(st["converged"]), restarts=np.int64(st["restarts"]),
            err_init=np.float64(st["err_init"]), err_opt=np.float64(st["err_opt"]),
            norm_ax0=np.float64(st["norm_ax0"]), log=np.array(st["log"]))
        print(f"{case}: {m.nblocks} blocks, iterations {st['iterations']}, converged {st['converged']}, "
              f"restarts {st['restarts']}, err {st['err_init']:.3e} -> {st['err_opt']:.3e}, {dt:.1f} s",
              flush=True)


def main() -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("what", choices=["assembly", "solve", "mean"])
    ap.add_argument("--out", default=str(HERE))
    ap.add_argument("--cases", default=",".join(SOLVE_CASES))
    a = ap.parse_args()
    out = Path(a.out)
    out.mkdir(parents=True, exist_ok=True)
    if a.what == "assembly":
        make_assembly(out)
    elif a.what == "mean":
        make_mean(out, list(MEAN_CASES) if a.cases == ",".join(SOLVE_CASES) else a.cases.split(","))
    else:
        make_solve(out, a.cases.split(","))
    return 0


if __name__ == "__main__":
    sys.exit(main())
