"""The C ABI library: loads, exports every declared entry point, validates
its arguments and reports errors by status without a GPU."""
import ctypes as C
import re
import subprocess
from pathlib import Path

import numpy as np
import pytest

from cup2d_b200 import Mesh
from cup2d_b200 import _lib as L

ROOT = Path(__file__).resolve().parent.parent
HEADERS = sorted((ROOT / "include").glob("*.h"))


def declared_functions():
    names = set()
    for h in HEADERS:
        text = h.read_text()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"\b(cup2d_[a-z0-9_]+)\s*\(", text):
            names.add(m.group(1))
    return sorted(names)


def test_headers_exist():
    assert HEADERS, "include/*.h missing"
    assert len(declared_functions()) >= 25


@pytest.mark.parametrize("name", declared_functions())
def test_symbol_exported(name):
    lib = L.lib()
    assert hasattr(lib, name), f"{name} declared in include/ but not exported"


def test_exports_match_declarations():
    out = subprocess.run(["nm", "-D", "--defined-only", str(L.LIB_PATH)], capture_output=True, text=True,
                         check=True).stdout
    exported = {ln.split()[-1] for ln in out.splitlines() if " T cup2d_" in ln}
    assert exported == set(declared_functions())


def test_ctypes_signatures_cover_declarations():
    assert set(L.SIGNATURES) == set(declared_functions())


def test_built_for_sm100a():
    from cup2d_b200 import build
    assert build.ARCH == ["-gencode", "arch=compute_100a,code=sm_100a"]


def test_version_and_status_strings():
    lib = L.lib()
    assert b"sm_100a" in lib.cup2d_version()
    for s in range(11):
        assert lib.cup2d_status_string(s)


def test_default_opts_match_reference():
    o = L.SolveOpts()
    L.lib().cup2d_default_opts(C.byref(o))
    assert o.max_iter == 1000          # BiCGSTAB.cu:468
    assert o.precision == L.PREC_FP64
    assert o.subtract_mean == 1        # ExpAMRSolver.cpp:383-415
    assert 0 < o.reliable_delta < 1


def test_argument_validation_without_gpu():
    lib = L.lib()
    h = C.c_void_p()
    # null forest / out pointer
    assert lib.cup2d_poisson_create(None, None, C.byref(h)) == L.INVALID_ARGUMENT
    m = Mesh.uniform(1, 1, 1, 0, 1.0)
    f = m.forest()
    assert lib.cup2d_poisson_create(C.byref(f), None, None) == L.INVALID_ARGUMENT
    o = L.SolveOpts()
    lib.cup2d_default_opts(C.byref(o))
    o.reliable_delta = 2.0
    assert lib.cup2d_poisson_create(C.byref(f), C.byref(o), C.byref(h)) == L.INVALID_ARGUMENT
    assert lib.cup2d_poisson_solve(None, None, None, None) == L.INVALID_ARGUMENT
    assert lib.cup2d_poisson_destroy(None) == L.OK


def test_create_without_gpu_reports_no_device(has_gpu):
    if has_gpu:
        pytest.skip("a GPU is present")
    m = Mesh.uniform(1, 1, 1, 0, 1.0)
    f = m.forest()
    h = C.c_void_p()
    st = L.lib().cup2d_poisson_create(C.byref(f), None, C.byref(h))
    assert st == L.NO_DEVICE
    assert not h.value


def test_mesh_abi_roundtrip():
    lib = L.lib()
    d = np.array([0.5, 0.5, 0.1])
    h = C.c_void_p()
    assert lib.cup2d_mesh_disks(2, 2, 3, 1.0, 0, 0, 1, d.ctypes.data_as(C.POINTER(C.c_double)), 0.05,
                                C.byref(h)) == L.OK
    f = L.Forest()
    assert lib.cup2d_mesh_forest(h, C.byref(f)) == L.OK
    assert f.nblocks > 4 and lib.cup2d_forest_validate(C.byref(f)) == L.OK
    hb = np.empty(f.nblocks)
    assert lib.cup2d_forest_cell_h(C.byref(f), hb.ctypes.data_as(C.POINTER(C.c_double))) == L.OK
    assert np.all(hb > 0)
    assert lib.cup2d_mesh_destroy(h) == L.OK
    # invalid generator arguments
    assert lib.cup2d_mesh_disks(0, 2, 3, 1.0, 0, 0, 0, None, 0.05, C.byref(h)) == L.INVALID_ARGUMENT


def test_oracle_library_loads():
    import oracle
    assert oracle.num_threads() >= 1
    P = oracle.pinv()
    assert P.shape == (64, 64)
