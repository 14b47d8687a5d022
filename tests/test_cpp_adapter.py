"""The C++ drop-in (include/cup2d_poisson.hpp) compiles against the C ABI
and runs the PoissonSolver::solve call path."""
import subprocess
from pathlib import Path

import pytest

from cup2d_b200 import _lib as L

ROOT = Path(__file__).resolve().parent.parent


def _build(tmp_path) -> Path:
    exe = tmp_path / "adapter_demo"
    subprocess.run(["g++", "-std=c++17", "-O1", "-Wall", "-Werror", "-I", str(ROOT / "include"),
                    str(ROOT / "tests" / "cpp" / "adapter_demo.cpp"), "-L", str(L.LIB_PATH.parent),
                    "-lcup2d_poisson", f"-Wl,-rpath,{L.LIB_PATH.parent}", "-o", str(exe)], check=True)
    return exe


def test_adapter_compiles_and_reports_no_device(tmp_path, has_gpu):
    exe = _build(tmp_path)
    if has_gpu:
        pytest.skip("a GPU is present; see the gpu-marked run")
    r = subprocess.run([str(exe)], capture_output=True, text=True)
    assert r.returncode == 2, r.stdout


@pytest.mark.gpu
def test_adapter_solves(tmp_path, cuda):
    exe = _build(tmp_path)
    r = subprocess.run([str(exe)], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "status 0" in r.stdout


def test_c_batch_caller_compiles_as_c(tmp_path, has_gpu):
    """The header compiles as strict C11 with the batch, graph and
    time-stepping declarations; without a device the batch reports it."""
    exe = tmp_path / "batch_demo"
    subprocess.run(["gcc", "-std=c11", "-O1", "-Wall", "-Wextra", "-Werror", "-pedantic", "-I", str(ROOT / "include"),
                    str(ROOT / "tests" / "cpp" / "batch_demo.c"), "-L", str(L.LIB_PATH.parent),
                    "-lcup2d_poisson", f"-Wl,-rpath,{L.LIB_PATH.parent}", "-o", str(exe)], check=True)
    if has_gpu:
        pytest.skip("a GPU is present: the batch path is covered by the gpu-marked batch tests")
    r = subprocess.run([str(exe)], capture_output=True, text=True)
    assert r.returncode == 2, r.stdout + r.stderr


def test_cpp_batch_wrapper_compiles(tmp_path, has_gpu):
    """The C++ batch wrapper (cup2d_poisson.hpp) compiles with -Wall -Werror
    and, without a device, reports it through its exception."""
    exe = tmp_path / "batch_cpp_demo"
    subprocess.run(["g++", "-std=c++17", "-O1", "-Wall", "-Wextra", "-Werror", "-I", str(ROOT / "include"),
                    str(ROOT / "tests" / "cpp" / "batch_cpp_demo.cpp"), "-L", str(L.LIB_PATH.parent),
                    "-lcup2d_poisson", f"-Wl,-rpath,{L.LIB_PATH.parent}", "-o", str(exe)], check=True)
    if has_gpu:
        pytest.skip("a GPU is present: the batch path is covered by the gpu-marked batch tests")
    r = subprocess.run([str(exe)], capture_output=True, text=True)
    assert r.returncode == 2 and "no CUDA device" in r.stdout, r.stdout + r.stderr
