"""The C-ABI from C, compiled with gcc against include/gpumat.h and the
in-tree libgpumat.so (the header is plain C) and run on the GPU, and from
C++ with the reference's own call forms (tests/c/test_cxx_callers.cpp).

tests/c/test_dropin.c follows the reference's main.cu call sequence
(hostLevinLaplacian, bmCopyToDevice, vecCopyToDevice, cgSolve / gradSolve,
computeError, the frees).  tests/c/test_native.c drives the native store API
(gm_levin_store_alloc, gm_levin_assemble, gm_levin_solve with CG / PCG / MG,
gm_levin_solve_mg_many, a gm_batch solve, gm_levin_adjoint) and checks each
solution on the host with an FP64 residual of the store's FP32 planes."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CUDA = os.environ.get("CUDA_HOME", "/usr/local/cuda")
PROGRAMS = ("test_dropin", "test_native", "test_cxx_callers")


def _build(name: str, out: str) -> None:
    cxx = os.path.exists(os.path.join(ROOT, "tests", "c", name + ".cpp"))
    compiler = "g++" if cxx else "gcc"
    if shutil.which(compiler) is None:
        pytest.skip(f"{compiler} not available")
    lib = os.path.join(ROOT, "gpumatting_b200")
    # C++: the reference's call forms (by-reference matrices, defaulted
    # arguments, float4 images); FMA contraction off so the program's own
    # host loops round as the reference's host build does
    std = ["-std=c++17", "-ffp-contract=off"] if cxx else ["-std=c99"]
    src = os.path.join(ROOT, "tests", "c", name + (".cpp" if cxx else ".c"))
    cmd = [compiler, *std, "-O2", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"),
           "-I", os.path.join(CUDA, "include"), src,
           "-L", lib, "-lgpumat", "-L", os.path.join(CUDA, "lib64"), "-lcudart",
           f"-Wl,-rpath,{lib}", f"-Wl,-rpath,{os.path.join(CUDA, 'lib64')}", "-lm", "-o", out]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr


@pytest.mark.parametrize("name", PROGRAMS)
def test_c_program_compiles_and_links(tmp_path, name):
    _build(name, str(tmp_path / name))


def _run(tmp_path, name: str) -> str:
    exe = str(tmp_path / name)
    _build(name, exe)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    print(r.stdout)
    assert r.returncode == 0 and "Test PASSED" in r.stdout, r.stdout + r.stderr
    return r.stdout


@pytest.mark.gpu
def test_c_program_runs_the_reference_sequence(tmp_path):
    assert "Ground truth MSE" in _run(tmp_path, "test_dropin")


@pytest.mark.gpu
def test_cxx_program_makes_the_reference_calls(tmp_path):
    """main.cu's C++ call forms compile unchanged against gpumat.h and give
    the reference's arithmetic (see tests/c/test_cxx_callers.cpp)."""
    assert "cg rel-res" in _run(tmp_path, "test_cxx_callers")


@pytest.mark.gpu
def test_c_program_drives_the_native_store_api(tmp_path):
    out = _run(tmp_path, "test_native")
    for what in ("CG:", "PCG:", "MG:", "mg_many[1]:", "batch[1]:", "adjoint:"):
        assert what in out
