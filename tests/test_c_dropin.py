"""The drop-in C-ABI from C: tests/c/test_dropin.c follows the reference's
main.cu call sequence (hostLevinLaplacian, bmCopyToDevice, vecCopyToDevice,
cgSolve / gradSolve, computeError, the frees).  It is compiled with gcc
against include/gpumat.h and the in-tree libgpumat.so here (the header is
plain C) and run on the GPU."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CUDA = os.environ.get("CUDA_HOME", "/usr/local/cuda")


def _build(out: str) -> None:
    if shutil.which("gcc") is None:
        pytest.skip("gcc not available")
    lib = os.path.join(ROOT, "gpumatting_b200")
    cmd = ["gcc", "-std=c99", "-O2", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"),
           "-I", os.path.join(CUDA, "include"), os.path.join(ROOT, "tests", "c", "test_dropin.c"),
           "-L", lib, "-lgpumat", "-L", os.path.join(CUDA, "lib64"), "-lcudart",
           f"-Wl,-rpath,{lib}", f"-Wl,-rpath,{os.path.join(CUDA, 'lib64')}", "-lm", "-o", out]
    subprocess.run(cmd, check=True, capture_output=True, text=True)


def test_c_program_compiles_and_links(tmp_path):
    _build(str(tmp_path / "test_dropin"))


@pytest.mark.gpu
def test_c_program_runs_the_reference_sequence(tmp_path):
    exe = str(tmp_path / "test_dropin")
    _build(exe)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    print(r.stdout)
    assert r.returncode == 0 and "Test PASSED" in r.stdout, r.stdout + r.stderr
    assert "Ground truth MSE" in r.stdout
