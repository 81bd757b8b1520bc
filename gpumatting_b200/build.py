"""Builds libgpumat.so (the C-ABI library) in-tree for sm_100a with nvcc.

Usage: python -m gpumatting_b200.build [--verbose-ptxas]
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libgpumat.so")
SOURCES = ["gm_common.cu", "gm_vector.cu", "gm_banded.cu", "gm_levin.cu", "gm_apply.cu", "gm_io.cu", "gm_solver.cu", "gm_mg.cu", "gm_capi.cu", "gm_hostsolve.cu"]
NVCC = os.environ.get("NVCC", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _deps() -> list[str]:
    out = [os.path.join(CSRC, f) for f in os.listdir(CSRC)]
    out.append(os.path.join(HERE, "..", "include", "gpumat.h"))
    return out


def up_to_date() -> bool:
    if not os.path.exists(LIB):
        return False
    t = os.path.getmtime(LIB)
    return all(os.path.getmtime(p) <= t for p in _deps())


def build(force: bool = False, ptxas_verbose: bool = False, jobs: int | None = None) -> str:
    if not force and up_to_date():
        return LIB
    objs = []
    procs = []
    odir = os.path.join(HERE, "_build")
    os.makedirs(odir, exist_ok=True)
    for src in SOURCES:
        obj = os.path.join(odir, src.replace(".cu", ".o"))
        cmd = [NVCC, "-O3", "-std=c++17", *ARCH, "-lineinfo", "-Xcompiler", "-fPIC,-O2",
               "-I", os.path.join(HERE, "..", "include"), "-c", os.path.join(CSRC, src), "-o", obj]
        if ptxas_verbose:
            cmd.insert(1, "-Xptxas=-v")
        procs.append((src, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)))
        objs.append(obj)
    failed = False
    for src, p in procs:
        out, _ = p.communicate()
        if out.strip():
            sys.stderr.write(out)
        if p.returncode != 0:
            failed = True
            sys.stderr.write(f"nvcc failed on {src}\n")
    if failed:
        raise RuntimeError("libgpumat build failed")
    tmp = LIB + ".tmp"
    subprocess.check_call([NVCC, "-shared", *ARCH, "-o", tmp, *objs, "-Xcompiler", "-fPIC"])
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, ptxas_verbose="--verbose-ptxas" in sys.argv)
    print(LIB)
