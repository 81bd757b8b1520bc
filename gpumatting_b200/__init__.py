"""gpumatting_b200: closed-form matting hot path for NVIDIA B200 (sm_100a).

The compute runs in libgpumat.so (CUDA kernels behind a C ABI, declared in
include/gpumat.h).  ``gpumatting_b200.api`` mirrors the reference's
BandedMatrix / Vector / Solve API over it; ``gpumatting_b200.synth`` builds
the seeded synthetic problems.
"""
from ._lib import LIB_PATH, load  # noqa: F401

__all__ = ["LIB_PATH", "load"]
