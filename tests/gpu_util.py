"""Shared helpers for the GPU tests (problem set-up via the CPU oracle)."""
import numpy as np

from gpumatting_b200.synth import make_problem


def torch_cuda():
    import torch

    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    return torch


def oracle_problem(orc, W, H, seed=0, eps=None):
    """Synthetic problem + its FP64 oracle operator pieces."""
    p = make_problem(W, H, seed, eps=eps)
    w = orc.levin_sym64(p.image.astype(np.float64) / 255.0, p.eps)
    g = p.gamma.ravel().astype(np.float64)
    b = (p.gamma * p.s).ravel().astype(np.float64)
    return p, w, g, b


def bands25_f32(orc, w, g, W, H):
    """Reference-layout FP32 bands of the FP64 Laplacian (diagonal = row sum
    of the rounded off-diagonals + gamma, as the GPU assembly builds it)."""
    a = orc.sym_to_bands64(w, g, W, H).astype(np.float32)
    off = np.delete(a, 12, axis=0).astype(np.float64)
    a[12] = (-off.sum(axis=0) + g).astype(np.float32)
    return a
