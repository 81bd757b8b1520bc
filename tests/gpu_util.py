"""Shared helpers for the tests (problem set-up via the CPU oracle); nothing
here needs a GPU until torch_cuda() is called."""
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


def edge_image(W, H, seed=0):
    """RGB8 soft edge with +-4 noise and column strokes (the problem of
    tests/c/test_native.c)."""
    v, u = np.mgrid[0:H, 0:W]
    a = 1.0 / (1.0 + np.exp(-(u - W // 2 + 5.0 * np.sin(v * 0.17 + seed)) / 2.0))
    i = (u + v * W).astype(np.int64)
    fg, bg = np.array([230.0, 60.0, 30.0]), np.array([25.0, 80.0, 200.0])
    img = np.empty((H, W, 3), np.uint8)
    for c in range(3):
        n = ((i * 7919 + c * 104729 + seed * 31) % 2**32) % 9 - 4
        val = a * fg[c] + (1 - a) * bg[c] + n
        img[..., c] = np.clip(np.floor(val + 0.5), 0, 255).astype(np.uint8)
    sc = np.full((H, W), 128, np.uint8)
    sc[(u >= W - 6) & (u < W - 2) & (v % 3 != 0)] = 255
    sc[(u >= 2) & (u < 6) & (v % 3 != 1)] = 0
    return img, sc
