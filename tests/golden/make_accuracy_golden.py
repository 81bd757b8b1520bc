"""Generates tests/golden/accuracy_1080p.npz: the FP64 solution of the
1920x1080 synthetic problem, the reference the GPU solvers' mattes are
checked against at the headline size.

Problem: the synthetic generator at 1920x1080, seed 0 (eps 1e-5, gamma 100
on ~10% scribbled pixels), image as uint8 RGB / 255 in FP64.  The FP64
oracle (oracle.levin_sym64 assembly, oracle.Operator.cg, OpenMP) solves
(L + diag(gamma)) alpha = gamma s from alpha = 0.5:
  alpha64  to relative residual 1e-12 (about 1e-6 max-abs from the exact
           solution on this system),
  alpha6   to relative residual 1e-6 (the accuracy any solver has there).
Both are stored on the grid of every 6th row and column starting at (3, 3)
(320 x 180 samples, float32), with err6 = max |alpha6 - alpha64| over the
WHOLE image and a checksum of the generated image and scribbles, so a change
of the generator fails loudly instead of comparing different problems.
Run from the repository root (a few minutes on 8 cores):
    python tests/golden/make_accuracy_golden.py
"""
from __future__ import annotations

import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from gpumatting_b200.synth import make_problem  # noqa: E402
from oracle import oracle as O  # noqa: E402

OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "accuracy_1080p.npz")
W, H, SEED = 1920, 1080, 0
STRIDE, OFF = 6, 3


def problem_checksum(p) -> np.ndarray:
    """Order-dependent checksum of the generated inputs (uint64 pair)."""
    img = p.image.astype(np.uint64).ravel()
    sc = p.scribbles.astype(np.uint64).ravel()
    k = np.arange(1, img.size + 1, dtype=np.uint64)
    ks = np.arange(1, sc.size + 1, dtype=np.uint64)
    return np.array([int(np.sum(img * k) % np.uint64(2**61 - 1)), int(np.sum(sc * ks) % np.uint64(2**61 - 1))],
                    np.uint64)


def sample(x: np.ndarray) -> np.ndarray:
    return np.ascontiguousarray(x.reshape(H, W)[OFF::STRIDE, OFF::STRIDE], np.float32)


def main():
    O.build(ref=False)
    t0 = time.time()
    p = make_problem(W, H, SEED)
    w = O.levin_sym64(p.image.astype(np.float64) / 255.0, p.eps)
    g = p.gamma.ravel().astype(np.float64)
    b = (p.gamma * p.s).ravel().astype(np.float64)
    op = O.Operator(W=W, H=H, w=w, gamma=g)
    x0 = np.full(W * H, 0.5)
    x64, it64, rel64 = op.cg(b, x0, rtol=1e-12, maxit=200000)
    x6, it6, rel6 = op.cg(b, x0, rtol=1e-6, maxit=200000)
    assert rel64 <= 1e-12 and rel6 <= 1e-6
    err6 = float(np.abs(x6 - x64).max())
    np.savez_compressed(OUT, W=np.int32(W), H=np.int32(H), seed=np.int32(SEED), eps=np.float64(p.eps),
                        stride=np.int32(STRIDE), off=np.int32(OFF), alpha64=sample(x64), alpha6=sample(x6),
                        err6=np.float64(err6), it64=np.int32(it64), rel64=np.float64(rel64), it6=np.int32(it6),
                        checksum=problem_checksum(p))
    print(f"wrote {OUT}: FP64 CG {it64} it to {rel64:.2e}, {it6} it to 1e-6 (max-abs {err6:.3f}), "
          f"{time.time() - t0:.0f} s")


if __name__ == "__main__":
    main()
