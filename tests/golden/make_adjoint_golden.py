"""Generates tests/golden/adjoint_512_fd.npz: FP64 central finite differences
of the matting loss at 512x512, the reference values the adjoint is checked
against.

Problem: the synthetic generator at 512x512, seed 0 (eps 1e-5, gamma 100 on
~10% scribbled pixels).  The image is the uint8 RGB divided by 255 in float32
(what the GPU path receives), then widened to FP64.  Loss = mean((alpha -
alpha_gt)^2) with alpha solving (L(I) + diag(gamma)) alpha = gamma s.

For 64 seeded pixels (one seeded channel each) it stores
  fd_image  (loss(I + h e) - loss(I - h e)) / 2h,  h = 1e-4,
  fd_gamma  the same for gamma_i,
  ref_image / ref_gamma  the FP64 reference adjoint (oracle.reference_adjoint)
at those pixels.

Each perturbed loss is evaluated exactly rather than by differencing two
large sums: with delta = alpha' - alpha,
  loss(alpha') - loss(alpha) = g . delta + |delta|^2 / N,  g = 2 (alpha - gt) / N,
where an image perturbation changes only a 5x5 patch of the operator and
delta solves (A + dA) delta = -dA alpha by FP64 CG, and a gamma perturbation
is rank one, so delta = +-h (s_p - alpha_p) z / (1 +- h z_p) with z = A^-1 e_p
(Sherman-Morrison).  Run from the repository root (about half an hour on 8
cores):
    python tests/golden/make_adjoint_golden.py
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

OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "adjoint_512_fd.npz")
W = H = 512
SEED = 0
NPIX = 64
STEP = 1e-4


def main() -> None:
    p = make_problem(W, H, SEED)
    im = (p.image.astype(np.float32) / np.float32(255)).astype(np.float64)
    gamma = p.gamma.astype(np.float64)
    s = p.s.astype(np.float64)
    t0 = time.time()
    ref = O.reference_adjoint(im, gamma, s, p.eps, p.alpha_gt)
    print(f"reference adjoint: iters {ref['iters']} rel {ref['rel']} ({time.time() - t0:.1f} s)", flush=True)
    n = W * H
    alpha = ref["alpha"].ravel()
    g = ref["dalpha"].ravel()
    w = ref["w"]
    op = O.Operator(W=W, H=H, w=w, gamma=gamma)
    zero = np.zeros(n)
    rng = np.random.default_rng(1234)
    vs = rng.integers(0, H, NPIX)
    us = rng.integers(0, W, NPIX)
    cs = rng.integers(0, 3, NPIX)
    fd_image = np.zeros(NPIX)
    fd_gamma = np.zeros(NPIX)

    def dloss(delta: np.ndarray) -> float:
        return float(g @ delta + delta @ delta / n)

    for k in range(NPIX):
        v, u, c = int(vs[k]), int(us[k]), int(cs[k])
        d = []
        for sign in (1.0, -1.0):
            imp = im.copy()
            imp[v, u, c] += sign * STEP
            wp = O.levin_sym64(imp, p.eps)
            dA = O.Operator(W=W, H=H, w=wp - w, gamma=np.zeros(n))
            rhs = -dA.apply(alpha)
            opp = O.Operator(W=W, H=H, w=wp, gamma=gamma)
            delta, _, _ = opp.cg(rhs, zero, rtol=1e-11, maxit=200000)
            d.append(dloss(delta))
        fd_image[k] = (d[0] - d[1]) / (2 * STEP)
        i = v * W + u
        e = np.zeros(n)
        e[i] = 1.0
        z, _, _ = op.cg(e, zero, rtol=1e-12, maxit=200000)
        d = []
        for sign in (1.0, -1.0):
            delta = sign * STEP * (s.ravel()[i] - alpha[i]) * z / (1.0 + sign * STEP * z[i])
            d.append(dloss(delta))
        fd_gamma[k] = (d[0] - d[1]) / (2 * STEP)
        print(f"{k:2d} ({v},{u},{c}) fd_I {fd_image[k]: .6e} ref {ref['dimage'][v, u, c]: .6e} | "
              f"fd_g {fd_gamma[k]: .6e} ref {ref['dgamma'][v, u]: .6e}  ({time.time() - t0:.0f} s)", flush=True)
    np.savez_compressed(
        OUT, W=W, H=H, seed=SEED, step=STEP, v=vs, u=us, c=cs, fd_image=fd_image, fd_gamma=fd_gamma,
        ref_image=ref["dimage"][vs, us, cs], ref_gamma=ref["dgamma"][vs, us], loss=ref["loss"],
        eps=p.eps)
    print("wrote", OUT)


if __name__ == "__main__":
    main()
