"""torch.autograd wrapper of the Levin matting solve and its adjoint.

alpha = levin_matte(image, gamma, s) assembles the Levin Laplacian of the
[0, 1] RGB image (Matting.cu:79-218 math, eps as a parameter), solves
(L + diag(gamma)) alpha = gamma * s on the GPU (multigrid-preconditioned CG
by default), and on backward runs gm_levin_adjoint: one more solve of the symmetric
system for lambda, then the window-statistics back-propagation to the image
and lambda * (s - alpha) for gamma.  The reference has no gradients; this is
the differentiable form of its cgSolve path (main.cu:458-526).
"""
from __future__ import annotations

import torch

from . import api


class LevinMatte(torch.autograd.Function):
    @staticmethod
    def forward(ctx, image, gamma, s, eps: float, precision: str, rtol: float, max_iters: int,
                adjoint_rtol: float, solver: str):
        if image.dim() != 3 or image.shape[2] != 3 or image.dtype != torch.float32 or not image.is_cuda:
            raise ValueError("image must be a CUDA float32 tensor of shape (H, W, 3)")
        H, W, _ = image.shape
        if gamma.shape != (H, W) or s.shape != (H, W):
            raise ValueError("gamma and s must be (H, W)")
        im4 = torch.zeros((H, W, 4), dtype=torch.float32, device=image.device)
        im4[..., :3] = image.detach()
        g = gamma.detach().to(torch.float32).contiguous()
        sv = s.detach().to(torch.float32).contiguous()
        store = api.LevinStore(W, H, precision).assemble(im4, gamma_map=g, s_map=sv, eps=eps)
        alpha = torch.full((H, W), 0.5, dtype=torch.float32, device=image.device)
        res = store.solve(alpha, solver, rtol=rtol, max_iters=max_iters)
        ctx.store = store
        ctx.solve = res
        ctx.adjoint_rtol = adjoint_rtol
        ctx.max_iters = max_iters
        ctx.solver = solver
        ctx.save_for_backward(alpha)
        return alpha

    @staticmethod
    def backward(ctx, grad_alpha):
        (alpha,) = ctx.saved_tensors
        dimage, dgamma, _, res = ctx.store.adjoint(alpha, grad_alpha.detach().to(torch.float32).contiguous(),
                                                   solver=ctx.solver, rtol=ctx.adjoint_rtol, max_iters=ctx.max_iters)
        ctx.adjoint_solve = res
        return dimage[..., :3].contiguous(), dgamma, None, None, None, None, None, None, None


def levin_matte(image, gamma, s, eps: float = 1e-5, precision: str = "fp16", rtol: float = 1e-6,
                max_iters: int = 5000, adjoint_rtol: float | None = None, solver: str = "mg"):
    """Differentiable matte: alpha (H, W) from image (H, W, 3) in [0, 1],
    per-pixel scribble weights gamma and targets s (both (H, W)).  solver:
    "mg" (multigrid-preconditioned CG, the default: the fastest solve, and the
    one whose adjoint converges at every size and eps tried), "cg" or "pcg"
    (Jacobi-preconditioned) for both the solve and the adjoint; an adjoint
    solve with "cg" or "pcg" that does not converge is redone with "mg"."""
    return LevinMatte.apply(image, gamma, s, eps, precision, rtol, max_iters,
                            rtol if adjoint_rtol is None else adjoint_rtol, solver)
