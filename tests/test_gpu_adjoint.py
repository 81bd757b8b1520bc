"""Adjoint (gm_levin_adjoint and the torch.autograd wrapper) against the FP64
oracle adjoint and FP64 central finite differences.

Loss = mean((alpha - alpha_gt)^2).  Bar: image and scribble-weight gradients
within 1e-3 relative of the finite differences (h = 1e-4) on 64 seeded
pixels at 512x512 (fixture tests/golden/adjoint_512_fd.npz), and within
1e-3 relative (norm-wise) of the FP64 reference adjoint on whole images.
"""
import os

import numpy as np
import pytest

from gpumatting_b200 import api
from gpumatting_b200.synth import make_problem
from tests.gpu_util import torch_cuda

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "adjoint_512_fd.npz")


def _inputs(torch, p):
    im = torch.from_numpy(p.image).cuda().float() / 255.0
    gamma = torch.from_numpy(p.gamma).cuda()
    s = torch.from_numpy(p.s).cuda()
    gt = torch.from_numpy(p.alpha_gt.astype(np.float32)).cuda()
    return im, gamma, s, gt


def _rel(a, b):
    return float(np.linalg.norm(np.ravel(a) - np.ravel(b)) / max(np.linalg.norm(np.ravel(b)), 1e-300))


@pytest.mark.parametrize("precision", ["fp32", "fp16", "bf16"])
def test_store_adjoint_matches_fp64_reference(orc, precision):
    torch = torch_cuda()
    W, H = 96, 64
    p = make_problem(W, H, 2)
    im, gamma, s, gt = _inputs(torch, p)
    im4 = torch.zeros((H, W, 4), device="cuda")
    im4[..., :3] = im
    st = api.LevinStore(W, H, precision).assemble(im4, gamma_map=gamma, s_map=s, eps=p.eps)
    alpha = torch.full((H, W), 0.5, device="cuda")
    r = st.solve(alpha, "cg", rtol=1e-9, max_iters=20000)
    assert r.rel_residual <= 1e-9
    dalpha = 2.0 * (alpha - gt) / (W * H)
    dimage, dgamma, lam, ra = st.adjoint(alpha, dalpha, rtol=1e-9, max_iters=20000)
    assert ra.rel_residual <= 1e-9
    assert dimage.shape == (H, W, 4) and float(dimage[..., 3].abs().max()) == 0.0
    ref = orc.reference_adjoint(im.cpu().double().numpy(), p.gamma.astype(np.float64), p.s.astype(np.float64),
                                p.eps, p.alpha_gt)
    assert _rel(lam.cpu().numpy(), ref["lam"]) <= 1e-4
    assert _rel(dimage[..., :3].cpu().numpy(), ref["dimage"]) <= 1e-3
    assert _rel(dgamma.cpu().numpy(), ref["dgamma"]) <= 1e-3


def test_adjoint_rgb8_layout_and_scribble_map(orc):
    """uint8 RGB input and a 0/128/255 scribble map: 3-channel gradient, and
    dgamma uses the map's targets (1 on 255, 0 elsewhere)."""
    torch = torch_cuda()
    W, H = 80, 56
    p = make_problem(W, H, 4)
    img = torch.from_numpy(p.image).cuda()
    scr = torch.from_numpy(p.scribbles).cuda()
    st = api.LevinStore(W, H, "fp32").assemble(img, scribbles=scr, eps=p.eps, gamma_value=100.0)
    alpha = torch.full((H, W), 0.5, device="cuda")
    st.solve(alpha, "cg", rtol=1e-9, max_iters=20000)
    gt = torch.from_numpy(p.alpha_gt.astype(np.float32)).cuda()
    dimage, dgamma, lam, _ = st.adjoint(alpha, 2.0 * (alpha - gt) / (W * H), rtol=1e-9, max_iters=20000)
    assert dimage.shape == (H, W, 3)
    im3 = p.image.astype(np.float64) / 255.0
    gam = np.where(p.scribbles != 128, 100.0, 0.0)
    tgt = (p.scribbles == 255).astype(np.float64)
    ref = orc.reference_adjoint(im3, gam, tgt, p.eps, p.alpha_gt)
    assert _rel(dimage.cpu().numpy(), ref["dimage"]) <= 1e-3
    assert _rel(dgamma.cpu().numpy(), ref["dgamma"]) <= 1e-3


@pytest.mark.parametrize("solver", ["cg", "mg"])
def test_autograd_512_matches_finite_differences(solver):
    """The torch.autograd path at 512x512 against the FP64 FD fixture, with
    the fused CG and with the multigrid-preconditioned CG."""
    torch = torch_cuda()
    from gpumatting_b200.autograd import levin_matte

    g = np.load(GOLDEN)
    p = make_problem(int(g["W"]), int(g["H"]), int(g["seed"]))
    im, gamma, s, gt = _inputs(torch, p)
    im.requires_grad_(True)
    gamma.requires_grad_(True)
    alpha = levin_matte(im, gamma, s, eps=float(g["eps"]), precision="fp16", rtol=1e-9,
                        max_iters=20000 if solver == "cg" else 3000, solver=solver)
    loss = torch.mean((alpha - gt) ** 2)
    loss.backward()
    assert abs(loss.item() - float(g["loss"])) <= 1e-4 * float(g["loss"])
    v, u, c = g["v"], g["u"], g["c"]
    gi = im.grad.cpu().numpy()[v, u, c].astype(np.float64)
    gg = gamma.grad.cpu().numpy()[v, u].astype(np.float64)
    for got, fd, ref in ((gi, g["fd_image"], g["ref_image"]), (gg, g["fd_gamma"], g["ref_gamma"])):
        assert _rel(got, fd) <= 1e-3
        assert _rel(got, ref) <= 1e-3
        # per pixel: 1e-3 relative, with a floor at 1e-3 of the largest sample
        floor = 1e-3 * np.abs(fd).max()
        assert np.all(np.abs(got - fd) <= 1e-3 * np.abs(fd) + floor)
