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


def test_default_adjoint_converges_at_1024_eps1e7(orc):
    """The large-configuration adjoint on the default path: at eps = 1e-7 the
    lambda solve of CG and Jacobi PCG stalls (4096^2), so the adjoint's
    default solver is the multigrid PCG.  Checked here: it converges; lambda
    has a true FP64 relative residual of 1e-6 (host, oracle operator over
    the store's FP32 planes); the image gradient equals the FP64 window
    back-propagation (oracle.levin_backward64) of the GPU's own lambda and
    alpha within 1e-3; dgamma = lambda (s - alpha)."""
    torch = torch_cuda()
    W = H = 1024
    p = make_problem(W, H, 0, eps=1e-7)
    im, gamma, s, gt = _inputs(torch, p)
    im4 = torch.zeros((H, W, 4), device="cuda")
    im4[..., :3] = im
    st = api.LevinStore(W, H, "fp16").assemble(im4, gamma_map=gamma, s_map=s, eps=p.eps)
    alpha = torch.full((H, W), 0.5, device="cuda")
    r = st.solve(alpha, rtol=1e-6, max_iters=5000)
    assert r.status == 0, r
    dalpha = 2.0 * (alpha - gt) / (W * H)
    dimage, dgamma, lam, ra = st.adjoint(alpha, dalpha, rtol=1e-6, max_iters=5000)
    print(f"1024^2 eps 1e-7 default adjoint: {ra}")
    assert ra.status == 0 and ra.solver == "mg" and ra.rel_residual <= 1e-6, ra
    g = p.gamma.ravel().astype(np.float64)
    w32 = st.planes("w32")[:, :, :W].reshape(12, -1).double().cpu().numpy()
    op = orc.Operator(W=W, H=H, w=w32, gamma=g)
    rhs = dalpha.double().cpu().numpy().ravel()
    lam64 = lam.double().cpu().numpy().ravel()
    # lambda comes back in FP32; on this ill-conditioned system rounding even
    # the exact solution to FP32 leaves a relative residual far above 1e-6.
    # The floor is the residual of a half-ulp relative perturbation of lambda;
    # the solver's own FP64 residual (of its FP64 iterate) is the 1e-6 above.
    rel = np.linalg.norm(rhs - op.apply(lam64)) / np.linalg.norm(rhs)
    u = np.random.default_rng(0).uniform(-2.0**-24, 2.0**-24, lam64.size)
    floor = np.linalg.norm(op.apply(lam64 * u)) / np.linalg.norm(rhs)
    print(f"host FP64 residual of the FP32 lambda {rel:.2e}, FP32 storage floor {floor:.2e}")
    assert floor < 1e-2 and rel <= 1.05e-6 + 2.0 * floor
    a64 = alpha.double().cpu().numpy().ravel()
    im3 = im.double().cpu().numpy()
    want = orc.levin_backward64(orc.sym_edge_grad(lam64, a64, W, H), im3, p.eps)
    assert _rel(dimage[..., :3].cpu().numpy(), want) <= 1e-3
    assert _rel(dgamma.cpu().numpy().ravel(), lam64 * (p.s.ravel() - a64)) <= 1e-5


def test_adjoint_falls_back_to_multigrid(orc):
    """A CG lambda solve that ends above rtol is redone from zero with the
    multigrid PCG: the result says so and equals the multigrid adjoint bit
    for bit."""
    torch = torch_cuda()
    W, H = 96, 64
    p = make_problem(W, H, 2)
    im, gamma, s, gt = _inputs(torch, p)
    im4 = torch.zeros((H, W, 4), device="cuda")
    im4[..., :3] = im
    st = api.LevinStore(W, H, "fp16").assemble(im4, gamma_map=gamma, s_map=s, eps=p.eps)
    alpha = torch.full((H, W), 0.5, device="cuda")
    st.solve(alpha, "mg", rtol=1e-9, max_iters=2000)
    dalpha = 2.0 * (alpha - gt) / (W * H)
    d1, g1, l1, r1 = st.adjoint(alpha, dalpha, "cg", rtol=1e-9, max_iters=400)  # CG needs more
    d2, g2, l2, r2 = st.adjoint(alpha, dalpha, "mg", rtol=1e-9, max_iters=400)
    assert r1.solver == "mg" and r2.solver == "mg" and r1.status == 0, (r1, r2)
    assert r1.iters == r2.iters
    for a, b in ((d1, d2), (g1, g2), (l1, l2)):
        assert torch.equal(a, b)
    d3, _, _, r3 = st.adjoint(alpha, dalpha, "cg", rtol=1e-9, max_iters=20000)  # converges: no fallback
    assert r3.solver == "cg" and r3.status == 0, r3
