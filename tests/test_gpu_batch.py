"""Batched solves (gm_batch_*): many uneven images in one persistent launch.

Each image of the batch must behave as if solved alone: its planes are the
ones a standalone store would hold (bit for bit), its solve reaches the same
true FP64 relative residual against the FP64 restatement of its own operator,
fixed-iteration GD / Jacobi match the oracle, and repeated solves (graph
replays) give identical bits.
"""
import ctypes as C

import numpy as np
import pytest

from gpumatting_b200 import _lib as L
from gpumatting_b200 import api
from gpumatting_b200.synth import make_problem
from tests.gpu_util import torch_cuda

pytestmark = pytest.mark.gpu

SIZES = [(37, 29), (300, 17), (256, 190), (97, 301), (513, 64), (200, 200), (1000, 12), (64, 700), (5, 3)]
TOL = 1e-4


def _batch(precision, sizes=SIZES):
    torch = torch_cuda()
    b = api.LevinBatch(sizes, precision)
    probs = []
    for k, (W, H) in enumerate(sizes):
        p = make_problem(W, H, 10 + k)
        b.assemble(k, torch.from_numpy(p.image).cuda(), torch.from_numpy(p.scribbles).cuda(), eps=p.eps,
                   gamma_value=100.0)
        probs.append(p)
    return b, probs


def _view_planes(b, k, W, H):
    """FP32 planes (12, H, W), gamma and b (H, W) of image k, read through its view."""
    torch = torch_cuda()
    v = b.store_view(k)
    P, ps = v.pitch, v.plane_stride
    w32 = api._wrap(v.w32, (11 * ps + H * P,), torch.float32).as_strided((12, H, W), (ps, P, 1))
    g = api._wrap(v.gamma, (H * P,), torch.float32).view(H, P)[:, :W]
    bb = api._wrap(v.b, (H * P,), torch.float32).view(H, P)[:, :W]
    return w32.double().cpu().numpy(), g.double().cpu().numpy(), bb.double().cpu().numpy()


def _relres(orc, w32, g, b, x, W, H):
    op = orc.Operator(W=W, H=H, w=w32.reshape(12, -1), gamma=g.ravel())
    return np.linalg.norm(b.ravel() - op.apply(x.ravel())) / np.linalg.norm(b.ravel())


def test_batch_planes_equal_standalone_store():
    torch = torch_cuda()
    b, probs = _batch("fp16", SIZES[:4])
    for k, (W, H) in enumerate(SIZES[:4]):
        p = probs[k]
        st = api.LevinStore(W, H, "fp16").assemble(torch.from_numpy(p.image).cuda(),
                                                   torch.from_numpy(p.scribbles).cuda(), eps=p.eps)
        w32, g, bb = _view_planes(b, k, W, H)
        assert np.array_equal(w32, st.planes("w32")[:, :, :W].double().cpu().numpy())
        assert np.array_equal(g, st.planes("gamma")[:, :W].double().cpu().numpy())
        assert np.array_equal(bb, st.planes("b")[:, :W].double().cpu().numpy())


@pytest.mark.parametrize("precision", ["fp16", "bf16", "fp32"])
def test_batch_cg_reaches_rtol_per_image(orc, precision):
    torch = torch_cuda()
    b, probs = _batch(precision)
    alphas = [torch.full((H, W), 0.5, device="cuda") for W, H in SIZES]
    res = b.solve(alphas, "cg", rtol=1e-6, max_iters=5000)
    info = b.info()
    assert info["graph_launches"] >= 1 and info["ctas_per_sm"] > 0
    for k, (W, H) in enumerate(SIZES):
        r = res[k]
        assert r.status == 0 and r.rel_residual <= 1e-6, (k, r)
        w32, g, bb = _view_planes(b, k, W, H)
        x = alphas[k].double().cpu().numpy()
        assert _relres(orc, w32, g, bb, x, W, H) <= 1.05e-6, k
        # the same image solved alone takes about as many iterations
        p = probs[k]
        st = api.LevinStore(W, H, precision).assemble(torch.from_numpy(p.image).cuda(),
                                                      torch.from_numpy(p.scribbles).cuda(), eps=p.eps)
        a1 = torch.full((H, W), 0.5, device="cuda")
        r1 = st.solve(a1, "cg", rtol=1e-6, max_iters=5000)
        assert abs(r.iters - r1.iters) <= 0.15 * r1.iters + 10, (k, r.iters, r1.iters)


def test_batch_gd_and_jacobi_fixed_iterations(orc):
    torch = torch_cuda()
    sizes = SIZES[:5]
    b, probs = _batch("fp32", sizes)
    for solver, kw in (("gd", {}), ("jacobi", {"omega": 0.6})):
        alphas = [torch.full((H, W), 0.5, device="cuda") for W, H in sizes]
        res = b.solve(alphas, solver, rtol=0.0, max_iters=25, **kw)
        for k, (W, H) in enumerate(sizes):
            w32, g, bb = _view_planes(b, k, W, H)
            op = orc.Operator(W=W, H=H, w=w32.reshape(12, -1), gamma=g.ravel())
            x0 = np.full(W * H, 0.5)
            if solver == "gd":
                ref, _, _ = op.gd(bb.ravel(), x0, maxit=25)
            else:
                ref, _, _ = op.jacobi(bb.ravel(), x0, omega=0.6, maxit=25)
                assert res[k].iters == 25
            assert np.abs(alphas[k].double().cpu().numpy().ravel() - ref).max() <= TOL, (solver, k)


def test_batch_replay_is_deterministic_and_tuned_shape_is_kept():
    torch = torch_cuda()
    b, _ = _batch("fp16")
    info0 = b.tune(iters=10)
    # 192-column strips at 3 (shallow rings) or 2 (deep) CTAs per SM, or
    # 128-column strips at 4
    assert (info0["ring_cfg"], info0["ctas_per_sm"]) in ((0, 3), (1, 2), (2, 4)), info0
    assert info0["strip_width"] == (128 if info0["ring_cfg"] == 2 else 192)
    outs = []
    for _ in range(2):
        alphas = [torch.full((H, W), 0.5, device="cuda") for W, H in SIZES]
        b.solve(alphas, "cg", rtol=0.0, max_iters=200)
        outs.append([a.cpu().numpy() for a in alphas])
    for x, y in zip(*outs):
        assert np.array_equal(x.view(np.uint32), y.view(np.uint32))
    info1 = b.info()
    assert info1["ctas_per_sm"] == info0["ctas_per_sm"] and info1["graph_launches"] >= info0["graph_launches"] + 2


def test_batch_timeout_status_and_recovery():
    """A first barrier that waits for an arrival that never comes ends every
    image with GM_ERR_TIMEOUT; the next solve of the same batch succeeds."""
    torch = torch_cuda()
    b, _ = _batch("fp16", SIZES[:3])
    alphas = [torch.full((H, W), 0.5, device="cuda") for W, H in SIZES[:3]]
    ptrs = (C.c_void_p * 3)(*[a.data_ptr() for a in alphas])
    infos = (L.GmSolveInfo * 3)()
    p = L.default_params(rtol=1e-6, timeout_s=0.2, inject=1, ctas_per_sm=3)
    rc = L.load().gm_batch_solve(b.h, ptrs, C.byref(p), infos, torch.cuda.current_stream().cuda_stream)
    assert rc == L.GM_ERR_TIMEOUT
    assert all(infos[k].status == L.GM_ERR_TIMEOUT for k in range(3))
    for a in alphas:
        a.fill_(0.5)
    res = b.solve(alphas, "cg", rtol=1e-6, ctas_per_sm=3)
    assert all(r.status == 0 and r.rel_residual <= 1e-6 for r in res)


def test_batch_pcg_reaches_rtol_per_image(orc):
    torch = torch_cuda()
    b, probs = _batch("fp16")
    alphas = [torch.full((H, W), 0.5, device="cuda") for W, H in SIZES]
    res = b.solve(alphas, "pcg", rtol=1e-6, max_iters=5000)
    alphas_cg = [torch.full((H, W), 0.5, device="cuda") for W, H in SIZES]
    res_cg = b.solve(alphas_cg, "cg", rtol=1e-6, max_iters=5000)
    for k, (W, H) in enumerate(SIZES):
        assert res[k].status == 0 and res[k].rel_residual <= 1e-6, (k, res[k])
        w32, g, bb = _view_planes(b, k, W, H)
        assert _relres(orc, w32, g, bb, alphas[k].double().cpu().numpy(), W, H) <= 1.05e-6, k
    assert sum(r.iters for r in res) < sum(r.iters for r in res_cg)
