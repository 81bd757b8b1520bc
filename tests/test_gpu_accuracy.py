"""Accuracy of the solved matte against the FP64 oracle solution, not only its
residual.

The Levin system at eps = 1e-5 is ill-conditioned: stopped at relative
residual 1e-6, every solver (the FP64 oracle's own CG included) leaves alpha
about 0.2 (640x480) to 0.3 (1920x1080) max-abs from the FP64 solution.  A
matte within 1e-4 of it takes rel-res about 1e-10.  The mixed solvers reach
that: their FP64 replacement runs on the FP32 planes, and the FP32 store's
exact solution lies within 1e-6 of the FP64 one.  The plain FP32 method
cannot: its FP32 iterate stalls near rel-res 1e-5.  Here:

* CG and Jacobi PCG to 1e-10 on FP16, BF16 and FP32 stores match the FP64
  oracle CG (run to 1e-12) within 1e-4 max-abs;
* at rel-res 1e-6 the mixed CG is as accurate as FP64 CG at 1e-6;
* steepest descent and damped Jacobi reach a true rel-res of 1e-6;
* with GM_LONG_TESTS=1, the same at 1920x1080 (the FP64 oracle solve takes
  a few minutes of host time).
"""
import os

import numpy as np
import pytest

from gpu_util import oracle_problem, torch_cuda

pytestmark = pytest.mark.gpu
TOL = 1e-4


def _fp64(orc, W, H, rtol):
    p, w, g, b = oracle_problem(orc, W, H, seed=0)
    op = orc.Operator(W=W, H=H, w=w, gamma=g)
    x0 = np.full(W * H, 0.5)
    x64, _, rel = op.cg(b, x0, rtol=rtol, maxit=100000)
    assert rel <= rtol
    x6, _, _ = op.cg(b, x0, rtol=1e-6, maxit=100000)
    return p, g, b, x64, float(np.abs(x6 - x64).max())


@pytest.fixture(scope="module")
def vga(orc):
    return _fp64(orc, 640, 480, 1e-12)


def _solve(p, prec, solver, rtol, max_iters=50000, st=None):
    torch = torch_cuda()
    from gpumatting_b200 import api

    if st is None:
        st = api.LevinStore(p.W, p.H, prec).assemble(torch.from_numpy(p.image).cuda(),
                                                     torch.from_numpy(p.scribbles).cuda(), eps=p.eps,
                                                     gamma_value=100.0)
    alpha = torch.full((p.H, p.W), 0.5, device="cuda")
    res = st.solve(alpha, solver, rtol=rtol, max_iters=max_iters)
    return st, res, alpha.double().cpu().numpy().ravel()


def _true_relres(orc, st, g, b, x):
    w32 = st.planes("w32")[:, :, :st.W].reshape(12, -1).double().cpu().numpy()
    op = orc.Operator(W=st.W, H=st.H, w=w32, gamma=g)
    return np.linalg.norm(b - op.apply(x)) / np.linalg.norm(b)


@pytest.mark.parametrize("prec,solver", [("fp16", "cg"), ("fp16", "pcg"), ("bf16", "cg"), ("fp32", "cg"),
                                         ("fp32", "pcg")])
def test_tight_solve_within_1e4_of_fp64(vga, prec, solver):
    p, g, b, x64, _ = vga
    _, res, x = _solve(p, prec, solver, 1e-10)
    assert res.status == 0 and res.rel_residual <= 1e-10, res
    err = np.abs(x - x64).max()
    print(f"640x480 {prec} {solver} rel-res 1e-10: {res.iters} it, alpha max-abs vs FP64 {err:.2e}")
    assert err <= TOL


def test_rel_res_1e6_as_accurate_as_fp64_cg(vga):
    p, g, b, x64, err64 = vga
    _, res, x = _solve(p, "fp16", "cg", 1e-6)
    assert res.status == 0, res
    err = np.abs(x - x64).max()
    print(f"640x480 rel-res 1e-6: alpha max-abs vs FP64 {err:.3f} (FP64 CG at 1e-6: {err64:.3f})")
    assert err <= 1.5 * err64


@pytest.mark.parametrize("solver", ["gd", "jacobi"])
def test_gd_and_jacobi_reach_1e6(orc, vga, solver):
    p, g, b, x64, _ = vga
    st, res, x = _solve(p, "fp16", solver, 1e-6, max_iters=400000)
    assert res.status == 0 and res.rel_residual <= 1e-6, res
    assert _true_relres(orc, st, g, b, x) <= 1.05e-6
    print(f"640x480 {solver} to 1e-6: {res.iters} it, alpha max-abs vs FP64 {np.abs(x - x64).max():.3f}")


@pytest.mark.skipif(not os.environ.get("GM_LONG_TESTS"), reason="set GM_LONG_TESTS=1 (minutes of host time)")
def test_1080p_accuracy(orc):
    p, g, b, x64, err64 = _fp64(orc, 1920, 1080, 1e-11)
    st = None
    for solver in ("cg", "pcg"):
        st, res, x = _solve(p, "fp16", solver, 1e-10, st=st)
        err = np.abs(x - x64).max()
        print(f"1080p fp16 {solver} rel-res 1e-10: {res.iters} it, alpha max-abs vs FP64 {err:.2e}")
        assert res.status == 0 and err <= TOL
    _, res, x = _solve(p, "fp16", "cg", 1e-6, st=st)
    err = np.abs(x - x64).max()
    print(f"1080p fp16 cg rel-res 1e-6: alpha max-abs vs FP64 {err:.3f} (FP64 CG at 1e-6: {err64:.3f})")
    assert res.status == 0 and err <= 1.5 * err64
    for solver in ("gd", "jacobi"):
        _, res, x = _solve(p, "fp16", solver, 1e-6, max_iters=400000, st=st)
        assert res.status == 0 and res.rel_residual <= 1e-6, res
        assert _true_relres(orc, st, g, b, x) <= 1.05e-6
        print(f"1080p {solver} to 1e-6: {res.iters} it, alpha max-abs vs FP64 {np.abs(x - x64).max():.3f}")
