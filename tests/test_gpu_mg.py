"""Multigrid-preconditioned CG (GM_SOLVER_MG) on the GPU against the FP64
oracle of oracle/mg.py: the Galerkin hierarchy level by level, one V-cycle,
solves to rel-res 1e-6 (FP16, BF16, FP32 stores) and 1e-10 (alpha within
1e-4 of the direct FP64 solve), determinism, odd shapes, and the status
paths.  The hierarchy is the 2x2-aggregate form of the reference's
unfinished aggregation operators (gridoperators.h:18-138)."""
import numpy as np
import pytest

from gpu_util import edge_image, oracle_problem, torch_cuda

pytestmark = pytest.mark.gpu
TOL = 1e-4


def _store(orc, W, H, prec, seed=2):
    torch = torch_cuda()
    from gpumatting_b200 import api

    p, w, g, b = oracle_problem(orc, W, H, seed)
    st = api.LevinStore(W, H, prec).assemble(torch.from_numpy(p.image).cuda(), torch.from_numpy(p.scribbles).cuda(),
                                             eps=p.eps, gamma_value=100.0)
    return st, p, w, g, b


def _oracle_levels(st, g, prec, use_low=True):
    from oracle import mg as M

    W, H = st.W, st.H
    low = use_low and prec != "fp32"
    wp = st.planes("w" if low else "w32")[:, :, :W].reshape(12, -1).double().cpu().numpy()
    dp = st.planes("d" if low else "d32")[:, :W].reshape(-1).double().cpu().numpy()
    return M, M.hierarchy(wp, dp, g, W, H)


def _true_relres(orc, st, g, b, x):
    W, H = st.W, st.H
    w32 = st.planes("w32")[:, :, :W].reshape(12, -1).double().cpu().numpy()
    op = orc.Operator(W=W, H=H, w=w32, gamma=g)
    return np.linalg.norm(b - op.apply(x)) / np.linalg.norm(b), op


@pytest.mark.parametrize("W,H,prec", [(160, 120, "fp16"), (37, 29, "fp32"), (300, 17, "bf16")])
def test_hierarchy_matches_oracle(orc, W, H, prec):
    st, p, w, g, b = _store(orc, W, H, prec)
    M, lv = _oracle_levels(st, g, prec)
    assert st.mg_levels() == [(l.W, l.H) for l in lv]
    for level in sorted({1, len(lv) - 1}):
        _, c, D = st.mg_inspect(None, level)
        ref = lv[level]
        scale = np.abs(ref.c).max()
        assert np.allclose(c, ref.c, rtol=1e-5, atol=1e-6 * scale), level
        assert np.allclose(D, ref.D, rtol=1e-5, atol=1e-6 * np.abs(ref.D).max()), level


@pytest.mark.parametrize("prec", ["fp16", "bf16", "fp32"])
def test_vcycle_matches_oracle(orc, prec):
    torch = torch_cuda()
    W, H = 200, 150
    st, p, w, g, b = _store(orc, W, H, prec)
    M, lv = _oracle_levels(st, g, prec)
    r = np.random.default_rng(7).standard_normal((H, W)).astype(np.float32)
    z, _, _ = st.mg_inspect(torch.from_numpy(r).cuda(), 0)
    ref = M.vcycle(lv, r.astype(np.float64))
    err = np.linalg.norm(z.double().cpu().numpy() - ref) / np.linalg.norm(ref)
    assert err <= 1e-4, err


@pytest.mark.parametrize("prec", ["fp16", "bf16", "fp32"])
def test_mg_solve_to_rtol(orc, prec):
    torch = torch_cuda()
    W, H = 160, 120
    st, p, w, g, b = _store(orc, W, H, prec)
    alpha = torch.full((H, W), 0.5, device="cuda")
    res = st.solve(alpha, "mg", rtol=1e-6, max_iters=2000)
    assert res.status == 0 and res.rel_residual <= 1e-6, res
    rel, op = _true_relres(orc, st, g, b, alpha.double().cpu().numpy().ravel())
    assert rel <= 1.05e-6
    M, lv = _oracle_levels(st, g, prec)
    _, it64, _ = M.mgpcg(lv, op.apply, b, np.full(W * H, 0.5), 1e-6, 2000)
    assert res.iters <= 1.3 * it64 + 10, (res.iters, it64)
    _, it_cg, _ = op.cg(b, np.full(W * H, 0.5), rtol=1e-6, maxit=20000)
    assert 4 * res.iters < it_cg, (res.iters, it_cg)


def test_mg_accurate_vs_direct(orc):
    """rtol 1e-10: alpha within 1e-4 max-abs of the FP64 direct solve."""
    import scipy.sparse as sp
    import scipy.sparse.linalg as spla

    torch = torch_cuda()
    W, H = 64, 48
    st, p, w, g, b = _store(orc, W, H, "fp16", seed=5)
    a = orc.sym_to_bands64(w, g, W, H)
    offs = orc.levin_offsets(W)
    N = W * H
    rows, cols, vals = [], [], []
    for k in range(25):
        i = np.arange(N)
        j = i + offs[k]
        m = (j >= 0) & (j < N) & (a[k] != 0)
        rows.append(i[m]); cols.append(j[m]); vals.append(a[k][m])
    Mx = sp.csr_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))), shape=(N, N))
    xs = spla.spsolve(Mx.tocsc(), b)
    alpha = torch.full((H, W), 0.5, device="cuda")
    res = st.solve(alpha, "mg", rtol=1e-10, max_iters=5000)
    assert res.status == 0 and res.rel_residual <= 1e-10, res
    assert np.abs(alpha.double().cpu().numpy().ravel() - xs).max() <= TOL


def test_mg_is_deterministic(orc):
    torch = torch_cuda()
    W, H = 300, 200
    st, p, w, g, b = _store(orc, W, H, "fp16")
    outs = []
    for _ in range(2):
        alpha = torch.full((H, W), 0.5, device="cuda")
        res = st.solve(alpha, "mg", rtol=0.0, max_iters=25)
        assert res.iters == 25 and res.status == 0
        outs.append(alpha.cpu().numpy())
    assert np.array_equal(outs[0].view(np.uint32), outs[1].view(np.uint32))


@pytest.mark.parametrize("W,H", [(8, 2), (5, 7), (97, 61), (130, 3)])
def test_mg_odd_shapes(orc, W, H):
    torch = torch_cuda()
    st, p, w, g, b = _store(orc, W, H, "fp16", seed=1)
    if not np.any(b):
        pytest.skip("no foreground scribble at this size")
    alpha = torch.full((H, W), 0.5, device="cuda")
    res = st.solve(alpha, "mg", rtol=1e-6, max_iters=2000)
    assert res.status == 0, res
    rel, _ = _true_relres(orc, st, g, b, alpha.double().cpu().numpy().ravel())
    assert rel <= 1.05e-6


def test_mg_zero_rhs_and_max_iters(orc):
    torch = torch_cuda()
    W, H = 96, 64
    st, p, w, g, b = _store(orc, W, H, "fp16")
    x = torch.full((H, W), 0.25, device="cuda")
    res = st.solve_rhs(torch.zeros((H, W), device="cuda"), x, "mg", rtol=1e-6)
    assert res.status == 0 and not x.any()
    alpha = torch.full((H, W), 0.5, device="cuda")
    res = st.solve(alpha, "mg", rtol=1e-30, max_iters=3)
    assert res.status == 6 and res.iters == 3  # NOT_CONVERGED, and the iterate is still written
    assert np.isfinite(alpha.cpu().numpy()).all()


def test_mg_adjoint_matches_cg_adjoint(orc):
    torch = torch_cuda()
    W, H = 96, 64
    st, p, w, g, b = _store(orc, W, H, "fp16")
    alpha = torch.full((H, W), 0.5, device="cuda")
    st.solve(alpha, "cg", rtol=1e-9, max_iters=20000)
    gt = torch.from_numpy(p.alpha_gt.astype(np.float32)).cuda()
    dalpha = 2.0 * (alpha - gt) / (W * H)
    d_cg, dg_cg, lam_cg, r_cg = st.adjoint(alpha, dalpha, "cg", rtol=1e-9, max_iters=20000)
    d_mg, dg_mg, lam_mg, r_mg = st.adjoint(alpha, dalpha, "mg", rtol=1e-9, max_iters=2000)
    assert r_mg.status == 0 and r_mg.iters * 4 < r_cg.iters, (r_mg, r_cg)
    for a_, b_ in ((lam_mg, lam_cg), (d_mg, d_cg), (dg_mg, dg_cg)):
        a_, b_ = a_.double().cpu().numpy(), b_.double().cpu().numpy()
        assert np.linalg.norm(a_ - b_) <= 1e-4 * np.linalg.norm(b_)


def test_mg_constant_rhs_from_zero_guess(orc):
    """The adjoint of loss = sum(alpha) solves A lambda = 1/2 from lambda = 0.
    lambda reaches ~190 there, so the first 50 iterations carry it all in the
    FP32 increment and the first true residual is ~100x the recurrence's; the
    solver must restart its direction there instead of stalling near 1e-4
    (which it did, hitting max_iters)."""
    torch = torch_cuda()
    from gpumatting_b200 import api

    W, H = 96, 64
    img, sc = edge_image(W, H)
    st = api.LevinStore(W, H, "fp16").assemble(torch.from_numpy(img).cuda(), torch.from_numpy(sc).cuda(), eps=1e-5,
                                               gamma_value=100.0)
    rhs = torch.full((H, W), 0.5, device="cuda")
    lam = torch.zeros((H, W), device="cuda")
    res = st.solve_rhs(rhs, lam, "mg", rtol=1e-6, max_iters=300)
    assert res.status == 0 and res.rel_residual <= 1e-6 and res.iters <= 100, res
    # FP64 residual of the returned FP32 lambda: its rounding alone leaves ~3e-5
    g = np.where(sc != 128, 100.0, 0.0).ravel()
    rel, _ = _true_relres(orc, st, g, np.full(W * H, 0.5), lam.double().cpu().numpy().ravel())
    assert rel <= 1e-4, rel
    assert float(lam.max()) > 100.0  # the large solution this case is about
    # and the adjoint through the same solve reports convergence
    alpha = torch.full((H, W), 0.5, device="cuda")
    assert st.solve(alpha, "mg", rtol=1e-6).status == 0
    _, _, _, ra = st.adjoint(alpha, torch.full((H, W), 0.5, device="cuda"), "mg", rtol=1e-6, max_iters=300)
    assert ra.status == 0, ra


def test_mg_on_restricted_store_matches_fp64_elimination(orc):
    """Hard constraints (gm_levin_restrict) then MG-PCG to 1e-10: within 1e-4
    of the FP64 elimination of the known pixels."""
    from tests.test_gpu_restrict import _reduced_solution

    torch = torch_cuda()
    from gpumatting_b200 import api
    from gpumatting_b200.synth import make_problem

    W, H = 96, 64
    p = make_problem(W, H, 8)
    scr = torch.from_numpy(p.scribbles).cuda()
    st = api.LevinStore(W, H, "fp16").assemble(torch.from_numpy(p.image).cuda(), scr, eps=p.eps).restrict(scribbles=scr)
    alpha = torch.full((H, W), 0.5, device="cuda")
    r = st.solve(alpha, "mg", rtol=1e-10, max_iters=5000)
    assert r.status == 0 and r.rel_residual <= 1e-10, r
    x, known, s = _reduced_solution(orc, p, W, H)
    assert np.abs(alpha.double().cpu().numpy().ravel() - x).max() <= TOL


def test_mg_on_batch_store_view(orc):
    """A batch image's store view (planes inside the canvas, plane_stride set)
    solves with MG like a standalone store of the same image."""
    import ctypes as C

    torch = torch_cuda()
    from gpumatting_b200 import _lib as L
    from gpumatting_b200 import api
    from gpumatting_b200.synth import make_problem

    sizes = [(70, 41), (96, 64)]
    b = api.LevinBatch(sizes, "fp16")
    probs = [make_problem(w, h, k) for k, (w, h) in enumerate(sizes)]
    for k, q in enumerate(probs):
        b.assemble(k, torch.from_numpy(q.image).cuda(), torch.from_numpy(q.scribbles).cuda(), eps=q.eps)
    W, H = sizes[1]
    q = probs[1]
    view = b.store_view(1)
    alpha = torch.full((H, W), 0.5, device="cuda")
    prm = L.default_params(solver=L.GM_SOLVER_MG, rtol=1e-8, max_iters=2000)
    info = L.GmSolveInfo()
    rc = L.load().gm_levin_solve(C.byref(view), alpha.data_ptr(), C.byref(prm), C.byref(info),
                                 torch.cuda.current_stream().cuda_stream)
    assert rc == 0 and info.rel_residual <= 1e-8, info.as_dict()
    st = api.LevinStore(W, H, "fp16").assemble(torch.from_numpy(q.image).cuda(), torch.from_numpy(q.scribbles).cuda(),
                                               eps=q.eps)
    ref = torch.full((H, W), 0.5, device="cuda")
    rs = st.solve(ref, "mg", rtol=1e-8, max_iters=2000)
    assert rs.iters == info.iters
    assert np.abs(alpha.cpu().numpy() - ref.cpu().numpy()).max() <= 1e-6


def test_mg_many_matches_single_solves(orc):
    """gm_levin_solve_mg_many (images spread over concurrent streams) gives
    each image the same result as its own solve, call after call."""
    torch = torch_cuda()
    from gpumatting_b200 import api
    from gpumatting_b200.synth import make_problem

    sizes = [(96, 64), (70, 41), (160, 120), (37, 29), (200, 150), (64, 48), (33, 90), (128, 128), (50, 40),
             (75, 20)]
    stores, probs = [], []
    for k, (w, h) in enumerate(sizes):
        q = make_problem(w, h, 20 + k)
        probs.append(q)
        stores.append(api.LevinStore(w, h, "fp16").assemble(torch.from_numpy(q.image).cuda(),
                                                            torch.from_numpy(q.scribbles).cuda(), eps=q.eps))
    refs = []
    for st, (w, h) in zip(stores, sizes):
        a = torch.full((h, w), 0.5, device="cuda")
        r = st.solve(a, "mg", rtol=1e-6, max_iters=2000)
        assert r.status == 0, r
        refs.append((a.cpu().numpy(), r.iters))
    for rep in range(2):
        alphas = [torch.full((h, w), 0.5, device="cuda") for w, h in sizes]
        res = api.mg_solve_many(stores, alphas, rtol=1e-6, max_iters=2000)
        for r, a, (ref, it) in zip(res, alphas, refs):
            assert r.status == 0 and r.rel_residual <= 1e-6 and r.iters == it, r
            assert np.array_equal(a.cpu().numpy().view(np.uint32), ref.view(np.uint32))


def test_mg_many_rejects_mixed_precisions_and_empty(orc):
    torch = torch_cuda()
    from gpumatting_b200 import _lib as L
    from gpumatting_b200 import api
    from gpumatting_b200.synth import make_problem

    q = make_problem(64, 48, 3)
    img, scr = torch.from_numpy(q.image).cuda(), torch.from_numpy(q.scribbles).cuda()
    a16 = api.LevinStore(64, 48, "fp16").assemble(img, scr, eps=q.eps)
    a32 = api.LevinStore(64, 48, "fp32").assemble(img, scr, eps=q.eps)
    alphas = [torch.full((48, 64), 0.5, device="cuda") for _ in range(2)]
    with pytest.raises(L.GmError) as e:
        api.mg_solve_many([a16, a32], alphas)
    assert e.value.status == L.GM_ERR_INVALID
    assert api.mg_solve_many([], []) == []


def test_mg_breakdown_status(orc):
    """A non-finite value in the operator ends the solve with GM_ERR_BREAKDOWN
    (no hang, the context stays usable)."""
    torch = torch_cuda()
    from gpumatting_b200 import _lib as L

    W, H = 64, 48
    st, p, w, g, b = _store(orc, W, H, "fp16")
    st.planes("gamma")[10, 10] = float("nan")
    torch.cuda.synchronize()
    alpha = torch.full((H, W), 0.5, device="cuda")
    with pytest.raises(L.GmError) as e:
        st.solve(alpha, "mg", rtol=1e-6)
    assert e.value.status == L.GM_ERR_BREAKDOWN
    st2, p2, w2, g2, b2 = _store(orc, W, H, "fp16", seed=3)
    alpha.fill_(0.5)
    r = st2.solve(alpha, "mg", rtol=1e-6)
    assert r.status == 0 and r.rel_residual <= 1e-6


_HOST_LOOP_SCRIPT = r"""
import sys, numpy as np, torch
sys.path.insert(0, sys.argv[1])
from gpumatting_b200 import api
from gpumatting_b200.synth import make_problem
q = make_problem(160, 120, 4)
st = api.LevinStore(160, 120, "fp16").assemble(torch.from_numpy(q.image).cuda(), torch.from_numpy(q.scribbles).cuda(),
                                               eps=q.eps)
a = torch.full((120, 160), 0.5, device="cuda")
r = st.solve(a, "mg", rtol=1e-6, max_iters=2000)
np.save(sys.argv[2], a.cpu().numpy())
print(r.iters, r.status)
"""


def test_mg_host_loop_matches_graph(orc, tmp_path):
    """GM_MG_GRAPH=0 (the same kernels launched one by one, the done flag
    read every 4 iterations) gives the graph path's result bit for bit."""
    import os
    import subprocess
    import sys

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    outs = {}
    for mode in ("1", "0"):
        path = str(tmp_path / f"alpha_{mode}.npy")
        env = dict(os.environ, GM_MG_GRAPH=mode)
        res = subprocess.run([sys.executable, "-c", _HOST_LOOP_SCRIPT, root, path], env=env, capture_output=True,
                             text=True, timeout=300)
        assert res.returncode == 0, res.stderr[-2000:]
        iters, status = res.stdout.split()[-2:]
        assert status == "0"
        outs[mode] = (int(iters), np.load(path))
    assert outs["0"][0] == outs["1"][0]
    assert np.array_equal(outs["0"][1].view(np.uint32), outs["1"][1].view(np.uint32))


def test_batch_solve_with_mg(orc):
    """gm_batch_solve with GM_SOLVER_MG gives every image of the canvas its own
    one-graph MG solve (concurrent streams): each result matches, bit for bit
    and in iterations, a solve of that image's store view alone."""
    import ctypes as C

    torch = torch_cuda()
    from gpumatting_b200 import _lib as L
    from gpumatting_b200 import api
    from gpumatting_b200.synth import make_problem

    sizes = [(70, 41), (96, 64), (33, 90)]
    b = api.LevinBatch(sizes, "fp16")
    for k, (w, h) in enumerate(sizes):
        q = make_problem(w, h, 40 + k)
        b.assemble(k, torch.from_numpy(q.image).cuda(), torch.from_numpy(q.scribbles).cuda(), eps=q.eps)
    outs = [torch.full((h, w), 0.5, device="cuda") for w, h in sizes]
    res = b.solve(outs, "mg", rtol=1e-6, max_iters=2000)
    prm = L.default_params(solver=L.GM_SOLVER_MG, rtol=1e-6, max_iters=2000)
    for k, (w, h) in enumerate(sizes):
        assert res[k].status == 0 and res[k].rel_residual <= 1e-6, res[k]
        view = b.store_view(k)
        a = torch.full((h, w), 0.5, device="cuda")
        info = L.GmSolveInfo()
        rc = L.load().gm_levin_solve(C.byref(view), a.data_ptr(), C.byref(prm), C.byref(info),
                                     torch.cuda.current_stream().cuda_stream)
        assert rc == 0 and info.iters == res[k].iters, (info.as_dict(), res[k])
        assert np.array_equal(a.cpu().numpy().view(np.uint32), outs[k].cpu().numpy().view(np.uint32))
