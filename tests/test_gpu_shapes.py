"""Launch shapes of the fused solver (gm_solve_params.strip_width and
ctas_per_sm): 192-column strips with shallow rings at three CTAs per SM or
deep rings at two, and 128-column strips at four.  Every shape runs the same
algorithm, so every shape must solve to the same true FP64 residual as the
oracle operator measures, in about the same iterations, follow the FP64
oracle's trajectory at fixed iteration counts, and repeat its own bits; the
batched solver's autotuner times each shape as a candidate."""
import numpy as np
import pytest

from gpu_util import oracle_problem, torch_cuda

pytestmark = pytest.mark.gpu

# (strip_width, ctas_per_sm)
SHAPES = [(0, 3), (0, 2), (128, 0)]
IDS = ["s192c3", "s192c2", "s128"]


def _store(orc, W, H, prec, seed=0):
    torch = torch_cuda()
    from gpumatting_b200 import api

    p, w, g, b = oracle_problem(orc, W, H, seed)
    st = api.LevinStore(W, H, prec).assemble(torch.from_numpy(p.image).cuda(), torch.from_numpy(p.scribbles).cuda(),
                                            eps=p.eps, gamma_value=100.0)
    return st, p, w, g, b


def _relres(orc, st, g, b, x):
    w32 = st.planes("w32")[:, :, :st.W].reshape(12, -1).double().cpu().numpy()
    op = orc.Operator(W=st.W, H=st.H, w=w32, gamma=g)
    return np.linalg.norm(b - op.apply(x)) / np.linalg.norm(b)


def _kw(shape):
    sw, cps = shape
    return dict(strip_width=sw, ctas_per_sm=cps)


@pytest.mark.parametrize("prec", ["fp16", "bf16"])
@pytest.mark.parametrize("solver", ["cg", "pcg"])
@pytest.mark.parametrize("shape", SHAPES, ids=IDS)
def test_shape_solves_to_rtol(orc, shape, solver, prec):
    torch = torch_cuda()
    W, H = 700, 433
    st, p, w, g, b = _store(orc, W, H, prec)
    alpha = torch.full((H, W), 0.5, device="cuda")
    base = st.solve(alpha, solver, rtol=1e-6, max_iters=5000, **_kw(SHAPES[0]))
    alpha.fill_(0.5)
    res = st.solve(alpha, solver, rtol=1e-6, max_iters=5000, **_kw(shape))
    assert res.status == 0 and res.rel_residual <= 1e-6, res
    assert _relres(orc, st, g, b, alpha.double().cpu().numpy().ravel()) <= 1.05e-6
    assert abs(res.iters - base.iters) <= 0.05 * base.iters + 3, (res.iters, base.iters)


@pytest.mark.parametrize("shape", SHAPES[1:], ids=IDS[1:])
def test_shape_matches_the_default_at_fixed_iterations(orc, shape):
    """GD and Jacobi on an FP16 store for fixed counts: the iterate agrees
    with the default shape's to FP32 rounding (the sweeps are elementwise in
    the iterate; only the FP64 sums are grouped differently)."""
    torch = torch_cuda()
    W, H = 333, 211
    st, p, w, g, b = _store(orc, W, H, "fp16", seed=4)
    outs = {}
    for sh in (SHAPES[0], shape):
        for solver in ("gd", "jacobi"):
            alpha = torch.full((H, W), 0.5, device="cuda")
            st.solve(alpha, solver, rtol=0.0, max_iters=30, **_kw(sh))
            outs[sh, solver] = alpha.double().cpu().numpy()
    for solver in ("gd", "jacobi"):
        assert np.abs(outs[shape, solver] - outs[SHAPES[0], solver]).max() <= 1e-5


def test_narrow_strips_follow_the_oracle_on_an_fp32_planes_solve(orc):
    """128-column strips exist for the 2-byte stores; on an FP32 store the
    request is refused with GM_ERR_UNSUPPORTED, and the default shape runs."""
    torch = torch_cuda()
    from gpumatting_b200 import _lib as L

    W, H = 120, 90
    st, p, w, g, b = _store(orc, W, H, "fp32", seed=3)
    alpha = torch.full((H, W), 0.5, device="cuda")
    with pytest.raises(L.GmError) as e:
        st.solve(alpha, "cg", rtol=0.0, max_iters=10, strip_width=128)
    assert e.value.status == L.GM_ERR_UNSUPPORTED
    with pytest.raises(L.GmError):
        st.solve(alpha, "cg", rtol=0.0, max_iters=10, strip_width=100)
    w32 = st.planes("w32")[:, :, :W].reshape(12, -1).double().cpu().numpy()
    op = orc.Operator(W=W, H=H, w=w32, gamma=g)
    alpha.fill_(0.5)
    st.solve(alpha, "cg", rtol=0.0, max_iters=40, strip_width=192)
    ref, _, _ = op.cg(b, np.full(W * H, 0.5), 0.0, 40, 0)
    assert np.abs(alpha.double().cpu().numpy().ravel() - ref).max() <= 1e-4


def test_narrow_strips_deterministic_and_small_images(orc):
    torch = torch_cuda()
    for W, H in ((300, 200), (129, 7), (8, 2), (3, 3), (1, 40)):
        st, p, w, g, b = _store(orc, W, H, "fp16")
        outs = []
        for _ in range(2):
            alpha = torch.full((H, W), 0.5, device="cuda")
            res = st.solve(alpha, "cg", rtol=1e-6, max_iters=3000, strip_width=128)
            outs.append(alpha.cpu().numpy())
            assert res.status == 0 and res.rel_residual <= 1e-6, (W, H, res)
        assert np.array_equal(outs[0].view(np.uint32), outs[1].view(np.uint32)), (W, H)
        assert _relres(orc, st, g, b, outs[0].astype(np.float64).ravel()) <= 1.05e-6, (W, H)


def test_batch_candidates_each_solve_and_repeat(orc):
    """Every launch shape the batch autotuner may pick (strip width x CTAs per
    SM x row multiplier) solves every image of an uneven batch to rtol, and
    replays bit for bit.  Across shapes the FP64 sums are grouped by
    different units, so their bits differ within rounding; the iterations
    agree within a few percent."""
    torch = torch_cuda()
    from gpumatting_b200 import api
    from gpumatting_b200.synth import make_problem

    sizes = [(300, 211), (129, 400), (64, 64), (517, 130)]
    probs = [make_problem(w, h, k) for k, (w, h) in enumerate(sizes)]
    batch = api.LevinBatch(sizes, "fp16")
    for k, pk in enumerate(probs):
        batch.assemble(k, torch.from_numpy(pk.image).cuda(), torch.from_numpy(pk.scribbles).cuda(), eps=pk.eps)
    its = {}
    for sw, cps in ((192, 3), (192, 2), (128, 4)):
        outs = []
        for _ in range(2):
            alphas = [torch.full((h, w), 0.5, device="cuda") for w, h in sizes]
            res = batch.solve(alphas, "cg", rtol=1e-6, strip_width=sw, ctas_per_sm=cps)
            assert all(r.status == 0 and r.rel_residual <= 1e-6 for r in res), (sw, cps, res)
            outs.append([a.cpu().numpy() for a in alphas])
        for a, b_ in zip(*outs):
            assert np.array_equal(a.view(np.uint32), b_.view(np.uint32)), (sw, cps)
        its[sw, cps] = [r.iters for r in res]
        for k, pk in enumerate(probs):
            w, h = sizes[k]
            wk = orc.levin_sym64(pk.image.astype(np.float64) / 255.0, pk.eps)
            op = orc.Operator(W=w, H=h, w=wk, gamma=pk.gamma.ravel().astype(np.float64))
            bk = (pk.gamma * pk.s).ravel().astype(np.float64)
            x = outs[0][k].astype(np.float64).ravel()
            assert np.linalg.norm(bk - op.apply(x)) / np.linalg.norm(bk) <= 2e-6, (sw, cps, k)
    base = its[192, 3]
    for key, v in its.items():
        assert all(abs(a - b_) <= 0.05 * b_ + 3 for a, b_ in zip(v, base)), (key, v, base)
    info = batch.tune(iters=10)
    assert info["strip_width"] in (128, 192) and info["ring_cfg"] in (0, 1, 2)
