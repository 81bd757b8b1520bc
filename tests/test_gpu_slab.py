"""The GPU data plane of the row-slab split (gpumatting_b200/slab.py,
LevinSlab): every slab's operator gives, for its own rows, exactly the rows
of the whole image's operator (band planes and matrix products bit for
bit), and the slab CG over several slabs of one image solves the whole
system to a true FP64 relative residual of 1e-6.  The slabs run in one
process on one GPU here, with their halo rows copied on the device; across
GPUs the same code moves them with NCCL send/recv."""
import numpy as np
import pytest

from gpu_util import torch_cuda

pytestmark = pytest.mark.gpu


def _setup(W, H, seed=0):
    torch = torch_cuda()
    from gpumatting_b200 import api
    from gpumatting_b200.synth import make_problem

    p = make_problem(W, H, seed)
    img = torch.from_numpy(p.image).cuda()
    scr = torch.from_numpy(p.scribbles).cuda()
    full = api.LevinStore(W, H, "fp32").assemble(img, scr, eps=p.eps, gamma_value=100.0)
    return p, img, scr, full


@pytest.mark.parametrize("nslabs", [2, 3, 7])
def test_slab_operator_rows_are_the_whole_image_rows(nslabs):
    torch = torch_cuda()
    from gpumatting_b200 import slab as S

    W, H = 300, 97
    p, img, scr, full = _setup(W, H)
    x = torch.rand((H, W + 4), device="cuda")[:, :W]
    y = full.apply(x, torch.empty((H, W + 4), device="cuda")[:, :W], true_op=True)
    w32 = full.planes("w32")
    for k in range(nslabs):
        r0, r1 = S.slab_bounds(H, nslabs, k)
        sl = S.LevinSlab(img, scr, p.eps, 100.0, r0, r1)
        lo = sl.skip + sl.above
        assert torch.equal(sl.store.planes("w32")[:, lo:lo + sl.R, :W], w32[:, r0:r1, :W]), k
        ys = sl.apply(x[r0 - sl.above:r1 + sl.below])
        assert torch.equal(ys[sl.above:sl.above + sl.R], y[r0:r1]), k
        assert torch.equal(sl.rhs(), full.planes("b")[r0:r1, :W]), k


def test_slab_cg_solves_the_whole_image(orc):
    torch = torch_cuda()
    from gpumatting_b200 import slab as S

    W, H = 480, 270
    p, img, scr, full = _setup(W, H, seed=1)
    nslabs = 3
    slabs = [S.LevinSlab(img, scr, p.eps, 100.0, *S.slab_bounds(H, nslabs, k)) for k in range(nslabs)]
    xs = [torch.full((s.R, W), 0.5, device="cuda") for s in slabs]
    bs = [s.rhs() for s in slabs]
    res = S.slab_cg(slabs, S.SlabComm(nslabs, 0, nslabs), xs, bs, rtol=1e-6, max_iters=5000)
    assert res.status == 0 and res.rel_residual <= 1e-6, res
    x = torch.cat(xs).double().cpu().numpy().ravel()
    w32 = full.planes("w32")[:, :, :W].reshape(12, -1).double().cpu().numpy()
    g = full.planes("gamma")[:, :W].double().cpu().numpy().ravel()
    b = full.planes("b")[:, :W].double().cpu().numpy().ravel()
    op = orc.Operator(W=W, H=H, w=w32, gamma=g)
    assert np.linalg.norm(b - op.apply(x)) / np.linalg.norm(b) <= 1.05e-6
    # the same CG on one slab takes about as many iterations
    one = [S.LevinSlab(img, scr, p.eps, 100.0, 0, H)]
    x1 = [torch.full((H, W), 0.5, device="cuda")]
    r1 = S.slab_cg(one, S.SlabComm(1, 0, 1), x1, [one[0].rhs()], rtol=1e-6, max_iters=5000)
    assert r1.status == 0 and abs(r1.iters - res.iters) <= 0.05 * r1.iters + 3, (r1, res)


@pytest.mark.parametrize("W,rows,pitch", [(1, 1, 4), (301, 37, 304), (1920, 540, 1920), (5, 2000, 8), (7, 0, 8)])
def test_cg_dots4_and_update_match_fp64(W, rows, pitch):
    """gm_cg_dots4 against FP64 sums (deterministic: bit-identical on a
    rerun) and gm_cg_update against the FP64 update, within FP32 rounding,
    on pitched row blocks."""
    torch = torch_cuda()
    from gpumatting_b200 import api

    g = torch.Generator(device="cuda").manual_seed(W * 1000 + rows)

    def blk():
        return torch.randn((rows, pitch), device="cuda", generator=g)[:, :W]

    x, r, p, q = blk(), blk(), blk(), blk()
    d = api.cg_dots4(r, p, q).cpu()
    assert torch.equal(d, api.cg_dots4(r, p, q).cpu())
    rd, pd, qd = r.double(), p.double(), q.double()
    pairs = [(rd, rd), (pd, qd), (rd, qd), (qd, qd)]
    for k, (u, v) in enumerate(pairs):
        ref = float((u * v).sum())
        scale = float((u * v).abs().sum())
        assert abs(float(d[k]) - ref) <= 1e-13 * scale + 1e-300, (k, float(d[k]), ref)
    alpha, beta = 0.375, -1.25  # exact in FP32
    x0, r0, p0 = x.double(), r.double(), p.double()
    api.cg_update(x, r, p, q, alpha, beta, update_p=True)
    torch.cuda.synchronize()
    ulp = 2.0 ** -23
    xe, re = x0 + alpha * p0, r0 - alpha * qd
    assert ((x.double() - xe).abs() <= ulp * (x0.abs() + abs(alpha) * p0.abs())).all()
    assert ((r.double() - re).abs() <= ulp * (r0.abs() + abs(alpha) * qd.abs())).all()
    pe = r.double() + beta * p0
    assert ((p.double() - pe).abs() <= ulp * (r.double().abs() + abs(beta) * p0.abs())).all()
    p1 = p.clone()
    api.cg_update(x, r, p, q, alpha, beta, update_p=False)
    assert torch.equal(p, p1)


def test_slab_cg_pitched_slabs():
    """An image width that is not a multiple of 4 gives slab buffers wider
    than W: the solve runs on the pitched views and still reaches 1e-6."""
    torch = torch_cuda()
    from gpumatting_b200 import slab as S

    W, H = 301, 90
    p, img, scr, full = _setup(W, H, seed=2)
    slabs = [S.LevinSlab(img, scr, p.eps, 100.0, *S.slab_bounds(H, 2, k)) for k in range(2)]
    assert not slabs[0].ext.is_contiguous()
    xs = [torch.full((s.R, W), 0.5, device="cuda") for s in slabs]
    res = S.slab_cg(slabs, S.SlabComm(2, 0, 2), xs, [s.rhs() for s in slabs], rtol=1e-6, max_iters=5000)
    assert res.status == 0 and res.rel_residual <= 1e-6, res


@pytest.mark.parametrize("sums,state", [
    ([4.0, 2.0, 1.0, 3.0], [-1.0, 0, 0, 7, 0, 50]),      # ordinary step
    ([4.0, 2.0, 1.0, 0.5], [3.0, 0, 0, 7, 0, 50]),       # next r.r 0 <= threshold: stop 1
    ([4.0, 2.0, 1.0, 3.0], [-1.0, 0, 0, 49, 0, 50]),     # replacement due: stop 1
    ([4.0, -2.0, 1.0, 3.0], [-1.0, 0, 0, 7, 0, 50]),     # p.q < 0: breakdown
    ([float("nan"), 2.0, 1.0, 3.0], [-1.0, 0, 0, 7, 0, 50]),
    ([4.0, 2.0, 1.0, 3.0], [-1.0, 9, 9, 7, 1, 50]),      # already stopped: nothing changes
])
def test_cg_scalars_match_the_host_rule(sums, state):
    """gm_cg_scalars against the same rule restated on the host (the CPU
    path of the slab CG), bit for bit."""
    torch = torch_cuda()
    from gpumatting_b200 import slab as S

    out = []
    for dev in ("cuda", "cpu"):
        coef = torch.full((3,), -7.0, dtype=torch.float64, device=dev)
        st = torch.tensor(state, dtype=torch.float64, device=dev)
        S._scalars(coef, st, torch.tensor(sums, dtype=torch.float64, device=dev))
        out.append((coef.cpu(), st.cpu()))
    (cg, sg), (cc, sc) = out
    assert torch.equal(cg, cc) and torch.allclose(sg, sc, equal_nan=True) and torch.equal(sg.isnan(), sc.isnan())
    assert torch.equal(sg[~sg.isnan()], sc[~sc.isnan()])


@pytest.mark.parametrize("chunk", [1, 10, 7])
def test_slab_cg_graph_replay_is_the_eager_loop(chunk):
    """The chunk captured as a CUDA graph gives bit-identical iterates and the
    same iteration count as the eager launches."""
    torch = torch_cuda()
    from gpumatting_b200 import slab as S

    W, H = 480, 270
    p, img, scr, full = _setup(W, H, seed=1)
    slabs = [S.LevinSlab(img, scr, p.eps, 100.0, *S.slab_bounds(H, 3, k)) for k in range(3)]
    bs = [s.rhs() for s in slabs]
    res, xs = [], []
    for graph in (False, True):
        x = [torch.full((s.R, W), 0.5, device="cuda") for s in slabs]
        res.append(S.slab_cg(slabs, S.SlabComm(3, 0, 3), x, bs, rtol=1e-6, max_iters=5000, chunk=chunk,
                             graph=graph))
        xs.append(torch.cat(x))
    assert res[0] == res[1] and res[0].status == 0, res
    assert torch.equal(xs[0], xs[1])
