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
