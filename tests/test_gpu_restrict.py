"""Restriction to the unknown pixels (gm_levin_restrict) against an FP64
elimination of the known pixels from the oracle's Laplacian.

With L the Levin Laplacian, U the unknown and K the known pixels, the
restricted problem is L_UU x_U = -L_UK s_K with x_K = s_K.  The GPU store
after restriction, solved to rel-res 1e-10, must match the direct FP64
solution within 1e-4, hold the known pixels at their targets (their rows
decouple: from alpha = 0.5 they converge with the rest, to 1e-9 here), and
its planes must carry no coupling that touches a known pixel."""
import numpy as np
import pytest
import scipy.sparse as sp
import scipy.sparse.linalg as spl

from gpumatting_b200 import api
from gpumatting_b200.synth import make_problem
from tests.gpu_util import torch_cuda

pytestmark = pytest.mark.gpu


def _reduced_solution(orc, p, W, H):
    w = orc.levin_sym64(p.image.astype(np.float64) / 255.0, p.eps)
    N = W * H
    a = orc.sym_to_bands64(w, np.zeros(N), W, H)  # the Laplacian L
    offs = orc.levin_offsets(W)
    rows, cols, vals = [], [], []
    for j in range(25):
        i = np.arange(N)
        k = i + offs[j]
        m = (k >= 0) & (k < N) & (a[j] != 0)
        rows.append(i[m]), cols.append(k[m]), vals.append(a[j][m])
    Lm = sp.csr_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))), shape=(N, N))
    known = (p.scribbles.ravel() != 128)
    s = (p.scribbles.ravel() == 255).astype(np.float64)
    U, K = np.where(~known)[0], np.where(known)[0]
    x = s.copy()
    x[U] = spl.spsolve(Lm[U][:, U].tocsc(), -(Lm[U][:, K] @ s[K]))
    return x, known, s


@pytest.mark.parametrize("prec", ["fp32", "fp16"])
def test_restricted_solve_matches_fp64_elimination(orc, prec):
    torch = torch_cuda()
    W, H = 80, 60
    p = make_problem(W, H, 7)
    scr = torch.from_numpy(p.scribbles).cuda()
    st = api.LevinStore(W, H, prec).assemble(torch.from_numpy(p.image).cuda(), scr, eps=p.eps, gamma_value=100.0)
    st.restrict(scribbles=scr)
    alpha = torch.full((H, W), 0.5, device="cuda")
    r = st.solve(alpha, "cg", rtol=1e-10, max_iters=20000)
    assert r.status == 0 and r.rel_residual <= 1e-10, r
    x, known, s = _reduced_solution(orc, p, W, H)
    got = alpha.double().cpu().numpy().ravel()
    assert np.abs(got[known] - s[known]).max() <= 1e-9
    assert np.abs(got - x).max() <= 1e-4
    # no coupling touches a known pixel
    w32 = st.planes("w32")[:, :, :W].cpu().numpy().reshape(12, -1)
    kn = known.reshape(H, W)
    for k in range(1, 13):
        dv = (k + 2) // 5
        du = k - 5 * dv
        for v in range(H):
            for u in range(W):
                uj, vj = u + du, v + dv
                if 0 <= uj < W and vj < H and (kn[v, u] or kn[vj, uj]):
                    assert w32[k - 1, v * W + u] == 0.0


def test_restricted_pcg_and_batch_view(orc):
    """PCG on a restricted store, and restriction of an image inside a batch."""
    torch = torch_cuda()
    W, H = 96, 64
    p = make_problem(W, H, 8)
    scr = torch.from_numpy(p.scribbles).cuda()
    img = torch.from_numpy(p.image).cuda()
    x, known, s = _reduced_solution(orc, p, W, H)
    st = api.LevinStore(W, H, "fp16").assemble(img, scr, eps=p.eps).restrict(scribbles=scr)
    alpha = torch.full((H, W), 0.5, device="cuda")
    r = st.solve(alpha, "pcg", rtol=1e-10, max_iters=20000)
    assert r.status == 0, r
    assert np.abs(alpha.double().cpu().numpy().ravel() - x).max() <= 1e-4
    b = api.LevinBatch([(W, H), (50, 40)], "fp16")
    b.assemble(0, img, scr, eps=p.eps)
    q = make_problem(50, 40, 9)
    b.assemble(1, torch.from_numpy(q.image).cuda(), torch.from_numpy(q.scribbles).cuda(), eps=q.eps)
    b.restrict(0, scribbles=scr)
    outs = [torch.full((H, W), 0.5, device="cuda"), torch.full((40, 50), 0.5, device="cuda")]
    res = b.solve(outs, "cg", rtol=1e-10, max_iters=20000, ctas_per_sm=3)
    assert all(r.status == 0 for r in res), res
    assert np.abs(outs[0].double().cpu().numpy().ravel() - x).max() <= 1e-4
