"""Standalone SpMV (gm_levin_apply) against an FP64 restatement of the same
operator built from the store's own planes.

Iteration operator: y_i = d_i x_i - sum_j w_ij x_j over the store's planes of
its precision; true operator: y_i = gamma_i x_i + sum_j w32_ij (x_i - x_j)
(the oracle's orc_apply_sym64 on w32).  Both accumulate in FP32 on the GPU,
so the bound is a few FP32 ulps of sum |terms|.
"""
import numpy as np
import pytest

from gpumatting_b200 import api
from gpumatting_b200.synth import make_problem
from tests.gpu_util import torch_cuda

pytestmark = pytest.mark.gpu


def _sym_apply_lo(w, d, x, W, H):
    """y = d x - sum_k [w_k(i) x(i + o_k) + w_k(i - o_k) x(i - o_k)], FP64,
    and the sum of |terms| for the error bound."""
    y = d * x
    mag = np.abs(d * x)
    for k in range(1, 13):
        dv = (k + 2) // 5
        du = k - 5 * dv
        wk = w[k - 1]
        u0, u1 = max(0, -du), min(W, W - du)
        v1 = H - dv
        if u1 <= u0 or v1 <= 0:
            continue
        f = wk[:v1, u0:u1] * x[dv:dv + v1, u0 + du:u1 + du]   # w_k(i) x(i + o)
        y[:v1, u0:u1] -= f
        mag[:v1, u0:u1] += np.abs(f)
        b = wk[:v1, u0:u1] * x[:v1, u0:u1]                     # w_k(j) x(j) into row i = j + o
        y[dv:dv + v1, u0 + du:u1 + du] -= b
        mag[dv:dv + v1, u0 + du:u1 + du] += np.abs(b)
    return y, mag


@pytest.mark.parametrize("W,H,precision", [(37, 29, "fp16"), (300, 17, "bf16"), (1000, 515, "fp16"),
                                           (257, 130, "fp32"), (5, 3, "fp16"), (129, 1, "fp32")])
def test_apply_matches_fp64(orc, W, H, precision):
    torch = torch_cuda()
    p = make_problem(W, H, 3)
    st = api.LevinStore(W, H, precision).assemble(torch.from_numpy(p.image).cuda(),
                                                 torch.from_numpy(p.scribbles).cuda(), eps=p.eps)
    P4 = (W + 3) // 4 * 4
    g = torch.Generator(device="cuda").manual_seed(W * 1000 + H)
    xbuf = torch.rand((H, P4), device="cuda", generator=g) - 0.5
    x = xbuf[:, :W]
    ybuf = torch.full((H, P4 + 2), float("nan"), device="cuda")
    y = ybuf[:, :W]
    xn = x.cpu().double().numpy()
    for true_op in (False, True):
        st.apply(x, y, true_op=true_op)
        torch.cuda.synchronize()
        got = y.cpu().double().numpy()
        if true_op:
            w32 = st.planes("w32")[:, :, :W].cpu().double().numpy()
            gam = st.planes("gamma")[:, :W].cpu().double().numpy()
            ref = orc.Operator(W=W, H=H, w=w32.reshape(12, -1), gamma=gam).apply(xn.ravel()).reshape(H, W)
            _, mag = _sym_apply_lo(w32, gam, xn, W, H)
        else:
            w = st.planes("w")[:, :, :W].float().cpu().double().numpy()
            d = st.planes("d32" if precision == "fp32" else "d")[:, :W].cpu().double().numpy()
            ref, mag = _sym_apply_lo(w, d, xn, W, H)
        err = np.abs(got - ref)
        assert np.all(np.isfinite(got))
        assert np.all(err <= 4e-7 * (mag + 1e-30) * 8), (true_op, float((err / (mag + 1e-30)).max()))
        # columns past W and the row padding stay untouched
        assert torch.isnan(ybuf[:, W:]).all()
