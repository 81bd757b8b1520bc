"""Laplacian assembly on the GPU: the reference-arithmetic kernel is
bit-identical to the reference's hostLevinLaplacian (golden fixtures), the
FP64 kernel matches the FP64 oracle to one rounding."""
import numpy as np
import pytest

from conftest import golden_cases, load_golden
from gpu_util import bands25_f32, oracle_problem, torch_cuda
from gpumatting_b200.synth import make_problem

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("case", golden_cases())
def test_reference_arithmetic_bit_exact(case):
    torch = torch_cuda()
    from gpumatting_b200 import api

    g = load_golden(case)
    im = torch.from_numpy(g["im4"]).cuda()
    sc = torch.from_numpy(g["scribbles"]).cuda()
    a, b = api.levin_bands25(im, sc, eps=float(g["lam"]), gamma_value=1.0, arithmetic="reference")
    assert np.array_equal(a.cpu().numpy().view(np.uint32), g["a"].view(np.uint32))
    assert np.array_equal(b.cpu().numpy().view(np.uint32), g["b"].view(np.uint32))


@pytest.mark.parametrize("case", ["s37x29", "data05", "s3x3"])
def test_hostLevinLaplacian_dropin(case):
    torch_cuda()
    from gpumatting_b200 import api

    g = load_golden(case)
    H, W = g["scribbles"].shape
    a = np.zeros((25, W * H), np.float32)
    b = np.zeros(W * H, np.float32)
    api.hostLevinLaplacian(a, b, float(g["lam"]), g["im4"], g["scribbles"], W, H)
    assert np.array_equal(a.view(np.uint32), g["a"].view(np.uint32))
    assert np.array_equal(b, g["b"])


def _row_diag(w, g, W, H):
    """gamma + sum over the 24 stencil neighbours of the stored affinities."""
    d = g.reshape(H, W).copy()
    wp = w.reshape(12, H, W)
    for k in range(1, 13):
        dv = (k + 2) // 5
        du = k - 5 * dv
        d += wp[k - 1]
        # lower neighbour (u - du, v - dv) holds w_k for the pair
        sh = np.zeros((H, W))
        v0, u0 = dv, max(0, du)
        u1 = min(W, W + du)
        sh[v0:, u0:u1] = wp[k - 1][: H - dv, u0 - du:u1 - du]
        d += sh
    return d.ravel()


def _ulp_close(x, ref, dtype, ulps=1):
    r = ref.astype(dtype).astype(np.float64)
    x = x.astype(np.float64)
    sp = np.spacing(np.abs(r).astype(dtype)).astype(np.float64)
    return np.all(np.abs(x - r) <= ulps * sp + 1e-30)


@pytest.mark.parametrize("W,H,prec,fmt", [(64, 48, "fp16", "rgb8"), (37, 29, "bf16", "rgb8"),
                                          (101, 7, "fp32", "rgba"), (5, 40, "fp16", "rgba")])
def test_fp64_assembly_matches_oracle(orc, W, H, prec, fmt):
    torch = torch_cuda()
    from gpumatting_b200 import api

    p, w, g, b = oracle_problem(orc, W, H, seed=9)
    img = torch.from_numpy(p.image).cuda() if fmt == "rgb8" else torch.from_numpy(
        np.concatenate([p.image.astype(np.float64) / 255.0, np.ones((H, W, 1))], axis=2).astype(np.float32)).cuda()
    if fmt == "rgba":  # the float image is the reference (rounded) one
        w = orc.levin_sym64(img.cpu().numpy()[..., :3].astype(np.float64), p.eps)
    sc = torch.from_numpy(p.scribbles).cuda()
    st = api.LevinStore(W, H, prec)
    Lm = api.DeviceBandedMatrix(torch.zeros((25, W * H), device="cuda"), torch.tensor(orc.levin_offsets(W)).cuda(),
                                W * H)
    b25 = torch.zeros(W * H, device="cuda")
    st.assemble(img, sc, eps=p.eps, gamma_value=100.0, bands25=Lm, b25=b25)
    torch.cuda.synchronize()
    w32 = st.planes("w32")[:, :, :W].reshape(12, -1).cpu().numpy()
    assert _ulp_close(w32, w, np.float32)
    wl = st.planes("w")[:, :, :W].reshape(12, -1).float().cpu().numpy()
    dt = {"fp16": np.float16, "fp32": np.float32}.get(prec)
    if dt is not None:
        assert _ulp_close(wl, w, dt)
    else:  # bf16: compare against the FP32 rounding at bf16 spacing
        assert np.all(np.abs(wl - w) <= np.abs(w) * 2.0 ** -8 + 1e-30)
    assert np.array_equal(st.planes("gamma")[:, :W].cpu().numpy().ravel(), g.astype(np.float32))
    # diagonal planes: gamma + row sum of exactly the rounded weights
    for dname, wp in (("d32", w32), ("d", wl)):
        exp = _row_diag(wp.astype(np.float64), g, W, H).astype(np.float32)
        got = st.planes(dname)[:, :W].cpu().numpy().ravel()
        assert np.all(np.abs(got.astype(np.float64) - exp) <= np.spacing(np.abs(exp)) + 1e-30), dname
    assert np.array_equal(st.planes("b")[:, :W].cpu().numpy().ravel(), b.astype(np.float32))
    a25 = Lm.a.cpu().numpy()
    ref = bands25_f32(orc, w, g, W, H)
    assert np.abs(a25 - ref).max() <= 2e-6 * np.abs(ref).max()
    assert np.array_equal(b25.cpu().numpy(), b.astype(np.float32))


def test_assembly_per_pixel_gamma_maps(orc):
    torch = torch_cuda()
    from gpumatting_b200 import api

    W, H = 33, 21
    p = make_problem(W, H, 12)
    rng = np.random.default_rng(3)
    gam = rng.uniform(0, 50, size=(H, W)).astype(np.float32)
    s = rng.uniform(0, 1, size=(H, W)).astype(np.float32)
    st = api.LevinStore(W, H, "fp16")
    st.assemble(torch.from_numpy(p.image).cuda(), None, eps=1e-4, gamma_map=torch.from_numpy(gam).cuda(),
                s_map=torch.from_numpy(s).cuda())
    torch.cuda.synchronize()
    assert np.array_equal(st.planes("gamma")[:, :W].cpu().numpy(), gam)
    assert np.array_equal(st.planes("b")[:, :W].cpu().numpy(), gam * s)
