"""Known-answer tests of the reference (tests/BandedMatrixTest.cu,
tests/VectorTest.cu) through libgpumat's C ABI."""
import numpy as np
import pytest

from gpu_util import torch_cuda

pytestmark = pytest.mark.gpu


def test_banded_matrix_kat():
    """BandedMatrixTest.cu:41-114: N = 1e6, bands {-10, 0, 10} of ones,
    zeroed out of range, x_i = i, x padded by 10; exact integers expected."""
    torch = torch_cuda()
    from gpumatting_b200 import api

    N = 1_000_000
    a = np.ones((3, N), np.float32)
    a[0, :10] = 0
    a[2, N - 10:] = 0
    Lm = api.DeviceBandedMatrix.from_host(a, [-10, 0, 10])
    x = api.PaddedVector(N, 10, np.arange(N, dtype=np.float32))
    y = torch.empty(N, dtype=torch.float32, device="cuda")
    api.bm_ax(y, Lm, x)
    i = np.arange(N)
    expect = np.where(i < 10, 10 + 2 * i, np.where(i < N - 10, 30 + 3 * (i - 10), 1999970 + 2 * (i - (N - 10))))
    assert np.array_equal(y.cpu().numpy(), expect.astype(np.float32))
    # b = A x - y and + y
    yy = torch.full((N,), 5.0, device="cuda")
    api.bm_axpy(y, Lm, x, yy, add=False)
    assert np.array_equal(y.cpu().numpy(), (expect - 5).astype(np.float32))


def test_inner_product_kat_and_determinism():
    """VectorTest.cu:20-68: sum of 1 * 2 over 1e6 elements is 2e6."""
    torch = torch_cuda()
    from gpumatting_b200 import api

    x = torch.ones(1_000_000, device="cuda")
    y = torch.full((1_000_000,), 2.0, device="cuda")
    assert api.inner_prod(x, y).item() == 2e6
    g = torch.Generator(device="cuda").manual_seed(0)
    u = torch.randn(3_000_001, device="cuda", generator=g)
    v = torch.randn(3_000_001, device="cuda", generator=g)
    r1 = api.inner_prod(u, v, f64=True).item()
    r2 = api.inner_prod(u, v, f64=True).item()
    assert r1 == r2
    ref = float(np.dot(u.cpu().numpy().astype(np.float64), v.cpu().numpy().astype(np.float64)))
    assert abs(r1 - ref) <= 1e-9 * abs(ref) + 1e-9
    z = torch.empty(0, device="cuda")
    assert api.inner_prod(z, z).item() == 0.0


def test_vector_ops():
    torch = torch_cuda()
    from gpumatting_b200 import _lib as L

    lib = L.load()
    n = 1000003
    x = torch.randn(n, device="cuda")
    y = torch.randn(n, device="cuda")
    out = torch.empty_like(x)
    s = torch.cuda.current_stream().cuda_stream
    L.check(lib.gm_vec_add(out.data_ptr(), x.data_ptr(), y.data_ptr(), n, s))
    assert torch.equal(out, x + y)
    L.check(lib.gm_vec_sub(out.data_ptr(), x.data_ptr(), y.data_ptr(), n, s))
    assert torch.equal(out, x - y)
    L.check(lib.gm_vec_scale_const(out.data_ptr(), x.data_ptr(), -1.0, n, s))
    assert torch.equal(out, -x)
    k = torch.tensor([0.25], device="cuda")
    L.check(lib.gm_vec_scale(out.data_ptr(), x.data_ptr(), k.data_ptr(), n, s))
    assert torch.equal(out, 0.25 * x)


def test_compute_error_gpu(orc):
    torch = torch_cuda()
    from gpumatting_b200 import api

    rng = np.random.default_rng(1)
    al = rng.uniform(-0.3, 1.3, size=(41, 37)).astype(np.float32)
    gt = rng.uniform(0, 1, size=(41, 37)).astype(np.float32)
    v = api.compute_error(torch.from_numpy(al).cuda(), torch.from_numpy(gt).cuda(), 37, 41)
    assert abs(v - orc.compute_error(al, gt)) <= 1e-12


@pytest.mark.parametrize("rows", [1_000_003, 4096 * 64])
def test_banded_product_four_row_path_matches_one_row_path(rows):
    """gm_bm_ax / gm_bm_axpy take four rows per thread with 128-bit band loads
    when the planes are 16-byte aligned with a pitch of a multiple of 4
    floats, and one row per thread otherwise; both sum every row in band
    order, so the results agree bit for bit (rows % 4 != 0 covers the tail)."""
    torch = torch_cuda()
    from gpumatting_b200 import api

    W = 4096
    offs = [du + W * dv for dv in range(-2, 3) for du in range(-2, 3)]
    rng = np.random.default_rng(rows)
    a = rng.standard_normal((25, rows)).astype(np.float32)
    pad = 2 * W + 2
    xh = rng.standard_normal(rows).astype(np.float32)
    x = api.PaddedVector(rows, pad, xh)
    yv = torch.from_numpy(rng.standard_normal(rows).astype(np.float32)).cuda()
    outs = []
    for apitch in (None, rows + 1):  # aligned pitch (four-row path), odd pitch (one-row path)
        Lm = api.DeviceBandedMatrix.from_host(a, offs, apitch)
        b = torch.empty(rows, dtype=torch.float32, device="cuda")
        api.bm_ax(b, Lm, x)
        c = torch.empty(rows, dtype=torch.float32, device="cuda")
        api.bm_axpy(c, Lm, x, yv, add=False)
        outs.append((b.cpu().numpy(), c.cpu().numpy()))
    for u, v in zip(*outs):
        assert np.array_equal(u.view(np.uint32), v.view(np.uint32))
    xs = np.zeros(rows + 2 * pad)
    xs[pad:pad + rows] = xh
    i = rng.integers(0, rows, 2000)
    ref = sum(a[j, i].astype(np.float64) * xs[pad + i + offs[j]] for j in range(25))
    assert np.abs(outs[0][0][i] - ref).max() <= 1e-4 * (1 + np.abs(ref).max())
