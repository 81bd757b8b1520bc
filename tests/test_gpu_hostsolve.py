"""The reference's CPU relaxations as GPU drop-ins (Solve.cpp:3-85), called
through the C ABI: gaussSeidel_host and jacobi_host must reproduce the
reference's iterates bit for bit -- against the fixture the reference itself
wrote (tests/golden/solve_host_s37x29.npz, from oracle/_ref) and against the
oracle's line-faithful restatement on other band patterns and sizes.  Also
the damped Jacobi step kernel (BandedMatrix.cu:61-98) on known answers."""
import numpy as np
import pytest

from conftest import load_golden
from gpu_util import bands25_f32, oracle_problem, torch_cuda

pytestmark = pytest.mark.gpu


def _padded(x0: np.ndarray, pad: int) -> np.ndarray:
    xp = np.zeros(x0.size + 2 * pad, np.float32)
    xp[pad:pad + x0.size] = x0
    return xp


def _fixture():
    g = load_golden("s37x29")
    s = load_golden("s37x29", "solve_host_")
    return g, s


def test_gauss_seidel_host_matches_the_reference_fixture_bitwise():
    torch_cuda()
    from gpumatting_b200 import api
    from oracle import oracle as O

    g, s = _fixture()
    H, W = g["scribbles"].shape
    offs = O.levin_offsets(W)
    pad = O.pad_for(W)
    xp = _padded(s["x0"], pad)
    api.gaussSeidel_host(xp, pad, g["a"], offs, g["b"], int(s["iters"]))
    got = xp[pad:pad + W * H]
    assert np.array_equal(got.view(np.uint32), s["gs"].view(np.uint32))
    assert not xp[:pad].any() and not xp[pad + W * H:].any()  # padding untouched


def test_jacobi_host_matches_the_reference_fixture_bitwise():
    torch_cuda()
    from gpumatting_b200 import api
    from oracle import oracle as O

    g, s = _fixture()
    H, W = g["scribbles"].shape
    offs = O.levin_offsets(W)
    pad = O.pad_for(W)
    xp = _padded(s["x0"], pad)
    api.jacobi_host(xp, pad, g["a"], offs, g["b"], int(s["iters"]), float(s["omega"]))
    assert np.array_equal(xp[pad:pad + W * H].view(np.uint32), s["jacobi"].view(np.uint32))


@pytest.mark.parametrize("iters", [1, 7, 30])
def test_host_relaxations_match_the_oracle_on_a_levin_system(orc, iters):
    """640x480 Levin system (FP32 bands of the FP64 assembly), odd and even
    sweep counts; the oracle restates Solve.cpp line by line (no FMA)."""
    torch_cuda()
    from gpumatting_b200 import api

    W, H = 640, 480
    p, w, gam, b = oracle_problem(orc, W, H, seed=1)
    a = bands25_f32(orc, w, gam, W, H)
    offs = orc.levin_offsets(W)
    x0 = np.full(W * H, 0.5, np.float32)
    b32 = b.astype(np.float32)
    pad = orc.pad_for(W)
    xp = _padded(x0, pad)
    api.gaussSeidel_host(xp, pad, a, offs, b32, iters)
    want = orc.gs_host(a, offs, b32, x0, iters)
    assert np.array_equal(xp[pad:pad + W * H].view(np.uint32), want.view(np.uint32))
    xp = _padded(x0, pad)
    api.jacobi_host(xp, pad, a, offs, b32, iters, 2.0 / 3.0)
    want = orc.jacobi_host(a, offs, b32, x0, iters, 2.0 / 3.0)
    assert np.array_equal(xp[pad:pad + W * H].view(np.uint32), want.view(np.uint32))


@pytest.mark.parametrize("offs", [[-1, 0, 1], [-9, -4, -1, 0, 2, 7, 30], [-300, -17, 0, 5, 64]])
def test_host_relaxations_accept_any_band_pattern(orc, offs):
    """Diagonally dominant random matrices with other patterns (zero where a
    band leaves the matrix, random zeros inside), against the oracle, bit
    for bit; Gauss-Seidel also converges to the direct solution."""
    torch_cuda()
    from gpumatting_b200 import api

    rng = np.random.default_rng(len(offs))
    n = 20_000
    offs = np.array(offs, np.int32)
    nb = offs.size
    a = (rng.random((nb, n)) - 0.5).astype(np.float32)
    a[rng.random((nb, n)) < 0.2] = 0.0
    for j, o in enumerate(offs):
        i = np.arange(n)
        a[j, (i + o < 0) | (i + o >= n)] = 0.0
    mid = nb // 2
    a[mid] = (np.abs(np.delete(a, mid, axis=0)).sum(axis=0) + 1.0).astype(np.float32)
    b = rng.standard_normal(n).astype(np.float32)
    x0 = np.zeros(n, np.float32)
    pad = int(np.abs(offs).max())
    for it in (1, 4, 25):
        xp = _padded(x0, pad)
        api.gaussSeidel_host(xp, pad, a, offs, b, it)
        want = orc.gs_host(a, offs, b, x0, it)
        assert np.array_equal(xp[pad:pad + n].view(np.uint32), want.view(np.uint32)), it
        xp = _padded(x0, pad)
        api.jacobi_host(xp, pad, a, offs, b, it, 0.7)
        want = orc.jacobi_host(a, offs, b, x0, it, 0.7)
        assert np.array_equal(xp[pad:pad + n].view(np.uint32), want.view(np.uint32)), it
    # the fixed point: after 25 sweeps the diagonally dominant system is solved
    import scipy.sparse as sp
    from scipy.sparse.linalg import spsolve

    rows, cols, vals = [], [], []
    for j, o in enumerate(offs):
        i = np.arange(n)
        m = (i + o >= 0) & (i + o < n)
        rows.append(i[m]); cols.append(i[m] + o); vals.append(a[j, m].astype(np.float64))
    A = sp.csr_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))), shape=(n, n))
    xs = spsolve(A.tocsc(), b.astype(np.float64))
    xp = _padded(x0, pad)
    api.gaussSeidel_host(xp, pad, a, offs, b, 60)
    assert np.abs(xp[pad:pad + n] - xs).max() <= 1e-4


def test_host_relaxations_reject_short_padding():
    torch_cuda()
    from gpumatting_b200 import _lib as L
    from gpumatting_b200 import api

    n = 100
    a = np.ones((3, n), np.float32)
    with pytest.raises(ValueError):
        api.jacobi_host(np.zeros(n + 2, np.float32), 1, a, [-5, 0, 5], np.ones(n, np.float32), 2)
    # through the C entry point: xpad below the reach is refused
    offs = np.array([-5, 0, 5], np.int32)
    m = L.BandedMatrix(a.ctypes.data, n, offs.ctypes.data, 3, n, n)
    x = np.zeros(n + 20, np.float32)
    b = np.ones(n, np.float32)
    import ctypes as C

    L.load().jacobi_host(x.ctypes.data + 40, C.byref(m), b.ctypes.data, 2, 2, 0.5)
    assert L.load().gm_last_status() == L.GM_ERR_INVALID


def test_jacobi_step_known_answers(orc):
    """gm_jacobi_step, xx = omega (x + (b - A x) / a_ii) + (1 - omega) x
    (BandedMatrix.cu:61-98), on the KAT pattern of BandedMatrixTest.cu:41-114
    ({-10, 0, 10}, ones off the diagonal) with a diagonal of 2, x_i = i mod
    97, b_i = i mod 13 and omega = 1/2: every intermediate is a small dyadic
    number, so the result is exact; then a random system against FP64."""
    torch = torch_cuda()
    from gpumatting_b200 import api

    N = 1_000_000
    a = np.ones((3, N), np.float32)
    a[0, :10] = 0
    a[2, N - 10:] = 0
    a[1] = 2.0
    i = np.arange(N)
    x = (i % 97).astype(np.float32)
    b = (i % 13).astype(np.float32)
    Lm = api.DeviceBandedMatrix.from_host(a, [-10, 0, 10])
    xv = api.PaddedVector(N, 10, x)
    xx = torch.empty(N, dtype=torch.float32, device="cuda")
    api.jacobi_step(xx, xv, Lm, torch.from_numpy(b).cuda(), 0.5)
    xpad = np.concatenate([np.zeros(10), x.astype(np.float64), np.zeros(10)])
    ax = a[0] * xpad[:-20] + a[1] * xpad[10:-10] + a[2] * xpad[20:]
    want = 0.5 * (x + (b - ax) / 2.0) + 0.5 * x
    assert np.array_equal(xx.cpu().numpy(), want.astype(np.float32))
    # random diagonally dominant system: FP32 kernel within a few ulps of FP64
    rng = np.random.default_rng(5)
    a = (rng.random((3, N)) - 0.5).astype(np.float32)
    a[0, :10] = 0
    a[2, N - 10:] = 0
    a[1] = 2.0 + rng.random(N).astype(np.float32)
    x = rng.standard_normal(N).astype(np.float32)
    b = rng.standard_normal(N).astype(np.float32)
    Lm = api.DeviceBandedMatrix.from_host(a, [-10, 0, 10])
    xv = api.PaddedVector(N, 10, x)
    api.jacobi_step(xx, xv, Lm, torch.from_numpy(b).cuda(), 2.0 / 3.0)
    xpad = np.concatenate([np.zeros(10), x.astype(np.float64), np.zeros(10)])
    a64 = a.astype(np.float64)
    ax = a64[0] * xpad[:-20] + a64[1] * xpad[10:-10] + a64[2] * xpad[20:]
    want = (2.0 / 3.0) * (x + (b - ax) / a64[1]) + (1.0 / 3.0) * x
    assert np.abs(xx.cpu().numpy() - want).max() <= 1e-5 * (1.0 + np.abs(want).max())
