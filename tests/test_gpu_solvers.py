"""Solver parity on the GPU: the reference-named drop-ins against the FP64
oracle at fixed iteration counts (trajectory tolerance 1e-4 max-abs), the
mixed-precision Levin solve against the FP64 solution, and the status paths
(timeout, breakdown, bad arguments)."""
import numpy as np
import pytest

from gpu_util import bands25_f32, oracle_problem, torch_cuda

from gpumatting_b200.synth import make_problem

pytestmark = pytest.mark.gpu
TOL = 1e-4  # max-abs alpha tolerance against the FP64 oracle


def _dropin_setup(orc, W, H, apitch=None, seed=1):
    torch = torch_cuda()
    from gpumatting_b200 import api

    p, w, g, b = oracle_problem(orc, W, H, seed)
    a = bands25_f32(orc, w, g, W, H)
    offs = orc.levin_offsets(W)
    Lm = api.DeviceBandedMatrix.from_host(a, offs, apitch)
    pad = api.levin_pad(W)
    x = api.PaddedVector(W * H, pad, np.full(W * H, 0.5, np.float32))
    bt = torch.tensor(b, dtype=torch.float32, device="cuda")
    op = orc.Operator(W=W, H=H, bands=a.astype(np.float64), offs=offs)
    return api, Lm, x, bt, b, op, pad


@pytest.mark.parametrize("W,H,apitch", [(64, 48, None), (37, 29, 1103), (200, 150, None)])
def test_cgSolve_dropin_vs_oracle(orc, W, H, apitch):
    api, Lm, x, bt, b, op, pad = _dropin_setup(orc, W, H, apitch)
    api.cgSolve(x, Lm, bt, pad, 60, 25)
    ref, _, _ = op.cg(b, np.full(W * H, 0.5), rtol=0.0, maxit=60, restart=25)
    got = x.data.cpu().numpy()
    assert np.abs(got - ref).max() <= TOL
    st = x.storage.cpu().numpy()
    assert not st[:pad].any() and not st[pad + W * H:].any()  # padding untouched


def test_gradSolve_dropin_vs_oracle(orc):
    W, H = 64, 48
    api, Lm, x, bt, b, op, pad = _dropin_setup(orc, W, H)
    api.gradSolve(x, Lm, bt, 30, pad)
    ref, _, _ = op.gd(b, np.full(W * H, 0.5), rtol=0.0, maxit=30)
    assert np.abs(x.data.cpu().numpy() - ref).max() <= TOL


@pytest.mark.parametrize("iters", [1, 30, 31])
def test_jacobi_dropin_vs_oracle(orc, iters):
    W, H = 64, 48
    api, Lm, x, bt, b, op, pad = _dropin_setup(orc, W, H)
    api.jacobi(x, Lm, bt, 2.0 / 3.0, pad, iters)
    ref, _, _ = op.jacobi(b, np.full(W * H, 0.5), omega=2.0 / 3.0, rtol=0.0, maxit=iters)
    assert np.abs(x.data.cpu().numpy() - ref).max() <= TOL


def test_generic_band_pattern_cg(orc):
    """A pattern that is not the Levin stencil runs the generic band path."""
    torch = torch_cuda()
    from gpumatting_b200 import api

    N = 20000
    a = np.zeros((3, N), np.float32)
    a[0, 1:] = -1.0
    a[1] = 2.5
    a[2, :-1] = -1.0
    Lm = api.DeviceBandedMatrix.from_host(a, [-1, 0, 1])
    rng = np.random.default_rng(0)
    b = rng.normal(size=N)
    x = api.PaddedVector(N, 32, np.zeros(N, np.float32))
    api.cgSolve(x, Lm, torch.tensor(b, dtype=torch.float32, device="cuda"), 32, 40, 0)
    op = orc.Operator(W=N, H=1, bands=a.astype(np.float64), offs=np.array([-1, 0, 1]))
    ref, _, _ = op.cg(b, np.zeros(N), rtol=0.0, maxit=40)
    assert np.abs(x.data.cpu().numpy() - ref).max() <= TOL * max(1.0, np.abs(ref).max())


def _store(orc, W, H, prec, seed=2):
    torch = torch_cuda()
    from gpumatting_b200 import api

    p, w, g, b = oracle_problem(orc, W, H, seed)
    st = api.LevinStore(W, H, prec).assemble(torch.from_numpy(p.image).cuda(), torch.from_numpy(p.scribbles).cuda(),
                                             eps=p.eps, gamma_value=100.0)
    return api, st, p, w, g, b


def _true_relres(orc, st, g, b, x):
    W, H = st.W, st.H
    w32 = st.planes("w32")[:, :, :W].reshape(12, -1).double().cpu().numpy()
    op = orc.Operator(W=W, H=H, w=w32, gamma=g)
    return np.linalg.norm(b - op.apply(x)) / np.linalg.norm(b)


@pytest.mark.parametrize("prec", ["fp16", "bf16", "fp32"])
def test_levin_solve_mixed_to_rtol(orc, prec):
    torch = torch_cuda()
    W, H = 160, 120
    api, st, p, w, g, b = _store(orc, W, H, prec)
    alpha = torch.full((H, W), 0.5, device="cuda")
    res = st.solve(alpha, "cg", rtol=1e-6, max_iters=5000)
    assert res.status == 0, res
    x = alpha.double().cpu().numpy().ravel()
    assert res.rel_residual <= 1e-6
    assert _true_relres(orc, st, g, b, x) <= 1.05e-6
    op = orc.Operator(W=W, H=H, w=w, gamma=g)
    _, it64, _ = op.cg(b, np.full(W * H, 0.5), rtol=1e-6, maxit=20000)
    assert res.iters <= 1.3 * it64 + 20, (res.iters, it64)


def test_levin_solve_accurate_vs_direct(orc):
    """rtol 1e-10: alpha within 1e-4 max-abs of the FP64 direct solve."""
    import scipy.sparse as sp
    import scipy.sparse.linalg as spla

    torch = torch_cuda()
    W, H = 64, 48
    api, st, p, w, g, b = _store(orc, W, H, "fp16", seed=5)
    a = orc.sym_to_bands64(w, g, W, H)
    offs = orc.levin_offsets(W)
    N = W * H
    rows, cols, vals = [], [], []
    for k in range(25):
        i = np.arange(N)
        j = i + offs[k]
        m = (j >= 0) & (j < N) & (a[k] != 0)
        rows.append(i[m]); cols.append(j[m]); vals.append(a[k][m])
    M = sp.csr_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))), shape=(N, N))
    xs = spla.spsolve(M.tocsc(), b)
    alpha = torch.full((H, W), 0.5, device="cuda")
    res = st.solve(alpha, "cg", rtol=1e-10, max_iters=50000)
    assert res.status == 0 and res.rel_residual <= 1e-10
    assert np.abs(alpha.double().cpu().numpy().ravel() - xs).max() <= TOL


@pytest.mark.parametrize("W,strip,solver", [(384, 192, "cg"), (384, 192, "pcg"), (256, 128, "cg"), (383, 192, "cg")])
def test_full_strip_widths_accurate_vs_direct(orc, W, strip, solver):
    """Widths that are a whole number of strips take the kernel's full-strip
    path (no per-lane column tests); both paths agree with the FP64 direct
    solve to 1e-4 at rel-res 1e-10."""
    import scipy.sparse as sp
    import scipy.sparse.linalg as spla

    torch = torch_cuda()
    H = 40
    api, st, p, w, g, b = _store(orc, W, H, "fp16", seed=7)
    a = orc.sym_to_bands64(w, g, W, H)
    offs = orc.levin_offsets(W)
    N = W * H
    rows, cols, vals = [], [], []
    for k in range(25):
        i = np.arange(N)
        j = i + offs[k]
        m = (j >= 0) & (j < N) & (a[k] != 0)
        rows.append(i[m]); cols.append(j[m]); vals.append(a[k][m])
    M = sp.csr_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))), shape=(N, N))
    xs = spla.spsolve(M.tocsc(), b)
    alpha = torch.full((H, W), 0.5, device="cuda")
    res = st.solve(alpha, solver, rtol=1e-10, max_iters=50000, strip_width=strip)
    assert res.status == 0 and res.rel_residual <= 1e-10, res
    assert np.abs(alpha.double().cpu().numpy().ravel() - xs).max() <= TOL


def test_levin_gd_and_jacobi_fixed_iterations(orc):
    torch = torch_cuda()
    W, H = 96, 64
    api, st, p, w, g, b = _store(orc, W, H, "fp32")
    w32 = st.planes("w32")[:, :, :W].reshape(12, -1).double().cpu().numpy()
    op = orc.Operator(W=W, H=H, w=w32, gamma=g)
    x0 = np.full(W * H, 0.5)
    alpha = torch.full((H, W), 0.5, device="cuda")
    st.solve(alpha, "gd", rtol=0.0, max_iters=25)
    ref, _, _ = op.gd(b, x0, maxit=25)
    assert np.abs(alpha.double().cpu().numpy().ravel() - ref).max() <= TOL
    alpha.fill_(0.5)
    res = st.solve(alpha, "jacobi", rtol=0.0, max_iters=25, omega=0.6)
    ref, _, _ = op.jacobi(b, x0, omega=0.6, maxit=25)
    assert res.iters == 25
    assert np.abs(alpha.double().cpu().numpy().ravel() - ref).max() <= TOL


def test_solve_is_deterministic(orc):
    torch = torch_cuda()
    W, H = 300, 200
    api, st, p, w, g, b = _store(orc, W, H, "fp16")
    outs = []
    for _ in range(2):
        alpha = torch.full((H, W), 0.5, device="cuda")
        st.solve(alpha, "cg", rtol=0.0, max_iters=300)
        outs.append(alpha.cpu().numpy())
    assert np.array_equal(outs[0].view(np.uint32), outs[1].view(np.uint32))


def test_timeout_status_and_recovery(orc):
    """A barrier waiting for an arrival that never comes must end with
    GM_ERR_TIMEOUT after the limit and leave the context usable."""
    torch = torch_cuda()
    from gpumatting_b200 import _lib as L

    W, H = 64, 48
    api, st, p, w, g, b = _store(orc, W, H, "fp16")
    alpha = torch.full((H, W), 0.5, device="cuda")
    p_ = L.default_params(rtol=1e-6, timeout_s=0.2, inject=1)
    info = L.GmSolveInfo()
    import ctypes as C

    rc = L.load().gm_levin_solve(C.byref(st.s), alpha.data_ptr(), C.byref(p_), C.byref(info),
                                 torch.cuda.current_stream().cuda_stream)
    assert rc == L.GM_ERR_TIMEOUT and info.status == L.GM_ERR_TIMEOUT and info.where == 1
    alpha.fill_(0.5)
    res = st.solve(alpha, "cg", rtol=1e-6)
    assert res.status == 0 and res.rel_residual <= 1e-6


def test_breakdown_status(orc):
    torch = torch_cuda()
    from gpumatting_b200 import _lib as L

    W, H = 64, 48
    api, st, p, w, g, b = _store(orc, W, H, "fp16")
    st.planes("gamma")[10, 10] = float("nan")
    torch.cuda.synchronize()
    alpha = torch.full((H, W), 0.5, device="cuda")
    with pytest.raises(L.GmError) as e:
        st.solve(alpha, "cg", rtol=1e-6)
    assert e.value.status == L.GM_ERR_BREAKDOWN


def test_bad_arguments():
    torch_cuda()
    from gpumatting_b200 import _lib as L
    from gpumatting_b200 import api

    with pytest.raises(L.GmError):
        api.LevinStore(0, 10)
    st = api.LevinStore(16, 16, "fp16")
    import torch

    alpha = torch.zeros((16, 16), device="cuda")
    with pytest.raises(L.GmError):
        st.solve(alpha, "cg", max_iters=-1)


def _pcg64(op, diag, b, x0, rtol, maxit=20000):
    """FP64 Jacobi-preconditioned CG (M = diag of the operator)."""
    x = x0.copy()
    r = b - op.apply(x)
    z = r / diag
    p = z.copy()
    rz = r @ z
    bn = np.linalg.norm(b)
    for it in range(maxit):
        if np.linalg.norm(r) <= rtol * bn:
            return x, it
        q = op.apply(p)
        al = rz / (p @ q)
        x += al * p
        r -= al * q
        z = r / diag
        rz2 = r @ z
        p = z + (rz2 / rz) * p
        rz = rz2
    return x, maxit


@pytest.mark.parametrize("prec", ["fp16", "bf16", "fp32"])
def test_levin_pcg_to_rtol(orc, prec):
    """Jacobi-preconditioned mixed CG: true FP64 residual at rtol, about as
    many iterations as FP64 Jacobi PCG, and fewer than plain CG."""
    torch = torch_cuda()
    W, H = 160, 120
    api, st, p, w, g, b = _store(orc, W, H, prec)
    alpha = torch.full((H, W), 0.5, device="cuda")
    res = st.solve(alpha, "pcg", rtol=1e-6, max_iters=5000)
    assert res.status == 0 and res.rel_residual <= 1e-6, res
    x = alpha.double().cpu().numpy().ravel()
    assert _true_relres(orc, st, g, b, x) <= 1.05e-6
    op = orc.Operator(W=W, H=H, w=w, gamma=g)
    diag = orc.sym_to_bands64(w, g, W, H)[12]
    _, it64 = _pcg64(op, diag, b, np.full(W * H, 0.5), 1e-6)
    assert res.iters <= 1.3 * it64 + 20, (res.iters, it64)
    alpha.fill_(0.5)
    res_cg = st.solve(alpha, "cg", rtol=1e-6, max_iters=5000)
    assert res.iters <= 0.85 * res_cg.iters, (res.iters, res_cg.iters)


def test_levin_pcg_accurate_and_deterministic(orc):
    torch = torch_cuda()
    W, H = 96, 64
    api, st, p, w, g, b = _store(orc, W, H, "fp16", seed=3)
    outs = []
    for _ in range(2):
        alpha = torch.full((H, W), 0.5, device="cuda")
        res = st.solve(alpha, "pcg", rtol=1e-10, max_iters=20000)
        assert res.status == 0 and res.rel_residual <= 1e-10, res
        outs.append(alpha.cpu().numpy())
    assert np.array_equal(outs[0].view(np.uint32), outs[1].view(np.uint32))
    w32 = st.planes("w32")[:, :, :W].reshape(12, -1).double().cpu().numpy()
    xs, _, _ = orc.Operator(W=W, H=H, w=w32, gamma=g).cg(b, np.full(W * H, 0.5), rtol=1e-13, maxit=100000)
    assert np.abs(outs[0].astype(np.float64).ravel() - xs).max() <= TOL


def test_pcg_rejected_on_25_band_store():
    torch = torch_cuda()
    from gpumatting_b200 import _lib as L
    from gpumatting_b200 import api

    p = make_problem(40, 30, 1)
    a, b = api.levin_bands25(torch.from_numpy(p.image).cuda(), torch.from_numpy(p.scribbles).cuda(), eps=p.eps)
    Lm = api.DeviceBandedMatrix(a, torch.tensor(api.levin_band_offsets(40), device="cuda"), 40 * 30)
    x = api.PaddedVector(40 * 30, api.levin_pad(40))
    with pytest.raises(L.GmError) as e:
        api.banded_solve(Lm, x, b, W=40, solver="pcg", rtol=1e-6)
    assert e.value.status == L.GM_ERR_UNSUPPORTED
