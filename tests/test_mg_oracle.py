"""CPU checks of the multigrid oracle (oracle/mg.py) that the GPU hierarchy,
V-cycle and solve are compared with.  The reference leaves its aggregation
operators unfinished (gridoperators.h:18-138), so there is no reference
output to pin against; the oracle is pinned by identities instead: each
coarse operator equals P^T A P, the V-cycle is a symmetric positive-definite
operator, and PCG with it converges on the synthetic problems."""
import numpy as np
import pytest

from gpumatting_b200.synth import make_problem


def _levels(orc, W, H, seed=0):
    from oracle import mg as M

    p = make_problem(W, H, seed)
    w = orc.levin_sym64(p.image.astype(np.float64) / 255.0, p.eps)
    g = p.gamma.ravel().astype(np.float64)
    d = g.reshape(H, W).copy()
    for k, (du, dv) in enumerate(M.fine_offsets()):
        wk = w[k].reshape(H, W)
        d += wk + M._shift(wk, -du, -dv)
    return M, p, w, g, d.ravel(), M.hierarchy(w, d.ravel(), g, W, H)


@pytest.mark.parametrize("W,H", [(40, 30), (37, 29), (9, 14)])
def test_level_zero_is_the_operator_and_coarse_levels_are_galerkin(orc, W, H):
    M, p, w, g, d, lv = _levels(orc, W, H)
    op = orc.Operator(W=W, H=H, w=w, gamma=g)
    x = np.random.default_rng(0).standard_normal(W * H)
    assert np.allclose(lv[0].apply(x.reshape(H, W)).ravel(), op.apply(x), rtol=1e-12, atol=1e-9)
    for l in range(len(lv) - 1):
        f, c = lv[l], lv[l + 1]
        assert (c.W, c.H) == ((f.W + 1) // 2, (f.H + 1) // 2)
        xc = np.random.default_rng(l).standard_normal((c.H, c.W))
        lhs = c.apply(xc)
        rhs = M.restrict(f.apply(M.prolong(xc, f.H, f.W)), c.H, c.W)
        assert np.allclose(lhs, rhs, rtol=1e-10, atol=1e-9 * np.abs(lhs).max())
    assert lv[-1].W * lv[-1].H <= M.COARSE_MAX < lv[-2].W * lv[-2].H or len(lv) == 2
    n = lv[-1].W * lv[-1].H
    assert np.allclose(lv[-1].inv @ lv[-1].A, np.eye(n), atol=1e-8)


def test_vcycle_is_symmetric_positive_definite(orc):
    M, p, w, g, d, lv = _levels(orc, 48, 36)
    rng = np.random.default_rng(3)
    u, v = rng.standard_normal((2, 36, 48))
    Mu, Mv = M.vcycle(lv, u), M.vcycle(lv, v)
    assert abs(np.sum(u * Mv) - np.sum(Mu * v)) <= 1e-10 * np.sqrt(np.sum(u * u) * np.sum(Mv * Mv))
    for t in (u, v):
        assert np.sum(t * M.vcycle(lv, t)) > 0.0


def test_mgpcg_converges_and_beats_cg(orc):
    W, H = 160, 120
    M, p, w, g, d, lv = _levels(orc, W, H)
    op = orc.Operator(W=W, H=H, w=w, gamma=g)
    b = (p.gamma * p.s).ravel().astype(np.float64)
    x, it, rel = M.mgpcg(lv, op.apply, b, np.full(W * H, 0.5), 1e-6, 400)
    assert rel <= 1e-6
    assert np.linalg.norm(b - op.apply(x.ravel())) / np.linalg.norm(b) <= 1.001e-6
    _, it_cg, _ = op.cg(b, np.full(W * H, 0.5), rtol=1e-6, maxit=20000)
    assert it * 4 < it_cg, (it, it_cg)


@pytest.mark.parametrize("W,H", [(1920, 1080), (4096, 4096), (37, 29), (8, 2), (1, 1), (1000, 3), (130, 3)])
def test_level_shapes_match_oracle(W, H):
    """gm_levin_mg_levels (host only, no device call) lists the oracle's
    hierarchy: 2x2 coarsening until a level has at most 128 cells."""
    import ctypes as C

    from gpumatting_b200 import _lib as L
    from oracle import mg as M

    n = C.c_int(0)
    dims = (C.c_int * 64)()
    assert L.load().gm_levin_mg_levels(W, H, C.byref(n), dims, 32) == 0
    got = [(dims[2 * i], dims[2 * i + 1]) for i in range(n.value)]
    want = [(W, H)]
    while True:
        w, h = want[-1]
        want.append(((w + 1) // 2, (h + 1) // 2))
        if want[-1][0] * want[-1][1] <= M.COARSE_MAX:
            break
    assert got == want


def test_level_shapes_reject_bad_sizes():
    import ctypes as C

    from gpumatting_b200 import _lib as L

    n = C.c_int(0)
    assert L.load().gm_levin_mg_levels(0, 5, C.byref(n), None, 0) == L.GM_ERR_INVALID
    assert L.load().gm_levin_mg_levels(5, -1, C.byref(n), None, 0) == L.GM_ERR_INVALID


def test_fp32_scheme_needs_the_restart_rule(orc):
    """The GPU solver's arithmetic scheme (oracle mg.mgpcg_fp32: FP32 vectors
    and increment, FP64 replacement every 50) on A lambda = 1/2 from
    lambda = 0, the adjoint of sum(alpha) on the 96x64 edge image of
    tests/c/test_native.c.  lambda reaches ~190, so the first 50 iterations
    carry all of it in the FP32 increment and the first true residual is far
    above the recurrence's.  Without the gap restart the next beta lets the
    stale direction swamp the new one and the solve stalls; with it the
    solve converges in about the FP64 PCG's iterations."""
    from gpu_util import edge_image
    from oracle import mg as M

    W, H = 96, 64
    img, sc = edge_image(W, H)
    w = np.asarray(orc.levin_sym64(img.astype(np.float64) / 255.0, 1e-5)).reshape(12, -1)
    g = np.where(sc != 128, 100.0, 0.0).ravel()
    offs = M.fine_offsets()

    def diag(wp):
        d = g.reshape(H, W).copy()
        for k, (du, dv) in enumerate(offs):
            wk = wp[k].astype(np.float64).reshape(H, W)
            d += wk + M._shift(wk, -du, -dv)
        return d.ravel()

    # V-cycle on FP16 planes, outer operator on FP32 planes (the GPU's split)
    w16 = w.astype(np.float16).astype(np.float64)
    lv = M.hierarchy(w16, diag(w16), g, W, H)
    w32 = w.astype(np.float32)
    d32 = diag(w32).astype(np.float32).reshape(H, W)

    def apply32(x):
        x = x.reshape(H, W).astype(np.float32)
        y = d32 * x
        for k, (du, dv) in enumerate(offs):
            c = w32[k].reshape(H, W)
            y = y - c * M._shift(x, du, dv) - M._shift(c * x, -du, -dv)
        return y.ravel()

    op = orc.Operator(W=W, H=H, w=w32.astype(np.float64), gamma=g)
    b = np.full(W * H, 0.5)
    x64, it64, rel64 = M.mgpcg(lv, op.apply, b, np.zeros(W * H), rtol=1e-6, maxit=300)
    assert rel64 <= 1e-6 and np.abs(x64).max() > 100.0
    _, it_no, rel_no = M.mgpcg_fp32(lv, op.apply, apply32, b, np.zeros(W * H), rtol=1e-6, maxit=300,
                                    restart_gap=False)
    assert rel_no > 1e-5, (it_no, rel_no)  # stalled
    _, it_yes, rel_yes = M.mgpcg_fp32(lv, op.apply, apply32, b, np.zeros(W * H), rtol=1e-6, maxit=300)
    assert rel_yes <= 1e-6 and it_yes <= 1.3 * it64 + 10, (it_yes, it64)


def test_fp16_outer_operator_pays_only_at_loose_tolerance(orc):
    """The GPU solver takes the FP16 planes for the outer matrix products of
    an FP16 store only when rtol >= 1e-7.  In its FP32 scheme (oracle
    mg.mgpcg_fp32) the FP16 outer operator costs a few iterations at 1e-6
    but many at 1e-10: between replacements each cycle can only refine as
    far as the FP16 operator allows."""
    from oracle import mg as M

    W, H = 240, 160
    p = make_problem(W, H, 0)
    w = np.asarray(orc.levin_sym64(p.image.astype(np.float64) / 255.0, p.eps)).reshape(12, -1)
    g = p.gamma.ravel().astype(np.float64)
    b = (p.gamma * p.s).ravel().astype(np.float64)
    offs = M.fine_offsets()

    def diag(wp):
        d = g.reshape(H, W).copy()
        for k, (du, dv) in enumerate(offs):
            wk = wp[k].astype(np.float64).reshape(H, W)
            d += wk + M._shift(wk, -du, -dv)
        return d.ravel()

    def operator32(wp):
        dp = diag(wp).astype(np.float32).reshape(H, W)

        def apply(x):
            x = x.reshape(H, W).astype(np.float32)
            y = dp * x
            for k, (du, dv) in enumerate(offs):
                c = wp[k].reshape(H, W)
                y = y - c * M._shift(x, du, dv) - M._shift(c * x, -du, -dv)
            return y.ravel()

        return apply

    w16 = w.astype(np.float16).astype(np.float32)
    w32 = w.astype(np.float32)
    lv = M.hierarchy(w16.astype(np.float64), diag(w16), g, W, H)
    op = orc.Operator(W=W, H=H, w=w32.astype(np.float64), gamma=g)
    it = {}
    for rtol in (1e-6, 1e-10):
        for name, wp in (("fp32", w32), ("fp16", w16)):
            _, n, rel = M.mgpcg_fp32(lv, op.apply, operator32(wp), b, np.full(W * H, 0.5), rtol=rtol, maxit=2000)
            assert rel <= rtol, (name, rtol, n, rel)  # both converge on the true operator
            it[name, rtol] = n
    loose = it["fp16", 1e-6] / it["fp32", 1e-6]
    tight = it["fp16", 1e-10] / it["fp32", 1e-10]
    assert loose <= 1.1, it
    assert tight >= loose + 0.15, it
