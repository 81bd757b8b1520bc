"""FP64 restatement of the aggregation multigrid preconditioner and the
multigrid-preconditioned CG of libgpumat (GM_SOLVER_MG).

TEST INFRASTRUCTURE ONLY: imported by tests/ and __graft_entry__.smoke() as
the checker of the GPU hierarchy, V-cycle and solve.  The product never
imports it.

The reference sketches this direction without finishing it: piecewise-
constant aggregation operators (gridoperators.h:18-138, `downsampleOps`
builds coordinate-matrix restrictions with unit entries, i = label, j = pixel,
k = 1) over SLIC superpixels (SLIC.cpp:32; the call is commented out at
main.cu:201-218).  Here the aggregates are fixed 2x2 blocks, so every level
keeps a banded (9-point) stencil:

  level 0   the store's iteration operator: A0 x = d x - W x, W symmetric with
            12 upper planes w_k (k = du + 5 dv, offset (du, dv)).
  level l+1 Galerkin A_{l+1} = P^T A_l P, P the 2x2 piecewise-constant
            aggregation; its upper couplings c_o for o in E (1,0), SW (-1,1),
            S (0,1), SE (1,1) are the sums of the fine couplings between the
            two aggregates; its diagonal is Gamma_I + sum of all couplings
            leaving I, with Gamma_I the summed scribble weight (exact
            Galerkin for the row-sum-preserving operator).
  coarsest  the first level with <= COARSE_MAX cells, solved exactly.

V-cycle on level l for right-hand side b (one damped Jacobi step before and
after the coarse correction, correction over-scaled by `scale`):
  x1 = omega b / D;  rho = b - A x1;  b_{l+1} = P^T rho
  x_{l+1} = V(l+1, b_{l+1})
  y = x1 + scale * P x_{l+1};  x = y + omega (b - A y) / D
The cycle is a symmetric linear operator, so plain PCG applies.
"""
from __future__ import annotations

import numpy as np

COARSE_MAX = 128
OMEGA = 0.8
SCALE = 1.5
# upper offsets of the coarse 9-point stencil, in plane order
COARSE_OFFS = ((1, 0), (-1, 1), (0, 1), (1, 1))


def fine_offsets():
    """(du, dv) of the 12 upper planes, k = du + 5 dv = 1..12."""
    return [(((k + 2) % 5) - 2, (k + 2) // 5) for k in range(1, 13)]


def _shift(x: np.ndarray, du: int, dv: int) -> np.ndarray:
    """out[y, x] = x[y + dv, x + du], zero outside."""
    H, W = x.shape
    out = np.zeros_like(x)
    ys0, ys1 = max(0, -dv), min(H, H - dv)
    xs0, xs1 = max(0, -du), min(W, W - du)
    if ys1 > ys0 and xs1 > xs0:
        out[ys0:ys1, xs0:xs1] = x[ys0 + dv:ys1 + dv, xs0 + du:xs1 + du]
    return out


class Level:
    """One level: upper-coupling planes c (n, H, W) with offsets offs, diagonal D."""

    def __init__(self, c: np.ndarray, offs, D: np.ndarray, gam: np.ndarray):
        self.c = c
        self.offs = list(offs)
        self.D = D
        self.gam = gam
        self.H, self.W = D.shape

    def apply(self, x: np.ndarray) -> np.ndarray:
        y = self.D * x
        for k, (du, dv) in enumerate(self.offs):
            y -= self.c[k] * _shift(x, du, dv)
            # lower coupling: the neighbour (x - du, y - dv) stores it
            y -= _shift(self.c[k] * x, -du, -dv)
        return y


def coarsen(lv: Level) -> Level:
    """Galerkin 2x2 aggregation of one level (FP64)."""
    H, W = lv.H, lv.W
    Hc, Wc = (H + 1) // 2, (W + 1) // 2
    c = np.zeros((4, Hc, Wc))
    ext = np.zeros((Hc, Wc))
    ys, xs = np.mgrid[0:H, 0:W]
    for k, (du, dv) in enumerate(lv.offs):
        xj, yj = xs + du, ys + dv
        ok = (xj >= 0) & (xj < W) & (yj >= 0) & (yj < H)
        w = lv.c[k][ok]
        I = (ys[ok] // 2, xs[ok] // 2)
        J = (yj[ok] // 2, xj[ok] // 2)
        oy, ox = J[0] - I[0], J[1] - I[1]
        cross = (oy != 0) | (ox != 0)
        np.add.at(ext, (I[0][cross], I[1][cross]), w[cross])
        np.add.at(ext, (J[0][cross], J[1][cross]), w[cross])
        for o, (cu, cv) in enumerate(COARSE_OFFS):
            fwd = cross & (ox == cu) & (oy == cv)
            np.add.at(c[o], (I[0][fwd], I[1][fwd]), w[fwd])
            bwd = cross & (ox == -cu) & (oy == -cv)
            np.add.at(c[o], (J[0][bwd], J[1][bwd]), w[bwd])
    gam = np.zeros((Hc, Wc))
    np.add.at(gam, (ys // 2, xs // 2), lv.gam)
    return Level(c, COARSE_OFFS, gam + ext, gam)


def hierarchy(w: np.ndarray, d: np.ndarray, gamma: np.ndarray, W: int, H: int, coarse_max: int = COARSE_MAX):
    """w: (12, H*W) iteration planes (values as the GPU sees them), d: the
    iteration diagonal, gamma: scribble weights.  Returns the level list; the
    last one is the coarsest, with its dense inverse in `.inv`."""
    lv = Level(np.asarray(w, np.float64).reshape(12, H, W), fine_offsets(),
               np.asarray(d, np.float64).reshape(H, W), np.asarray(gamma, np.float64).reshape(H, W))
    levels = [lv]
    while True:
        lv = coarsen(lv)
        levels.append(lv)
        if lv.H * lv.W <= coarse_max:
            break
    n = lv.H * lv.W
    A = np.zeros((n, n))
    for j in range(n):
        e = np.zeros(n)
        e[j] = 1.0
        A[:, j] = lv.apply(e.reshape(lv.H, lv.W)).ravel()
    lv.A = A
    lv.inv = np.linalg.inv(A)
    return levels


def prolong(xc: np.ndarray, H: int, W: int) -> np.ndarray:
    return np.repeat(np.repeat(xc, 2, axis=0), 2, axis=1)[:H, :W]


def restrict(r: np.ndarray, Hc: int, Wc: int) -> np.ndarray:
    H, W = r.shape
    out = np.zeros((Hc, Wc))
    ys, xs = np.mgrid[0:H, 0:W]
    np.add.at(out, (ys // 2, xs // 2), r)
    return out


def vcycle(levels, b: np.ndarray, l: int = 0, omega: float = OMEGA, scale: float = SCALE) -> np.ndarray:
    lv = levels[l]
    if l == len(levels) - 1:
        return (lv.inv @ b.ravel()).reshape(lv.H, lv.W)
    x1 = omega * b / lv.D
    rho = b - lv.apply(x1)
    nx = levels[l + 1]
    xc = vcycle(levels, restrict(rho, nx.H, nx.W), l + 1, omega, scale)
    y = x1 + scale * prolong(xc, lv.H, lv.W)
    return y + omega * (b - lv.apply(y)) / lv.D


def mgpcg(levels, op_apply, b: np.ndarray, x0: np.ndarray, rtol: float = 1e-6, maxit: int = 500,
          omega: float = OMEGA, scale: float = SCALE):
    """PCG with the V-cycle on the operator op_apply (FP64).  Returns
    (x, iterations, relative residual)."""
    H, W = levels[0].H, levels[0].W
    x = np.asarray(x0, np.float64).reshape(H, W).copy()
    bb = np.asarray(b, np.float64).reshape(H, W)
    bn = np.linalg.norm(bb)
    r = bb - op_apply(x.ravel()).reshape(H, W)
    if np.linalg.norm(r) <= rtol * bn:
        return x, 0, np.linalg.norm(r) / bn
    z = vcycle(levels, r, 0, omega, scale)
    p = z.copy()
    rz = float(np.sum(r * z))
    for it in range(1, maxit + 1):
        q = op_apply(p.ravel()).reshape(H, W)
        al = rz / float(np.sum(p * q))
        x += al * p
        r -= al * q
        rel = np.linalg.norm(r) / bn
        if rel <= rtol:
            return x, it, rel
        z = vcycle(levels, r, 0, omega, scale)
        rz1 = float(np.sum(r * z))
        p = z + (rz1 / rz) * p
        rz = rz1
    return x, maxit, np.linalg.norm(r) / bn


def mgpcg_fp32(levels, op_true, apply32, b: np.ndarray, x0: np.ndarray, rtol: float = 1e-6, maxit: int = 500,
               replace_every: int = 50, restart_gap: bool = True, omega: float = OMEGA, scale: float = SCALE):
    """The GPU solver's arithmetic scheme around the same V-cycle, for
    checking its update rules on the CPU (the V-cycle itself stays FP64 here).

    FP64 solution x plus an FP32 increment; FP32 r, p, q; FP64 scalars;
    apply32(p) the FP32 outer operator.  Every `replace_every` iterations and
    at apparent convergence the increment folds into x and the FP64 true
    residual b - op_true(x) replaces r; convergence is declared only there.
    restart_gap: a replacement whose true residual norm exceeds twice the
    recurrence's sets beta = 0 for the next direction (the GPU rule);
    without it beta = (true r.z) / (recurrence r.z).  Returns (x, iterations,
    true relative residual)."""
    f32 = np.float32
    H, W = levels[0].H, levels[0].W
    bb = np.asarray(b, np.float64).ravel()
    bn2 = float(bb @ bb)
    x = np.asarray(x0, np.float64).ravel().copy()
    rt = bb - op_true(x)
    rel = np.sqrt(float(rt @ rt) / bn2)
    if rel <= rtol:
        return x, 0, rel
    r = rt.astype(f32)
    inc = np.zeros_like(r)

    def prec(v):
        return vcycle(levels, v.reshape(H, W).astype(np.float64), 0, omega, scale).ravel().astype(f32)

    z = prec(r)
    p = z.copy()
    rz = float(r.astype(np.float64) @ z)
    for it in range(1, maxit + 1):
        q = apply32(p).astype(f32)
        al = rz / float(p.astype(np.float64) @ q)
        inc = (inc + f32(al) * p).astype(f32)
        r = (r - f32(al) * q).astype(f32)
        rr = float(r.astype(np.float64) @ r)
        restart = False
        if it % replace_every == 0 or rr <= rtol * rtol * bn2 or it == maxit:
            x += inc
            inc[:] = 0
            rt = bb - op_true(x)
            rrt = float(rt @ rt)
            rel = np.sqrt(rrt / bn2)
            if rel <= rtol or it == maxit:
                return x, it, rel
            restart = restart_gap and rrt > 4.0 * rr
            r = rt.astype(f32)
        z = prec(r)
        rz1 = float(r.astype(np.float64) @ z)
        p = (z + f32(0.0 if restart else rz1 / rz) * p).astype(f32)
        rz = rz1
    return x, maxit, rel
