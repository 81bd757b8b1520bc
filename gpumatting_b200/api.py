"""Python mirror of the reference's BandedMatrix / Vector / Solve API over
libgpumat's C ABI.

Device memory comes from torch (CUDA tensors); every computation runs in
libgpumat.so.  Names follow the reference (main.cu, BandedMatrix.cu,
Vector.cu, Matting.cu, Solve.cpp); the gm_* native layer adds the symmetric
mixed-precision store, solver parameters and results.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _lib as L


def _torch():
    import torch

    return torch


def _stream(stream=None) -> int:
    torch = _torch()
    s = torch.cuda.current_stream() if stream is None else stream
    return s.cuda_stream


def _ptr(t) -> int | None:
    return None if t is None else t.data_ptr()


def levin_band_offsets(W: int) -> np.ndarray:
    """main.cu:164-190: offsets du + W dv at band 12 + du + 5 dv."""
    o = (C.c_int * 25)()
    L.load().gm_levin_band_offsets(W, o)
    return np.array(list(o), np.int32)


def levin_pad(W: int) -> int:
    """main.cu:229."""
    return int(L.load().gm_levin_pad(W))


# ---------------------------------------------------------------------------
# Reference data types
# ---------------------------------------------------------------------------
class DeviceBandedMatrix:
    """A device BandedMatrix (BandedMatrix.h:23-38) backed by torch tensors.

    ``a`` is (nbands, apitch) float32, band j of row i at a[j, i];
    ``bands`` holds the int32 offsets on the device (as bmCopyToDevice leaves
    them, BandedMatrix.cu:23-41).
    """

    def __init__(self, a, bands, rows: int):
        torch = _torch()
        assert a.dtype == torch.float32 and a.is_cuda and a.dim() == 2
        self.a = a
        self.bands = bands
        self.rows = rows
        self.nbands = a.shape[0]
        self.apitch = a.stride(0)

    @classmethod
    def from_host(cls, a_host: np.ndarray, offsets, apitch: int | None = None, device="cuda"):
        torch = _torch()
        nb, rows = a_host.shape
        ap = apitch or ((rows + 63) // 64) * 64
        a = torch.zeros((nb, ap), dtype=torch.float32, device=device)
        a[:, :rows] = torch.from_numpy(np.ascontiguousarray(a_host, np.float32)).to(device)
        bands = torch.tensor(np.asarray(offsets, np.int32), dtype=torch.int32, device=device)
        return cls(a, bands, rows)

    @property
    def struct(self) -> L.BandedMatrix:
        return L.BandedMatrix(self.a.data_ptr(), self.apitch, self.bands.data_ptr(), self.nbands, self.rows,
                              self.rows)


class PaddedVector:
    """Zero-padded device vector (Vector.cu:23-46): ``ptr`` is element 0."""

    def __init__(self, n: int, pad: int, init=None, device="cuda"):
        torch = _torch()
        self.n, self.pad = n, pad
        self.storage = torch.zeros(n + 2 * pad, dtype=torch.float32, device=device)
        if init is not None:
            self.storage[pad:pad + n] = torch.as_tensor(np.asarray(init, np.float32).ravel(), device=device)

    @property
    def ptr(self) -> int:
        return self.storage.data_ptr() + 4 * self.pad

    @property
    def data(self):
        return self.storage[self.pad:self.pad + self.n]


# ---------------------------------------------------------------------------
# Drop-in solvers (main.cu:406-556), device data, legacy stream
# ---------------------------------------------------------------------------
def cgSolve(alpha: PaddedVector, Lm: DeviceBandedMatrix, b, pad: int, iterations: int, restartInterval: int):
    lib = L.load()
    lib.cgSolve(alpha.ptr, Lm.struct, _ptr(b), pad, iterations, restartInterval)
    L.check(lib.gm_last_status())


def gradSolve(alpha: PaddedVector, Lm: DeviceBandedMatrix, b, iterations: int, pad: int):
    lib = L.load()
    lib.gradSolve(alpha.ptr, Lm.struct, _ptr(b), iterations, pad)
    L.check(lib.gm_last_status())


def jacobi(x: PaddedVector, a: DeviceBandedMatrix, b, omega: float, pad: int, iterations: int):
    lib = L.load()
    lib.jacobi(x.ptr, a.struct, _ptr(b), omega, pad, iterations)
    L.check(lib.gm_last_status())


def hostLevinLaplacian(bands_host: np.ndarray, b_host: np.ndarray, lam: float, im4: np.ndarray,
                       scribs: np.ndarray, W: int, H: int, imPitch: int | None = None):
    """Matting.cu:39-219 with host arrays; fills bands_host (25, N) and b_host."""
    lib = L.load()
    assert bands_host.dtype == np.float32 and bands_host.flags.c_contiguous and bands_host.shape[0] == 25
    offs = levin_band_offsets(W)
    m = L.BandedMatrix(bands_host.ctypes.data, bands_host.shape[1], offs.ctypes.data, 25, W * H, W * H)
    im4 = np.ascontiguousarray(im4, np.float32)
    sc = np.ascontiguousarray(scribs, np.uint8)
    lib.hostLevinLaplacian(m, b_host.ctypes.data, lam, im4.ctypes.data, sc.ctypes.data, W, H, imPitch or W)
    L.check(lib.gm_last_status())


def _host_matrix(bands_host: np.ndarray, offsets, x_padded: np.ndarray, pad: int):
    """BandedMatrix view of host bands (nbands, N) + checks that x_padded is a
    float32 vector with `pad` >= max |offset| elements either side, since the
    library reads x as far as the pattern reaches."""
    offs = np.ascontiguousarray(offsets, np.int32)
    a = np.ascontiguousarray(bands_host, np.float32)
    if a.ndim != 2 or a.shape[0] != offs.size:
        raise ValueError("bands_host must be (nbands, N) with one offset per band")
    n = a.shape[1]
    if x_padded.dtype != np.float32 or not x_padded.flags.c_contiguous or x_padded.size != n + 2 * pad:
        raise ValueError(f"x_padded must be contiguous float32 of N + 2*pad = {n + 2 * pad} elements")
    if offs.size and pad < int(np.abs(offs).max()):
        raise ValueError(f"pad {pad} is smaller than the band reach {int(np.abs(offs).max())}")
    m = L.BandedMatrix(a.ctypes.data, n, offs.ctypes.data, a.shape[0], n, n)
    return m, (a, offs)


def jacobi_host(x_padded: np.ndarray, pad: int, bands_host: np.ndarray, offsets, b: np.ndarray, iterations: int,
                omega: float = 2.0 / 3.0):
    """Solve.cpp:35-85 on host arrays (x_padded has `pad` elements each side);
    the iterates are bit-identical to the reference's."""
    lib = L.load()
    m, keep = _host_matrix(bands_host, offsets, x_padded, pad)
    bb = np.ascontiguousarray(b, np.float32)
    lib.jacobi_host(x_padded.ctypes.data + 4 * pad, C.byref(m), bb.ctypes.data, iterations, pad, omega)
    L.check(lib.gm_last_status())


def gaussSeidel_host(x_padded: np.ndarray, pad: int, bands_host: np.ndarray, offsets, b: np.ndarray,
                     iterations: int):
    """Solve.cpp:3-33 on host arrays, any band pattern; bit-identical to the
    reference's sequential sweep."""
    lib = L.load()
    m, keep = _host_matrix(bands_host, offsets, x_padded, pad)
    bb = np.ascontiguousarray(b, np.float32)
    lib.gaussSeidel_host(x_padded.ctypes.data + 4 * pad, C.byref(m), bb.ctypes.data, iterations)
    L.check(lib.gm_last_status())


def gs_host_levels(bands_host: np.ndarray, offsets) -> int:
    """Levels of gaussSeidel_host's schedule (dependent steps per sweep)."""
    offs = np.ascontiguousarray(offsets, np.int32)
    a = np.ascontiguousarray(bands_host, np.float32)
    n = a.shape[1]
    m = L.BandedMatrix(a.ctypes.data, n, offs.ctypes.data, a.shape[0], n, n)
    return int(L.load().gm_gs_host_levels(C.byref(m)))


# ---------------------------------------------------------------------------
# L2 kernels
# ---------------------------------------------------------------------------
def bm_ax(b, Lm: DeviceBandedMatrix, x: PaddedVector, stream=None):
    L.check(L.load().gm_bm_ax(_ptr(b), Lm.struct, x.ptr, _stream(stream)))


def bm_axpy(b, Lm: DeviceBandedMatrix, x: PaddedVector, y, add: bool, stream=None):
    L.check(L.load().gm_bm_axpy(_ptr(b), Lm.struct, x.ptr, _ptr(y), int(add), _stream(stream)))


def jacobi_step(xx, x: PaddedVector, Lm: DeviceBandedMatrix, b, omega: float, stream=None):
    L.check(L.load().gm_jacobi_step(_ptr(xx), x.ptr, Lm.struct, _ptr(b), omega, _stream(stream)))


def _check_dot_operands(x, y):
    torch = _torch()
    if not (isinstance(x, torch.Tensor) and isinstance(y, torch.Tensor)):
        raise TypeError("x and y must be torch tensors")
    if x.dtype != torch.float32 or y.dtype != torch.float32:
        raise TypeError(f"x and y must be float32 (got {x.dtype}, {y.dtype})")
    if not (x.is_cuda and y.is_cuda) or x.device != y.device:
        raise ValueError("x and y must be CUDA tensors on one device")
    if not (x.is_contiguous() and y.is_contiguous()):
        raise ValueError("x and y must be contiguous")
    if x.numel() != y.numel():
        raise ValueError(f"x and y differ in length ({x.numel()} vs {y.numel()})")
    if x.numel() > 2**31 - 1:
        raise ValueError("vectors longer than 2^31 - 1 elements are not supported")


def inner_prod(x, y, stream=None, f64: bool = False):
    torch = _torch()
    _check_dot_operands(x, y)
    out = torch.zeros(1, dtype=torch.float64 if f64 else torch.float32, device=x.device)
    fn = L.load().gm_inner_prod_f64 if f64 else L.load().gm_inner_prod
    L.check(fn(out.data_ptr(), x.data_ptr(), y.data_ptr(), x.numel(), _stream(stream)))
    return out


def inner_prod_noalloc(x, y, out, stream=None):
    """<x, y> in FP64 into the device double `out`, allocating nothing.

    `out` must be a float64 CUDA tensor on the operands' device: the library
    writes one 8-byte double there, so a float32 or host tensor is refused
    here rather than overrun on the device."""
    torch = _torch()
    _check_dot_operands(x, y)
    if not isinstance(out, torch.Tensor) or out.dtype != torch.float64 or not out.is_cuda or out.numel() < 1:
        raise TypeError("out must be a float64 CUDA tensor with at least one element")
    if out.device != x.device:
        raise ValueError("out must be on the operands' device")
    if not out.is_contiguous():
        raise ValueError("out must be contiguous")
    L.check(L.load().gm_inner_prod_f64_noalloc(out.data_ptr(), x.data_ptr(), y.data_ptr(), x.numel(),
                                               _stream(stream)))
    return out


def compute_error(alpha, gt, W: int, H: int, stream=None) -> float:
    v = C.c_double(0)
    L.check(L.load().gm_compute_error(C.byref(v), alpha.data_ptr(), gt.data_ptr(), W, H, _stream(stream)))
    return v.value


def _row_blocks(*ts):
    """(rows, W, pitches) of equally shaped [rows, W] float32 CUDA blocks
    whose rows are contiguous (a row pitch of stride(0) floats)."""
    torch = _torch()
    t0 = ts[0]
    for t in ts:
        if not isinstance(t, torch.Tensor) or t.dtype != torch.float32:
            raise TypeError("operands must be float32 torch tensors")
        if not t.is_cuda or t.device != t0.device:
            raise ValueError("operands must be CUDA tensors on one device")
        if t.dim() != 2 or t.shape != t0.shape:
            raise ValueError(f"operands must be [rows, W] blocks of one shape (got {[tuple(u.shape) for u in ts]})")
        if t.shape[1] > 1 and t.stride(1) != 1:
            raise ValueError("rows must be contiguous")
        if t.stride(0) < t.shape[1] or t.stride(0) > 2**31 - 1:
            raise ValueError("row pitch out of range")
    return int(t0.shape[0]), int(t0.shape[1]), [max(int(t.stride(0)), int(t.shape[1])) for t in ts]


def cg_dots4(r, p, q, out=None, stream=None):
    """FP64 [r.r, p.q, r.q, q.q] over [rows, W] row blocks, into the device
    tensor `out` (4 doubles; allocated when None)."""
    torch = _torch()
    rows, W, (rp, pp, qp) = _row_blocks(r, p, q)
    if out is None:
        out = torch.empty(4, dtype=torch.float64, device=r.device)
    if out.dtype != torch.float64 or out.device != r.device or out.numel() < 4 or not out.is_contiguous():
        raise TypeError("out must be a contiguous float64 tensor of 4 elements on the operands' device")
    L.check(L.load().gm_cg_dots4(out.data_ptr(), r.data_ptr(), rp, p.data_ptr(), pp, q.data_ptr(), qp, W, rows,
                                 _stream(stream)))
    return out


def cg_update(x, r, p, q, alpha: float, beta: float, update_p: bool = True, stream=None):
    """x += alpha p; r -= alpha q; then p = r + beta p when update_p (FP32)."""
    rows, W, (xp, rp, pp, qp) = _row_blocks(x, r, p, q)
    L.check(L.load().gm_cg_update(x.data_ptr(), xp, r.data_ptr(), rp, p.data_ptr(), pp, q.data_ptr(), qp, W, rows,
                                  float(alpha), float(beta), 1 if update_p else 0, _stream(stream)))


def _f64_dev(t, n: int, name: str, device):
    torch = _torch()
    if (not isinstance(t, torch.Tensor) or t.dtype != torch.float64 or t.device != device or t.numel() < n
            or not t.is_contiguous()):
        raise TypeError(f"{name} must be a contiguous float64 tensor of {n} elements on {device}")


def cg_scalars(coef, state, sums4, stream=None):
    """One thread on the device: coef = [alpha, beta, mode] from the summed
    sums4 = [r.r, p.q, r.q, q.q], advancing the 6-double device state
    (threshold, r.r, next r.r, iterations, stop code, stop-at count)."""
    torch = _torch()
    if not isinstance(sums4, torch.Tensor):
        raise TypeError("sums4 must be a float64 CUDA tensor")
    _f64_dev(sums4, 4, "sums4", sums4.device)
    _f64_dev(coef, 3, "coef", sums4.device)
    _f64_dev(state, 6, "state", sums4.device)
    if not sums4.is_cuda:
        raise ValueError("cg_scalars needs CUDA tensors")
    L.check(L.load().gm_cg_scalars(coef.data_ptr(), state.data_ptr(), sums4.data_ptr(), _stream(stream)))


def cg_update_dev(x, r, p, q, coef, stream=None):
    """cg_update with [alpha, beta, mode] read from the device tensor coef."""
    rows, W, (xp, rp, pp, qp) = _row_blocks(x, r, p, q)
    _f64_dev(coef, 3, "coef", x.device)
    L.check(L.load().gm_cg_update_dev(x.data_ptr(), xp, r.data_ptr(), rp, p.data_ptr(), pp, q.data_ptr(), qp, W,
                                      rows, coef.data_ptr(), _stream(stream)))


# ---------------------------------------------------------------------------
# Native: symmetric Levin store
# ---------------------------------------------------------------------------
PRECISIONS = {"fp32": L.GM_PREC_FP32, "fp16": L.GM_PREC_FP16, "bf16": L.GM_PREC_BF16}
SOLVERS = {"cg": L.GM_SOLVER_CG, "gd": L.GM_SOLVER_GD, "jacobi": L.GM_SOLVER_JACOBI, "pcg": L.GM_SOLVER_PCG,
           "mg": L.GM_SOLVER_MG}


def _image_desc(image) -> L.GmImage:
    torch = _torch()
    if image.dtype == torch.uint8:
        assert image.dim() == 3 and image.shape[2] == 3 and image.is_contiguous()
        return L.GmImage(image.data_ptr(), L.GM_IMAGE_RGB8, image.shape[1] * 3)
    assert image.dtype == torch.float32 and image.dim() == 3 and image.shape[2] == 4 and image.is_contiguous()
    return L.GmImage(image.data_ptr(), L.GM_IMAGE_RGBA32F, image.shape[1] * 16)


def _scrib_desc(scribbles=None, gamma_value: float = 100.0, gamma_map=None, s_map=None) -> L.GmScribbles:
    sc = L.GmScribbles()
    sc.gamma_value = gamma_value
    if scribbles is not None:
        sc.map = scribbles.data_ptr()
        sc.map_pitch = scribbles.shape[1]
    if gamma_map is not None:
        sc.gamma_map = gamma_map.data_ptr()
        sc.s_map = None if s_map is None else s_map.data_ptr()
    return sc


@dataclass
class SolveResult:
    status: int
    iters: int
    replacements: int
    rel_residual: float
    kernel_ms: float
    grid: int

    solver: str = ""

    @classmethod
    def from_info(cls, info: L.GmSolveInfo) -> "SolveResult":
        name = {v: k for k, v in SOLVERS.items()}.get(info.solver, str(info.solver))
        return cls(info.status, info.iters, info.replacements, info.rel_residual, info.kernel_ms, info.grid, name)


class LevinStore:
    """gm_levin_store: 12 planes of upper affinities (+ FP32 copy), gamma, b."""

    def __init__(self, W: int, H: int, precision: str = "fp16"):
        self.s = L.GmLevinStore()
        L.check(L.load().gm_levin_store_alloc(C.byref(self.s), W, H, PRECISIONS[precision]))
        self.W, self.H, self.precision = W, H, precision

    def __del__(self):
        try:
            if self.s.owns:
                L.load().gm_levin_store_free(C.byref(self.s))
        except Exception:
            pass

    def assemble(self, image, scribbles=None, eps: float = 1e-5, gamma_value: float = 100.0, gamma_map=None,
                 s_map=None, bands25: DeviceBandedMatrix | None = None, b25=None, stream=None):
        im = _image_desc(image)
        sc = _scrib_desc(scribbles, gamma_value, gamma_map, s_map)
        bm = None if bands25 is None else C.byref(bands25.struct)
        L.check(L.load().gm_levin_assemble(C.byref(self.s), C.byref(im), C.byref(sc), eps, bm, _ptr(b25),
                                           _stream(stream)))
        # The adjoint recomputes window statistics from the same inputs.
        self._inputs = (image, scribbles, eps, gamma_value, gamma_map, s_map)
        return self

    def restrict(self, scribbles=None, gamma_map=None, s_map=None, stream=None):
        """Hard-constrain the known pixels (scribbled, or gamma_map > 0) to their
        targets and eliminate them: the store then holds the system on the
        unknown pixels (gm_levin_restrict)."""
        sc = _scrib_desc(scribbles, 1.0, gamma_map, s_map)
        L.check(L.load().gm_levin_restrict(C.byref(self.s), C.byref(sc), _stream(stream)))
        return self

    def planes(self, which: str = "w32"):
        """Views of the store's device planes as torch tensors (H, pitch)."""
        torch = _torch()
        W, H, P = self.W, self.H, self.s.pitch
        n = H * P
        if which == "w32":
            return _wrap(self.s.w32, (12, H, P), torch.float32)
        if which == "w":
            dt = {"fp32": torch.float32, "fp16": torch.float16, "bf16": torch.bfloat16}[self.precision]
            return _wrap(self.s.w, (12, H, P), dt)
        if which == "gamma":
            return _wrap(self.s.gamma, (H, P), torch.float32)
        if which == "b":
            return _wrap(self.s.b, (H, P), torch.float32)
        if which == "d":
            return _wrap(self.s.d, (H, P), torch.float32)
        if which == "d32":
            return _wrap(self.s.d32, (H, P), torch.float32)
        raise KeyError(which)

    def solve(self, alpha, solver: str = "cg", stream=None, **params) -> SolveResult:
        p = L.default_params(solver=SOLVERS[solver], **params)
        info = L.GmSolveInfo()
        rc = L.load().gm_levin_solve(C.byref(self.s), alpha.data_ptr(), C.byref(p), C.byref(info), _stream(stream))
        if rc not in (L.GM_OK, L.GM_ERR_NOT_CONVERGED):
            L.check(rc)
        return SolveResult.from_info(info)

    def mg_levels(self) -> list:
        """(width, height) of each level of the GM_SOLVER_MG hierarchy."""
        n = C.c_int(0)
        dims = (C.c_int * 64)()
        L.check(L.load().gm_levin_mg_levels(self.W, self.H, C.byref(n), dims, 32))
        return [(dims[2 * i], dims[2 * i + 1]) for i in range(n.value)]

    def mg_inspect(self, r=None, level: int = 0, use_low: bool = True, stream=None):
        """Builds the multigrid hierarchy; returns (z, c, D): z = one V-cycle
        applied to r ([H, W] device floats, or None), and for level >= 1 that
        level's coupling planes (4, H_l, W_l) and diagonal (H_l, W_l) as numpy
        arrays (None for level 0)."""
        import numpy as np

        torch = _torch()
        z = None if r is None else torch.empty_like(r)
        c = d = None
        if level >= 1:
            Wl, Hl = self.mg_levels()[level]
            c = np.zeros((4, Hl, Wl), np.float32)
            d = np.zeros((Hl, Wl), np.float32)
        L.check(L.load().gm_levin_mg_inspect(C.byref(self.s), 1 if use_low else 0, _ptr(r), _ptr(z), level,
                                             None if c is None else c.ctypes.data,
                                             None if d is None else d.ctypes.data, _stream(stream)))
        return z, c, d

    def apply(self, x, y=None, true_op: bool = False, stream=None):
        """y = A x ([H, W'] device floats, W' >= W a multiple of 4) with the
        iteration operator (true_op False) or the true FP32 operator."""
        torch = _torch()
        if y is None:
            y = torch.empty_like(x)
        L.check(L.load().gm_levin_apply(C.byref(self.s), x.data_ptr(), x.stride(0), y.data_ptr(), y.stride(0),
                                        1 if true_op else 0, _stream(stream)))
        return y

    def solve_rhs(self, rhs, x, solver: str = "cg", stream=None, **params) -> SolveResult:
        """Solve the store's system for rhs ([H, W] device floats); x holds the
        initial guess and receives the solution."""
        p = L.default_params(solver=SOLVERS[solver], **params)
        info = L.GmSolveInfo()
        rc = L.load().gm_levin_solve_rhs(C.byref(self.s), rhs.data_ptr(), x.data_ptr(), C.byref(p), C.byref(info),
                                         _stream(stream))
        if rc not in (L.GM_OK, L.GM_ERR_NOT_CONVERGED):
            L.check(rc)
        return SolveResult.from_info(info)

    def adjoint(self, alpha, dalpha, solver: str = "mg", want_dgamma: bool = True, stream=None, **params):
        """Gradients of a loss of alpha through solve and assembly.

        The lambda solve defaults to the multigrid-preconditioned CG, the one
        solver that converges on this right-hand side at every size and eps
        tried (CG and Jacobi PCG stall at 4096^2 with eps = 1e-7; asked for,
        they fall back to it when they do not converge).

        dalpha = dloss/dalpha ([H, W] device floats).  Returns (dimage, dgamma,
        lam, SolveResult of the lam solve): dimage has the channel count of the
        assembled image layout (3 for RGB8, 4 for RGBA32F with the last 0) and
        is the gradient for the [0, 1] channel values."""
        torch = _torch()
        image, scribbles, eps, gamma_value, gamma_map, s_map = self._inputs
        W, H = self.W, self.H
        ch = 4 if image.dtype == torch.float32 else 3
        dimage = torch.empty((H, W, ch), dtype=torch.float32, device=alpha.device)
        lam = torch.empty((H, W), dtype=torch.float32, device=alpha.device)
        dgamma = torch.empty((H, W), dtype=torch.float32, device=alpha.device) if want_dgamma else None
        im = _image_desc(image)
        sc = _scrib_desc(scribbles, gamma_value, gamma_map, s_map)
        p = L.default_params(solver=SOLVERS[solver], **params)
        info = L.GmSolveInfo()
        rc = L.load().gm_levin_adjoint(C.byref(self.s), C.byref(im), C.byref(sc), eps, alpha.data_ptr(),
                                       dalpha.data_ptr(), lam.data_ptr(), dimage.data_ptr(), W * ch, ch,
                                       _ptr(dgamma), C.byref(p), C.byref(info), _stream(stream))
        if rc not in (L.GM_OK, L.GM_ERR_NOT_CONVERGED):
            L.check(rc)
        return dimage, dgamma, lam, SolveResult.from_info(info)


class LevinBatch:
    """gm_batch: many images of different sizes solved in one persistent
    launch (replayed from a CUDA graph), with a tuned launch shape."""

    def __init__(self, sizes, precision: str = "fp16"):
        self.sizes = [(int(w), int(h)) for w, h in sizes]
        n = len(self.sizes)
        ws = (C.c_int * n)(*[w for w, _ in self.sizes])
        hs = (C.c_int * n)(*[h for _, h in self.sizes])
        self.h = C.c_void_p()
        L.check(L.load().gm_batch_create(C.byref(self.h), n, ws, hs, PRECISIONS[precision]))
        self.precision = precision
        self._inputs = [None] * n

    def __del__(self):
        try:
            if self.h:
                L.load().gm_batch_destroy(self.h)
                self.h = C.c_void_p()
        except Exception:
            pass

    def __len__(self):
        return len(self.sizes)

    def assemble(self, k: int, image, scribbles=None, eps: float = 1e-5, gamma_value: float = 100.0, gamma_map=None,
                 s_map=None, stream=None):
        im = _image_desc(image)
        sc = _scrib_desc(scribbles, gamma_value, gamma_map, s_map)
        L.check(L.load().gm_batch_assemble(self.h, k, C.byref(im), C.byref(sc), eps, _stream(stream)))
        self._inputs[k] = (image, scribbles, gamma_map, s_map)
        return self

    def restrict(self, k: int, scribbles=None, gamma_map=None, s_map=None, stream=None):
        """gm_levin_restrict on image k's store view: its known pixels are
        fixed and eliminated (hard constraints)."""
        v = self.store_view(k)
        sc = _scrib_desc(scribbles, 1.0, gamma_map, s_map)
        L.check(L.load().gm_levin_restrict(C.byref(v), C.byref(sc), _stream(stream)))
        return self

    def store_view(self, k: int) -> L.GmLevinStore:
        v = L.GmLevinStore()
        L.check(L.load().gm_batch_store(self.h, k, C.byref(v)))
        return v

    def tune(self, iters: int = 20, stream=None, **params) -> dict:
        p = L.default_params(**params)
        L.check(L.load().gm_batch_tune(self.h, C.byref(p), iters, _stream(stream)))
        return self.info()

    def info(self) -> dict:
        v = [C.c_int() for _ in range(5)]
        L.check(L.load().gm_batch_info(self.h, *[C.byref(x) for x in v]))
        d = dict(zip(["ctas_per_sm", "ring_cfg", "row_mult", "graph_launches", "grid"], [x.value for x in v]))
        # launch configurations of the fused solver: 0, 1 = 192-column strips
        # (shallow / deep rings), 2 = 128-column strips
        d["strip_width"] = {0: 192, 1: 192, 2: 128}.get(d["ring_cfg"], 0)
        return d

    def solve(self, alphas, solver: str = "cg", stream=None, **params) -> list:
        n = len(self.sizes)
        assert len(alphas) == n
        ptrs = (C.c_void_p * n)(*[a.data_ptr() for a in alphas])
        infos = (L.GmSolveInfo * n)()
        p = L.default_params(solver=SOLVERS[solver], **params)
        rc = L.load().gm_batch_solve(self.h, ptrs, C.byref(p), infos, _stream(stream))
        if rc not in (L.GM_OK, L.GM_ERR_NOT_CONVERGED):
            L.check(rc)
        return [SolveResult.from_info(infos[k]) for k in range(n)]


class _CudaArray:
    """Minimal __cuda_array_interface__ holder so torch can view device
    memory that libgpumat owns (no copy)."""

    def __init__(self, ptr: int, shape, typestr: str):
        self.__cuda_array_interface__ = {"shape": tuple(shape), "typestr": typestr, "data": (ptr, False),
                                         "version": 3, "strides": None}


def _wrap(ptr: int, shape, dtype):
    """Non-owning torch view of device memory owned by libgpumat."""
    torch = _torch()
    if dtype == torch.bfloat16:
        return torch.as_tensor(_CudaArray(ptr, shape, "<i2"), device="cuda").view(torch.bfloat16)
    ts = {torch.float32: "<f4", torch.float16: "<f2", torch.float64: "<f8"}[dtype]
    return torch.as_tensor(_CudaArray(ptr, shape, ts), device="cuda")


def mg_solve_many(stores, alphas, stream=None, **params) -> list:
    """gm_levin_solve_mg_many: independent multigrid solves, one graph launch
    each, on up to 8 concurrent streams.  stores: LevinStore objects or
    GmLevinStore structs (e.g. LevinBatch.store_view(k)); alphas: [H_k, W_k]
    device float tensors (initial guess in, solution out)."""
    n = len(stores)
    assert len(alphas) == n
    structs = [s.s if isinstance(s, LevinStore) else s for s in stores]
    sp = (C.POINTER(L.GmLevinStore) * n)(*[C.pointer(x) for x in structs])
    ap = (C.c_void_p * n)(*[a.data_ptr() for a in alphas])
    infos = (L.GmSolveInfo * n)()
    p = L.default_params(solver=L.GM_SOLVER_MG, **params)
    rc = L.load().gm_levin_solve_mg_many(sp, ap, n, C.byref(p), infos, _stream(stream))
    if rc not in (L.GM_OK, L.GM_ERR_NOT_CONVERGED):
        L.check(rc)
    return [SolveResult.from_info(infos[k]) for k in range(n)]


def levin_bands25(image, scribbles=None, eps: float = 1e-5, gamma_value: float = 100.0, gamma_map=None, s_map=None,
                  arithmetic: str = "fp64", stream=None):
    """25-band FP32 reference-layout store (a (25, N), b (N,)) on the device."""
    torch = _torch()
    H, W = image.shape[0], image.shape[1]
    N = W * H
    a = torch.empty((25, N), dtype=torch.float32, device=image.device)
    b = torch.empty(N, dtype=torch.float32, device=image.device)
    im = _image_desc(image)
    sc = _scrib_desc(scribbles, gamma_value, gamma_map, s_map)
    ar = L.GM_ASSEMBLY_REFERENCE if arithmetic == "reference" else L.GM_ASSEMBLY_FP64
    L.check(L.load().gm_levin_assemble_bands25(a.data_ptr(), N, b.data_ptr(), C.byref(im), C.byref(sc), eps, W, H,
                                               ar, _stream(stream)))
    return a, b


def banded_solve(Lm: DeviceBandedMatrix, alpha: PaddedVector, b, W: int = 0, solver: str = "cg", stream=None,
                 **params) -> SolveResult:
    p = L.default_params(solver=SOLVERS[solver], **params)
    info = L.GmSolveInfo()
    rc = L.load().gm_banded_solve(Lm.struct, W, alpha.ptr, alpha.pad, _ptr(b), C.byref(p), C.byref(info),
                                  _stream(stream))
    if rc not in (L.GM_OK, L.GM_ERR_NOT_CONVERGED):
        L.check(rc)
    return SolveResult.from_info(info)


# ---------------------------------------------------------------------------
# Data formats either side of the solve (ppm.h, main.cu:334-355)
# ---------------------------------------------------------------------------
def read_pnm(path: str):
    """PNM file -> (uint8 array (H, W) or (H, W, 3), maxval) (ppm.h:32-127, :178-278)."""
    img = L.GmPnm()
    L.check(L.load().gm_pnm_read(str(path).encode(), C.byref(img)))
    shape = (img.h, img.w) if img.channels == 1 else (img.h, img.w, 3)
    maxval = img.maxval
    try:
        data = np.ctypeslib.as_array(img.data, shape=(img.w * img.h * img.channels,)).copy()
    finally:
        L.load().gm_pnm_free(C.byref(img))
    return data.reshape(shape), maxval


def write_pgm(path: str, gray: np.ndarray, comment: str | None = None, binary: bool = True):
    """8-bit graymap file, the reference's pgmwrite bytes (ppm.h:345-414)."""
    g = np.ascontiguousarray(gray, dtype=np.uint8)
    h, w = g.shape
    L.check(L.load().gm_pgm_write(str(path).encode(), w, h, g.ctypes.data, None if comment is None else
                                  comment.encode(), int(binary)))


def rgb8_to_float4(rgb, maxval: int = 255, stream=None):
    """Device RGB bytes (H, W, 3) -> (H, W, 4) float32, (r, g, b, 1) / maxval (ppm.h:309-333)."""
    torch = _torch()
    H, W, _ = rgb.shape
    out = torch.empty((H, W, 4), dtype=torch.float32, device=rgb.device)
    L.check(L.load().gm_rgb8_to_float4(out.data_ptr(), rgb.contiguous().data_ptr(), H * W, maxval, _stream(stream)))
    return out


def alpha_to_gray8(alpha, stream=None):
    """Device alpha -> uint8 matte, clamped and truncated as pgmwrite_float (ppm.h:430-451)."""
    torch = _torch()
    out = torch.empty(alpha.shape, dtype=torch.uint8, device=alpha.device)
    L.check(L.load().gm_alpha_to_gray8(out.data_ptr(), alpha.contiguous().data_ptr(), alpha.numel(), _stream(stream)))
    return out


def write_alpha_pgm(path: str, alpha, comment: str | None = None, binary: bool = True, stream=None):
    """The reference's alpha.pgm: quantised on the device, written on the host."""
    g = alpha_to_gray8(alpha, stream).cpu().numpy()
    write_pgm(path, g, comment, binary)


def dump_bands(path: str, Lm: DeviceBandedMatrix):
    """A.bin: nbands x rows float32, band-major (main.cu:334-355)."""
    L.check(L.load().gm_bands_dump(str(path).encode(), Lm.struct, 1))
