"""ctypes bindings for the CPU oracle (oracle/liborc.so) and, where it was
built, the reference's own CPU code (oracle/_ref/libgmref.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py.  The product package never imports this.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIBORC = os.path.join(HERE, "liborc.so")
LIBREF = os.path.join(HERE, "_ref", "libgmref.so")
# The reference tree (rocketman768/gpumatting sources), used only to build
# oracle/_ref: GM_REFERENCE_TREE when set, else a "reference" directory beside
# the repository.
REF_TREE = os.environ.get("GM_REFERENCE_TREE") or os.path.abspath(os.path.join(HERE, "..", "..", "reference"))

_d = C.POINTER(C.c_double)
_f = C.POINTER(C.c_float)
_i = C.POINTER(C.c_int)
_u8 = C.POINTER(C.c_uint8)


def build(ref: bool | None = None) -> None:
    """Compile liborc.so and, when the reference tree is present, _ref."""
    subprocess.check_call(["make", "-s", "-C", HERE, "all"])
    if ref is None:
        ref = os.path.isdir(REF_TREE)
    if ref:
        subprocess.check_call(["make", "-s", "-C", HERE, "ref", f"REF={REF_TREE}"])


class _Op(C.Structure):
    _fields_ = [("kind", C.c_int), ("W", C.c_int), ("H", C.c_int), ("N", C.c_int),
                ("w", _d), ("gamma", _d), ("a", _d), ("offs", _i), ("nb", C.c_int)]


_lib = None
_ref = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIBORC):
            build(ref=False)
        L = C.CDLL(LIBORC)
        L.orc_levin_offsets.argtypes = [C.c_int, _i]
        L.orc_levin_ref32.argtypes = [_f, C.c_size_t, _f, C.c_float, C.c_float, _f, _u8,
                                      C.c_int, C.c_int, C.c_size_t]
        L.orc_levin_sym64.argtypes = [_d, _d, C.c_double, C.c_int, C.c_int]
        L.orc_sym_to_bands64.argtypes = [_d, _d, _d, C.c_int, C.c_int]
        L.orc_apply_bands64.argtypes = [_d, _d, _i, C.c_int, _d, C.c_int]
        L.orc_apply_sym64.argtypes = [_d, _d, _d, _d, C.c_int, C.c_int]
        L.orc_cg64.argtypes = [C.POINTER(_Op), _d, _d, C.c_double, C.c_int, C.c_int, _d]
        L.orc_cg64.restype = C.c_int
        L.orc_gd64.argtypes = [C.POINTER(_Op), _d, _d, C.c_double, C.c_int, _d]
        L.orc_gd64.restype = C.c_int
        L.orc_jacobi64.argtypes = [C.POINTER(_Op), _d, _d, C.c_double, C.c_double, C.c_int, _d]
        L.orc_jacobi64.restype = C.c_int
        L.orc_gs_host.argtypes = [_f, _f, C.c_size_t, _i, C.c_int, C.c_int, _f, C.c_size_t]
        L.orc_jacobi_host.argtypes = [_f, _f, C.c_size_t, _i, C.c_int, C.c_int, _f, C.c_size_t,
                                      C.c_int, C.c_float]
        L.orc_compute_error.argtypes = [_f, _f, C.c_int, C.c_int]
        L.orc_compute_error.restype = C.c_double
        L.orc_levin_backward64.argtypes = [_d, _d, _d, C.c_double, C.c_int, C.c_int]
        L.orc_num_threads.restype = C.c_int
        _lib = L
    return _lib


def ref_available() -> bool:
    return os.path.exists(LIBREF)


def reflib():
    global _ref
    if _ref is None:
        if not os.path.exists(LIBREF):
            raise FileNotFoundError(LIBREF)
        R = C.CDLL(LIBREF)
        R.ref_hostLevinLaplacian.argtypes = [_f, C.c_size_t, _i, _f, C.c_float, _f, _u8,
                                             C.c_int, C.c_int, C.c_size_t]
        R.ref_gaussSeidel_host.argtypes = [_f, _f, C.c_size_t, _i, C.c_int, C.c_int, _f, C.c_size_t]
        R.ref_jacobi_host.argtypes = [_f, _f, C.c_size_t, _i, C.c_int, C.c_int, _f, C.c_size_t,
                                      C.c_int, C.c_float]
        R.ref_jacobi_host.restype = C.c_int
        R.ref_pgmread.argtypes = [C.c_char_p, C.POINTER(C.c_int), C.POINTER(C.c_int)]
        R.ref_pgmread.restype = C.c_void_p
        R.ref_ppmread.argtypes = [C.c_char_p, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int)]
        R.ref_ppmread.restype = C.c_void_p
        R.ref_ppmread_float4.argtypes = [C.c_char_p, C.POINTER(C.c_int), C.POINTER(C.c_int)]
        R.ref_ppmread_float4.restype = C.c_void_p
        R.ref_pgmwrite_float.argtypes = [C.c_char_p, C.c_int, C.c_int, _f, C.c_char_p, C.c_int]
        R.ref_pgmwrite_float.restype = C.c_int
        R.ref_free.argtypes = [C.c_void_p]
        _ref = R
    return _ref


def ref_read_pnm(path: str, color: bool):
    """The reference's ppmread / pgmread (valid files only): (bytes array, maxval or None)."""
    R = reflib()
    w, h, mv = C.c_int(0), C.c_int(0), C.c_int(0)
    if color:
        ptr = R.ref_ppmread(str(path).encode(), C.byref(w), C.byref(h), C.byref(mv))
        n, shape = w.value * h.value * 3, (h.value, w.value, 3)
    else:
        ptr = R.ref_pgmread(str(path).encode(), C.byref(w), C.byref(h))
        n, shape = w.value * h.value, (h.value, w.value)
    data = np.ctypeslib.as_array(C.cast(ptr, C.POINTER(C.c_ubyte)), shape=(n,)).copy().reshape(shape)
    R.ref_free(ptr)
    return data, (mv.value if color else None)


def ref_ppmread_float4(path: str) -> np.ndarray:
    R = reflib()
    w, h = C.c_int(0), C.c_int(0)
    ptr = R.ref_ppmread_float4(str(path).encode(), C.byref(w), C.byref(h))
    out = np.ctypeslib.as_array(C.cast(ptr, C.POINTER(C.c_float)), shape=(w.value * h.value * 4,)).copy()
    R.ref_free(ptr)
    return out.reshape(h.value, w.value, 4)


def ref_pgmwrite_float(path: str, alpha: np.ndarray, comment: str | None, binary: bool) -> int:
    a = np.ascontiguousarray(alpha, np.float32)
    h, w = a.shape
    return reflib().ref_pgmwrite_float(str(path).encode(), w, h, P(a, _f),
                                       None if comment is None else comment.encode(), int(binary))


def P(a: np.ndarray, t):
    return a.ctypes.data_as(t)


def levin_offsets(W: int) -> np.ndarray:
    o = np.zeros(25, np.int32)
    lib().orc_levin_offsets(W, P(o, _i))
    return o


def pad_for(W: int) -> int:
    """Vector padding of main.cu:229: a multiple of 32 above 2W+2."""
    return ((2 * W + 2) // 32) * 32 + 32


def levin_ref32(im4: np.ndarray, scribs: np.ndarray, lam: float, gamma: float = 1.0):
    """Oracle restatement of hostLevinLaplacian -> (bands (25,N) f32, b (N,))."""
    H, W = scribs.shape
    N = W * H
    a = np.zeros((25, N), np.float32)
    b = np.zeros(N, np.float32)
    im4 = np.ascontiguousarray(im4, np.float32)
    sc = np.ascontiguousarray(scribs, np.uint8)
    lib().orc_levin_ref32(P(a, _f), N, P(b, _f), lam, gamma, P(im4, _f), P(sc, _u8), W, H, W)
    return a, b


def ref_levin(im4: np.ndarray, scribs: np.ndarray, lam: float):
    """The reference's own hostLevinLaplacian (gamma fixed at 1 there)."""
    H, W = scribs.shape
    N = W * H
    a = np.zeros((25, N), np.float32)
    b = np.zeros(N, np.float32)
    offs = levin_offsets(W)
    im4 = np.ascontiguousarray(im4, np.float32)
    sc = np.ascontiguousarray(scribs, np.uint8)
    reflib().ref_hostLevinLaplacian(P(a, _f), N, P(offs, _i), P(b, _f), lam, P(im4, _f),
                                    P(sc, _u8), W, H, W)
    return a, b


def levin_sym64(im3: np.ndarray, eps: float) -> np.ndarray:
    """FP64 affinities, 12 planes (k=1..12) of N doubles."""
    H, W, _ = im3.shape
    w = np.zeros((12, W * H), np.float64)
    im = np.ascontiguousarray(im3, np.float64)
    lib().orc_levin_sym64(P(w, _d), P(im, _d), eps, W, H)
    return w


def sym_to_bands64(w: np.ndarray, gamma: np.ndarray | None, W: int, H: int) -> np.ndarray:
    a = np.zeros((25, W * H), np.float64)
    g = None if gamma is None else np.ascontiguousarray(gamma, np.float64).ravel()
    lib().orc_sym_to_bands64(P(a, _d), P(np.ascontiguousarray(w), _d),
                             None if g is None else P(g, _d), W, H)
    return a


class Operator:
    """Keeps the arrays an orc_op points at alive."""

    def __init__(self, *, W: int, H: int, w=None, gamma=None, bands=None, offs=None):
        self.W, self.H, self.N = W, H, W * H
        if bands is not None:
            self.a = np.ascontiguousarray(bands, np.float64)
            self.offs = np.ascontiguousarray(offs, np.int32)
            self.op = _Op(1, W, H, self.N, None, None, P(self.a, _d), P(self.offs, _i), self.a.shape[0])
        else:
            self.w = np.ascontiguousarray(w, np.float64)
            self.g = np.ascontiguousarray(gamma, np.float64).ravel()
            self.op = _Op(0, W, H, self.N, P(self.w, _d), P(self.g, _d), None, None, 0)

    def apply(self, x: np.ndarray) -> np.ndarray:
        x = np.ascontiguousarray(x, np.float64).ravel()
        y = np.zeros(self.N, np.float64)
        if self.op.kind == 0:
            lib().orc_apply_sym64(P(y, _d), P(self.w, _d), P(self.g, _d), P(x, _d), self.W, self.H)
        else:
            lib().orc_apply_bands64(P(y, _d), P(self.a, _d), P(self.offs, _i), self.a.shape[0],
                                    P(x, _d), self.N)
        return y

    def cg(self, b, x0, rtol=0.0, maxit=1000, restart=0):
        x = np.ascontiguousarray(x0, np.float64).ravel().copy()
        bb = np.ascontiguousarray(b, np.float64).ravel()
        rel = C.c_double(0)
        it = lib().orc_cg64(C.byref(self.op), P(bb, _d), P(x, _d), rtol, maxit, restart, C.byref(rel))
        return x, it, rel.value

    def gd(self, b, x0, rtol=0.0, maxit=1000):
        x = np.ascontiguousarray(x0, np.float64).ravel().copy()
        bb = np.ascontiguousarray(b, np.float64).ravel()
        rel = C.c_double(0)
        it = lib().orc_gd64(C.byref(self.op), P(bb, _d), P(x, _d), rtol, maxit, C.byref(rel))
        return x, it, rel.value

    def jacobi(self, b, x0, omega=2.0 / 3.0, rtol=0.0, maxit=1000):
        x = np.ascontiguousarray(x0, np.float64).ravel().copy()
        bb = np.ascontiguousarray(b, np.float64).ravel()
        rel = C.c_double(0)
        it = lib().orc_jacobi64(C.byref(self.op), P(bb, _d), P(x, _d), omega, rtol, maxit, C.byref(rel))
        return x, it, rel.value


def gs_host(bands: np.ndarray, offs: np.ndarray, b: np.ndarray, x0: np.ndarray, iters: int,
            use_ref: bool = False) -> np.ndarray:
    nb, N = bands.shape
    pad = int(max(abs(int(o)) for o in offs)) + 32
    xp = np.zeros(N + 2 * pad, np.float32)
    xp[pad:pad + N] = x0
    a = np.ascontiguousarray(bands, np.float32)
    o = np.ascontiguousarray(offs, np.int32)
    bb = np.ascontiguousarray(b, np.float32)
    xptr = C.cast(C.c_void_p(xp.ctypes.data + 4 * pad), _f)
    if use_ref:
        reflib().ref_gaussSeidel_host(xptr, P(a, _f), N, P(o, _i), nb, N, P(bb, _f), iters)
    else:
        lib().orc_gs_host(xptr, P(a, _f), N, P(o, _i), nb, N, P(bb, _f), iters)
    return xp[pad:pad + N].copy()


def jacobi_host(bands: np.ndarray, offs: np.ndarray, b: np.ndarray, x0: np.ndarray, iters: int,
                omega: float = 2.0 / 3.0, use_ref: bool = False) -> np.ndarray:
    nb, N = bands.shape
    pad = int(max(abs(int(o)) for o in offs)) + 32
    xp = np.zeros(N + 2 * pad, np.float32)
    xp[pad:pad + N] = x0
    a = np.ascontiguousarray(bands, np.float32)
    o = np.ascontiguousarray(offs, np.int32)
    bb = np.ascontiguousarray(b, np.float32)
    xptr = C.cast(C.c_void_p(xp.ctypes.data + 4 * pad), _f)
    if use_ref:
        if reflib().ref_jacobi_host(xptr, P(a, _f), N, P(o, _i), nb, N, P(bb, _f), iters, pad, omega) != 0:
            raise ValueError("reference jacobi_host needs an even iteration count")
    else:
        lib().orc_jacobi_host(xptr, P(a, _f), N, P(o, _i), nb, N, P(bb, _f), iters, pad, omega)
    return xp[pad:pad + N].copy()


def compute_error(alpha: np.ndarray, gt: np.ndarray) -> float:
    H, W = gt.shape
    a = np.ascontiguousarray(alpha, np.float32).ravel()
    g = np.ascontiguousarray(gt, np.float32).ravel()
    return float(lib().orc_compute_error(P(a, _f), P(g, _f), W, H))


def levin_backward64(gw: np.ndarray, im3: np.ndarray, eps: float) -> np.ndarray:
    H, W, _ = im3.shape
    d = np.zeros(W * H * 3, np.float64)
    lib().orc_levin_backward64(P(d, _d), P(np.ascontiguousarray(gw, np.float64), _d),
                               P(np.ascontiguousarray(im3, np.float64), _d), eps, W, H)
    return d.reshape(H, W, 3)


def sym_edge_grad(lam: np.ndarray, alpha: np.ndarray, W: int, H: int) -> np.ndarray:
    """dloss/dw_k(i) = -(lam_i - lam_j)(alpha_i - alpha_j), j = i + (du_k, dv_k)."""
    lam = np.asarray(lam, np.float64).reshape(H, W)
    al = np.asarray(alpha, np.float64).reshape(H, W)
    gw = np.zeros((12, H, W), np.float64)
    for k in range(1, 13):
        dv = (k + 2) // 5
        du = k - 5 * dv
        u0, u1 = max(0, -du), min(W, W - du)
        v1 = H - dv
        if u1 <= u0 or v1 <= 0:
            continue
        li = lam[:v1, u0:u1]
        lj = lam[dv:dv + v1, u0 + du:u1 + du]
        ai = al[:v1, u0:u1]
        aj = al[dv:dv + v1, u0 + du:u1 + du]
        gw[k - 1, :v1, u0:u1] = -(li - lj) * (ai - aj)
    return gw.reshape(12, W * H)


def reference_adjoint(im3: np.ndarray, gamma: np.ndarray, s: np.ndarray, eps: float, gt: np.ndarray,
                      rtol: float = 1e-13, maxit: int = 200000):
    """FP64 forward + adjoint for loss = mean((alpha - gt)^2).

    alpha solves (L + diag(gamma)) alpha = gamma s with L = levin_sym64(im3);
    lam solves the same symmetric system for dloss/dalpha; the image gradient
    back-propagates the pair gradients -(lam_i - lam_j)(alpha_i - alpha_j)
    through the window statistics (levin_backward64) and
    dloss/dgamma_i = lam_i (s_i - alpha_i).  Returns a dict."""
    H, W, _ = im3.shape
    w = levin_sym64(im3, eps)
    g = np.asarray(gamma, np.float64).ravel()
    sv = np.asarray(s, np.float64).ravel()
    op = Operator(W=W, H=H, w=w, gamma=g)
    alpha, it_a, rel_a = op.cg(g * sv, np.full(W * H, 0.5), rtol=rtol, maxit=maxit)
    n = W * H
    dalpha = 2.0 * (alpha - np.asarray(gt, np.float64).ravel()) / n
    lam, it_l, rel_l = op.cg(dalpha, np.zeros(n), rtol=rtol, maxit=maxit)
    dI = levin_backward64(sym_edge_grad(lam, alpha, W, H), im3, eps)
    return {"alpha": alpha.reshape(H, W), "lam": lam.reshape(H, W), "dimage": dI,
            "dgamma": (lam * (sv - alpha)).reshape(H, W), "dalpha": dalpha.reshape(H, W),
            "loss": float(np.mean((alpha - np.asarray(gt, np.float64).ravel()) ** 2)),
            "iters": (it_a, it_l), "rel": (rel_a, rel_l), "w": w}
