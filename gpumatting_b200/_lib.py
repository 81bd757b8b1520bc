"""ctypes binding of libgpumat.so (include/gpumat.h).

The library is built in-tree (gpumatting_b200/libgpumat.so).  Importing this
module never falls back to anything else: if the library is missing or
fails to load, an ImportError says so.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libgpumat.so")

GM_OK = 0
GM_ERR_INVALID = 1
GM_ERR_CUDA = 2
GM_ERR_UNSUPPORTED = 3
GM_ERR_TIMEOUT = 4
GM_ERR_BREAKDOWN = 5
GM_ERR_NOT_CONVERGED = 6
GM_ERR_NOMEM = 7
STATUS_NAMES = {0: "OK", 1: "INVALID", 2: "CUDA", 3: "UNSUPPORTED", 4: "TIMEOUT", 5: "BREAKDOWN",
                6: "NOT_CONVERGED", 7: "NOMEM"}

GM_PREC_FP32, GM_PREC_FP16, GM_PREC_BF16 = 0, 1, 2
GM_SOLVER_CG, GM_SOLVER_GD, GM_SOLVER_JACOBI, GM_SOLVER_PCG, GM_SOLVER_MG = 0, 1, 2, 3, 4
GM_IMAGE_RGB8, GM_IMAGE_RGBA32F = 0, 1
GM_ASSEMBLY_FP64, GM_ASSEMBLY_REFERENCE = 0, 1


class BandedMatrix(C.Structure):
    """BandedMatrix.h:23-38."""
    _fields_ = [("a", C.c_void_p), ("apitch", C.c_size_t), ("bands", C.c_void_p), ("nbands", C.c_int),
                ("rows", C.c_int), ("cols", C.c_int)]


class GmImage(C.Structure):
    _fields_ = [("data", C.c_void_p), ("format", C.c_int), ("pitch_bytes", C.c_size_t)]


class GmScribbles(C.Structure):
    _fields_ = [("map", C.c_void_p), ("map_pitch", C.c_size_t), ("gamma_value", C.c_float),
                ("gamma_map", C.c_void_p), ("s_map", C.c_void_p)]


class GmPnm(C.Structure):
    _fields_ = [("w", C.c_int), ("h", C.c_int), ("channels", C.c_int), ("maxval", C.c_int),
                ("data", C.POINTER(C.c_ubyte))]


class GmLevinStore(C.Structure):
    _fields_ = [("W", C.c_int), ("H", C.c_int), ("pitch", C.c_int), ("precision", C.c_int), ("w", C.c_void_p),
                ("w32", C.c_void_p), ("gamma", C.c_void_p), ("b", C.c_void_p), ("d", C.c_void_p),
                ("d32", C.c_void_p), ("owns", C.c_int), ("plane_stride", C.c_size_t)]


class GmSolveParams(C.Structure):
    _fields_ = [("solver", C.c_int), ("rtol", C.c_double), ("max_iters", C.c_int), ("restart", C.c_int),
                ("replace_every", C.c_int), ("omega", C.c_float), ("use_low", C.c_int), ("timeout_s", C.c_double),
                ("ctas_per_sm", C.c_int), ("strip_width", C.c_int), ("inject", C.c_int), ("mg_omega", C.c_float),
                ("mg_scale", C.c_float)]


class GmSolveInfo(C.Structure):
    _fields_ = [("status", C.c_int), ("iters", C.c_int), ("replacements", C.c_int), ("rel_residual", C.c_double),
                ("bnorm", C.c_double), ("kernel_ms", C.c_float), ("grid", C.c_int), ("where", C.c_int),
                ("solver", C.c_int)]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


# name -> (restype, argtypes); every symbol include/gpumat.h declares.
_vp, _i, _f, _d, _sz = C.c_void_p, C.c_int, C.c_float, C.c_double, C.c_size_t
SIGNATURES = {
    "gm_last_status": (_i, []),
    "gm_last_error": (C.c_char_p, []),
    "gm_version": (C.c_char_p, []),
    "bmCopyToDevice": (None, [C.POINTER(BandedMatrix), C.POINTER(BandedMatrix)]),
    "bmDeviceFree": (None, [C.POINTER(BandedMatrix)]),
    "vecDeviceMalloc": (None, [C.POINTER(C.c_void_p), _i, _i, _i]),
    "vecCopyToDevice": (None, [C.POINTER(C.c_void_p), _vp, _i, _i, _i]),
    "vecDeviceFree": (None, [_vp, _i]),
    "cgSolve": (None, [_vp, BandedMatrix, _vp, _i, _i, _i]),
    "gradSolve": (None, [_vp, BandedMatrix, _vp, _i, _i]),
    "jacobi": (None, [_vp, BandedMatrix, _vp, _f, _i, _i]),
    "hostLevinLaplacian": (None, [BandedMatrix, _vp, _f, _vp, _vp, _i, _i, _sz]),
    "gaussSeidel_host": (None, [_vp, C.POINTER(BandedMatrix), _vp, _sz]),
    "jacobi_host": (None, [_vp, C.POINTER(BandedMatrix), _vp, _sz, _i, _f]),
    "gm_gs_host_levels": (_i, [C.POINTER(BandedMatrix)]),
    "computeError": (None, [_vp, _vp, _i, _i]),
    "gm_bm_ax": (_i, [_vp, BandedMatrix, _vp, _vp]),
    "gm_bm_axpy": (_i, [_vp, BandedMatrix, _vp, _vp, _i, _vp]),
    "gm_jacobi_step": (_i, [_vp, _vp, BandedMatrix, _vp, _f, _vp]),
    "gm_inner_prod": (_i, [_vp, _vp, _vp, _i, _vp]),
    "gm_inner_prod_f64": (_i, [_vp, _vp, _vp, _i, _vp]),
    "gm_inner_prod_f64_noalloc": (_i, [_vp, _vp, _vp, _i, _vp]),
    "gm_vec_add": (_i, [_vp, _vp, _vp, _i, _vp]),
    "gm_vec_sub": (_i, [_vp, _vp, _vp, _i, _vp]),
    "gm_vec_scale_const": (_i, [_vp, _vp, _f, _i, _vp]),
    "gm_vec_scale": (_i, [_vp, _vp, _vp, _i, _vp]),
    "gm_levin_band_offsets": (None, [_i, C.POINTER(C.c_int)]),
    "gm_levin_pad": (_i, [_i]),
    "gm_compute_error": (_i, [C.POINTER(C.c_double), _vp, _vp, _i, _i, _vp]),
    "gm_cg_dots4": (_i, [_vp, _vp, _i, _vp, _i, _vp, _i, _i, _i, _vp]),
    "gm_cg_update": (_i, [_vp, _i, _vp, _i, _vp, _i, _vp, _i, _i, _i, _f, _f, _i, _vp]),
    "gm_cg_scalars": (_i, [_vp, _vp, _vp, _vp]),
    "gm_cg_update_dev": (_i, [_vp, _i, _vp, _i, _vp, _i, _vp, _i, _i, _i, _vp, _vp]),
    "gm_levin_store_alloc": (_i, [C.POINTER(GmLevinStore), _i, _i, _i]),
    "gm_levin_store_free": (_i, [C.POINTER(GmLevinStore)]),
    "gm_levin_assemble": (_i, [C.POINTER(GmLevinStore), C.POINTER(GmImage), C.POINTER(GmScribbles), _d,
                               C.POINTER(BandedMatrix), _vp, _vp]),
    "gm_levin_assemble_bands25": (_i, [_vp, _sz, _vp, C.POINTER(GmImage), C.POINTER(GmScribbles), _d, _i, _i, _i,
                                       _vp]),
    "gm_default_params": (None, [C.POINTER(GmSolveParams)]),
    "gm_levin_solve": (_i, [C.POINTER(GmLevinStore), _vp, C.POINTER(GmSolveParams), C.POINTER(GmSolveInfo), _vp]),
    "gm_batch_create": (_i, [C.POINTER(C.c_void_p), _i, C.POINTER(C.c_int), C.POINTER(C.c_int), _i]),
    "gm_batch_destroy": (_i, [_vp]),
    "gm_batch_store": (_i, [_vp, _i, C.POINTER(GmLevinStore)]),
    "gm_batch_assemble": (_i, [_vp, _i, C.POINTER(GmImage), C.POINTER(GmScribbles), C.c_double, _vp]),
    "gm_batch_tune": (_i, [_vp, C.POINTER(GmSolveParams), _i, _vp]),
    "gm_batch_solve": (_i, [_vp, C.POINTER(C.c_void_p), C.POINTER(GmSolveParams), C.POINTER(GmSolveInfo), _vp]),
    "gm_batch_info": (_i, [_vp, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int),
                           C.POINTER(C.c_int)]),
    "gm_pnm_read": (_i, [C.c_char_p, C.POINTER(GmPnm)]),
    "gm_pnm_free": (None, [C.POINTER(GmPnm)]),
    "gm_pgm_write": (_i, [C.c_char_p, _i, _i, _vp, C.c_char_p, _i]),
    "gm_rgb8_to_float4": (_i, [_vp, _vp, _i, _i, _vp]),
    "gm_alpha_to_gray8": (_i, [_vp, _vp, _i, _vp]),
    "gm_bands_dump": (_i, [C.c_char_p, BandedMatrix, _i]),
    "gm_levin_restrict": (_i, [C.POINTER(GmLevinStore), C.POINTER(GmScribbles), _vp]),
    "gm_levin_apply": (_i, [C.POINTER(GmLevinStore), _vp, _i, _vp, _i, _i, _vp]),
    "gm_levin_solve_rhs": (_i, [C.POINTER(GmLevinStore), _vp, _vp, C.POINTER(GmSolveParams),
                                C.POINTER(GmSolveInfo), _vp]),
    "gm_levin_adjoint": (_i, [C.POINTER(GmLevinStore), C.POINTER(GmImage), C.POINTER(GmScribbles), C.c_double,
                              _vp, _vp, _vp, _vp, C.c_size_t, _i, _vp, C.POINTER(GmSolveParams),
                              C.POINTER(GmSolveInfo), _vp]),
    "gm_banded_solve": (_i, [BandedMatrix, _i, _vp, _i, _vp, C.POINTER(GmSolveParams), C.POINTER(GmSolveInfo),
                             _vp]),
    "gm_levin_mg_levels": (_i, [_i, _i, C.POINTER(C.c_int), C.POINTER(C.c_int), _i]),
    "gm_levin_solve_mg_many": (_i, [C.POINTER(C.POINTER(GmLevinStore)), C.POINTER(C.c_void_p), _i,
                                    C.POINTER(GmSolveParams), C.POINTER(GmSolveInfo), _vp]),
    "gm_levin_mg_inspect": (_i, [C.POINTER(GmLevinStore), _i, _vp, _vp, _i, _vp, _vp, _vp]),
}

_lib = None


def load() -> C.CDLL:
    """Loads libgpumat.so; raises ImportError when it is absent."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: run `python -m gpumatting_b200.build` (needs nvcc)")
    lib = C.CDLL(LIB_PATH)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


class GmError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {msg}")
        self.status = status


def check(status: int) -> int:
    if status != GM_OK:
        raise GmError(status, load().gm_last_error().decode(errors="replace"))
    return status


def last_error() -> str:
    return load().gm_last_error().decode(errors="replace")


def default_params(**kw) -> GmSolveParams:
    p = GmSolveParams()
    load().gm_default_params(C.byref(p))
    for k, v in kw.items():
        if not hasattr(p, k):
            raise AttributeError(k)
        setattr(p, k, v)
    return p
