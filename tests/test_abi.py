"""libgpumat.so loads on a machine without a GPU and exports every symbol
include/gpumat.h declares.  Only host-side helpers are called here."""
import ctypes
import os
import re

import numpy as np

from conftest import ROOT


def header_functions():
    src = open(os.path.join(ROOT, "include", "gpumat.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    src = re.sub(r"//[^\n]*", "", src)
    names = set()
    for m in re.finditer(r"\b([A-Za-z_][A-Za-z0-9_]*)\s*\(([^;{}]*)\)\s*;", src):
        name = m.group(1)
        if name in {"if", "while", "for", "return", "sizeof"}:
            continue
        names.add(name)
    return names


def test_library_loads_and_exports_header():
    from gpumatting_b200 import _lib

    lib = _lib.load()
    names = header_functions()
    assert len(names) >= 30
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    assert set(names) == set(_lib.SIGNATURES), set(names) ^ set(_lib.SIGNATURES)


def test_no_oracle_in_product_library():
    from gpumatting_b200 import _lib

    data = open(_lib.LIB_PATH, "rb").read()
    assert b"orc_" not in data and b"libgmref" not in data and b"liborc" not in data


def test_host_helpers(orc):
    from gpumatting_b200 import _lib, api

    for W in (3, 5, 64, 1920):
        assert np.array_equal(api.levin_band_offsets(W), orc.levin_offsets(W))
        assert api.levin_pad(W) == ((2 * W + 2) // 32) * 32 + 32
    p = _lib.default_params()
    assert p.solver == _lib.GM_SOLVER_CG and p.rtol == 1e-6 and p.max_iters == 5000 and p.replace_every == 50
    assert abs(p.omega - 2.0 / 3.0) < 1e-7
    assert _lib.load().gm_version().startswith(b"gpumatting_b200")


def test_struct_layout_matches_reference():
    """BandedMatrix.h:23-38 field order and sizes on LP64."""
    from gpumatting_b200._lib import BandedMatrix

    assert ctypes.sizeof(BandedMatrix) == 40
    assert BandedMatrix.apitch.offset == 8 and BandedMatrix.bands.offset == 16
    assert BandedMatrix.nbands.offset == 24 and BandedMatrix.rows.offset == 28 and BandedMatrix.cols.offset == 32


def test_noalloc_dot_refuses_bad_operands_before_the_call():
    """The Python wrapper checks dtype, device and length before handing
    pointers to the library: the entry point writes one FP64 value into out
    and reads len floats from x and y, so a float32 or host out, or a short
    y, would be an out-of-bounds access on the device."""
    import pytest
    import torch

    from gpumatting_b200 import api

    x = torch.zeros(8)
    out = torch.zeros(1, dtype=torch.float64)
    with pytest.raises(ValueError):  # host tensors
        api.inner_prod_noalloc(x, x, out)
    with pytest.raises(TypeError):
        api.inner_prod_noalloc(x.double(), x.double(), out)
    with pytest.raises((TypeError, ValueError)):
        api.inner_prod_noalloc(x, x, None)
    with pytest.raises((TypeError, ValueError)):
        api.inner_prod_noalloc(x, torch.zeros(4), out)
