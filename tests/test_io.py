"""PNM in, alpha.pgm and A.bin out: the host side of gm_io against the
reference's own ppm.h (compiled into oracle/_ref) on the same files.

Readers: identical bytes, size and maxval for binary and ASCII graymaps and
pixmaps with comment lines; writer: identical file bytes; band dump: the
layout of main.cu:334-355.  Malformed files are errors, not aborts."""
import numpy as np
import pytest

from gpumatting_b200 import _lib as L
from gpumatting_b200 import api


def _write_pnm(path, arr, maxval=255, binary=True, comments=("made by the test",)):
    color = arr.ndim == 3
    magic = ("P6" if binary else "P3") if color else ("P5" if binary else "P2")
    h, w = arr.shape[:2]
    with open(path, "wb") as f:
        f.write(f"{magic}\n".encode())
        for c in comments:
            f.write(f"# {c}\n".encode())
        f.write(f"{w} {h}\n{maxval}\n".encode())
        if binary:
            f.write(np.ascontiguousarray(arr, np.uint8).tobytes())
        else:
            vals = np.asarray(arr).ravel()
            for k in range(0, len(vals), 17):  # ragged line breaks
                f.write((" ".join(str(int(v)) for v in vals[k:k + 17]) + "\n").encode())


CASES = [((37, 29, 3), 255, True), ((5, 7, 3), 200, True), ((16, 12, 3), 255, False), ((9, 4, 3), 90, False),
         ((64, 48), 255, True), ((3, 3), 255, False), ((1, 1, 3), 255, True)]


@pytest.mark.parametrize("shape,maxval,binary", CASES)
def test_pnm_reader_matches_reference(orc, tmp_path, shape, maxval, binary):
    rng = np.random.default_rng(shape[0] * 1000 + shape[1] + maxval + int(binary))
    size = (shape[1], shape[0], 3) if len(shape) == 3 else (shape[1], shape[0])  # shape is (W, H[, 3])
    arr = rng.integers(0, maxval + 1, size=size).astype(np.uint8)
    path = tmp_path / ("img.ppm" if arr.ndim == 3 else "img.pgm")
    _write_pnm(path, arr, maxval, binary)
    got, mv = api.read_pnm(path)
    assert got.shape == arr.shape and mv == maxval and np.array_equal(got, arr)
    if orc.ref_available():
        ref, ref_mv = orc.ref_read_pnm(path, arr.ndim == 3)
        assert np.array_equal(got, ref)
        if arr.ndim == 3:
            assert ref_mv == mv


@pytest.mark.parametrize("binary,comment", [(True, None), (True, "alpha matte"), (False, None)])
def test_pgm_writer_bytes_match_reference(orc, tmp_path, binary, comment):
    if not orc.ref_available():
        pytest.skip("reference CPU code not built")
    rng = np.random.default_rng(4)
    alpha = rng.uniform(-0.3, 1.3, size=(23, 31)).astype(np.float32)
    alpha[0, :5] = [0.0, 1.0, 0.5, 1.0 / 255, 254.5 / 255]
    # the reference's quantisation (ppm.h:430-451), restated on the host
    g = np.where(alpha < 0, 0, np.where(alpha > 1, 255, (np.float32(255) * alpha).astype(np.uint8))).astype(np.uint8)
    ours, ref = tmp_path / "ours.pgm", tmp_path / "ref.pgm"
    api.write_pgm(ours, g, comment, binary)
    assert orc.ref_pgmwrite_float(ref, alpha, comment, binary) == 0
    assert ours.read_bytes() == ref.read_bytes()
    back, _ = api.read_pnm(ours)
    assert np.array_equal(back, g)


def test_band_dump_layout(tmp_path):
    rows, nb, apitch = 50, 25, 64
    a = np.random.default_rng(1).normal(size=(nb, apitch)).astype(np.float32)
    offs = np.arange(nb, dtype=np.int32)
    bm = L.BandedMatrix(a.ctypes.data, apitch, offs.ctypes.data, nb, rows, rows)
    path = tmp_path / "A.bin"
    L.check(L.load().gm_bands_dump(str(path).encode(), bm, 0))
    assert np.array_equal(np.fromfile(path, np.float32), a[:, :rows].ravel())


def test_malformed_files_are_errors(tmp_path):
    bad = tmp_path / "x.ppm"
    bad.write_bytes(b"P9\n2 2\n255\n" + bytes(12))
    for content in (b"P9\n2 2\n255\n" + bytes(12), b"P6\n2 2\n255\n" + bytes(5), b"P6\n2 2\n300\n" + bytes(12),
                    b"P3\n2 1\n255\n1 2 3 4\n", b"hello"):
        bad.write_bytes(content)
        with pytest.raises(L.GmError) as e:
            api.read_pnm(bad)
        assert e.value.status == L.GM_ERR_INVALID
    with pytest.raises(L.GmError):
        api.read_pnm(tmp_path / "missing.pgm")
