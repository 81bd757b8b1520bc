"""Device side of the data formats: ppmread_float4's normalisation and
pgmwrite_float's quantisation as kernels, the A.bin dump of device bands,
and a file-to-file run (PPM + PGM scribbles in, alpha.pgm out)."""
import numpy as np
import pytest

from gpumatting_b200 import api
from gpumatting_b200.synth import make_problem
from tests.gpu_util import torch_cuda
from tests.test_io import _write_pnm

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("maxval", [255, 200, 1])
def test_rgb8_to_float4_matches_ppmread_float4(orc, tmp_path, maxval):
    torch = torch_cuda()
    rng = np.random.default_rng(maxval)
    arr = rng.integers(0, maxval + 1, size=(21, 34, 3)).astype(np.uint8)
    path = tmp_path / "img.ppm"
    _write_pnm(path, arr, maxval)
    got = api.rgb8_to_float4(torch.from_numpy(arr).cuda(), maxval).cpu().numpy()
    if orc.ref_available():
        ref = orc.ref_ppmread_float4(path)
    else:
        ref = np.concatenate([arr.astype(np.float32) / np.float32(maxval), np.ones((21, 34, 1), np.float32)], 2)
    assert np.array_equal(got.view(np.uint32), ref.view(np.uint32))


def test_alpha_quantisation_and_pgm_bytes(orc, tmp_path):
    torch = torch_cuda()
    rng = np.random.default_rng(9)
    alpha = rng.uniform(-0.3, 1.3, size=(40, 57)).astype(np.float32)
    alpha[0, :6] = [0.0, 1.0, 0.5, 1.0 / 255, 254.5 / 255, 0.99999994]
    g = api.alpha_to_gray8(torch.from_numpy(alpha).cuda()).cpu().numpy()
    want = np.where(alpha < 0, 0, np.where(alpha > 1, 255, (np.float32(255) * alpha).astype(np.uint8)))
    assert np.array_equal(g, want.astype(np.uint8))
    if orc.ref_available():
        ours, ref = tmp_path / "alpha.pgm", tmp_path / "ref.pgm"
        api.write_alpha_pgm(ours, torch.from_numpy(alpha).cuda())
        orc.ref_pgmwrite_float(ref, alpha, None, True)
        assert ours.read_bytes() == ref.read_bytes()


def test_band_dump_from_device(tmp_path):
    torch = torch_cuda()
    p = make_problem(33, 21, 2)
    a, b = api.levin_bands25(torch.from_numpy(p.image).cuda(), torch.from_numpy(p.scribbles).cuda(), eps=p.eps)
    Lm = api.DeviceBandedMatrix(a, torch.tensor(api.levin_band_offsets(33), device="cuda"), 33 * 21)
    path = tmp_path / "A.bin"
    api.dump_bands(path, Lm)
    assert np.array_equal(np.fromfile(path, np.float32).reshape(25, -1), a[:, :33 * 21].cpu().numpy())


def test_file_in_alpha_pgm_out(tmp_path):
    """PPM + scribble PGM on disk -> store from the RGB bytes and from the
    normalised float4 image -> solve -> alpha.pgm.  The FP64 assembly
    normalises bytes exactly while the float4 image is rounded to FP32 first,
    so the two stores agree to rounding and their mattes to 1e-4."""
    torch = torch_cuda()
    p = make_problem(120, 90, 6)
    _write_pnm(tmp_path / "img.ppm", p.image)
    _write_pnm(tmp_path / "scribs.pgm", p.scribbles)
    img, mv = api.read_pnm(tmp_path / "img.ppm")
    scr, _ = api.read_pnm(tmp_path / "scribs.pgm")
    assert mv == 255 and np.array_equal(img, p.image) and np.array_equal(scr, p.scribbles)
    img_d, scr_d = torch.from_numpy(img).cuda(), torch.from_numpy(scr).cuda()
    s1 = api.LevinStore(120, 90, "fp16").assemble(img_d, scr_d, eps=p.eps)
    s2 = api.LevinStore(120, 90, "fp16").assemble(api.rgb8_to_float4(img_d, mv), scr_d, eps=p.eps)
    for name in ("gamma", "b"):
        assert torch.equal(s1.planes(name), s2.planes(name)), name
    alpha = torch.full((90, 120), 0.5, device="cuda")
    alpha2 = torch.full((90, 120), 0.5, device="cuda")
    assert s1.solve(alpha, "cg", rtol=1e-8, max_iters=20000).status == 0
    assert s2.solve(alpha2, "cg", rtol=1e-8, max_iters=20000).status == 0
    assert float((alpha - alpha2).abs().max()) <= 1e-4
    api.write_alpha_pgm(tmp_path / "alpha.pgm", alpha)
    g, _ = api.read_pnm(tmp_path / "alpha.pgm")
    assert np.array_equal(g, api.alpha_to_gray8(alpha).cpu().numpy())
