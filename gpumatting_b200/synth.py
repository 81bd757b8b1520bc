"""Seeded synthetic matting problems (image, scribbles, ground-truth alpha).

The reference ships one sample image (an 800x552 photo with a scribble map and
a ground-truth matte); the workloads this package is measured on are
synthetic stand-ins with a fixed recipe so every run sees identical inputs:

* foreground and background are two 8x8 grids of uniform[0,255] RGB values,
  bilinearly upsampled to W x H;
* the ground-truth alpha is ``sigmoid(8 z)`` where ``z`` is uniform[-1,1]
  noise Gaussian-smoothed with ``sigma`` (6 px by default, 24 px for the
  4096x4096 case) and standardised to zero mean and unit variance;
* the image is ``clip(round(alpha F + (1 - alpha) B + N(0, 4^2)))`` as uint8;
* scribbles are 20 random smooth strokes, 7 px wide, whose length is chosen
  so that about ``scrib_frac`` of the pixels are marked; a stroke pixel is
  marked 0 (background) where alpha < 0.02, 255 (foreground) where
  alpha > 0.98 and left 128 (unknown) elsewhere.  This is the 0/128/255
  convention of the reference's scribble map (Matting.cu:205-216).

``gamma`` is the per-pixel scribble weight (``gamma_value`` on scribbled
pixels, 0 elsewhere) and ``s`` the scribble target (1 on foreground
scribbles), so the system solved is ``(L + diag(gamma)) alpha = gamma * s``.
"""
from __future__ import annotations

import dataclasses

import numpy as np


@dataclasses.dataclass
class Problem:
    W: int
    H: int
    image: np.ndarray      # (H, W, 3) uint8
    scribbles: np.ndarray  # (H, W) uint8 in {0, 128, 255}
    alpha_gt: np.ndarray   # (H, W) float64
    gamma: np.ndarray      # (H, W) float32 per-pixel scribble weight
    s: np.ndarray          # (H, W) float32 scribble target in {0, 1}
    eps: float
    seed: int

    @property
    def n(self) -> int:
        return self.W * self.H

    def image_float4(self) -> np.ndarray:
        """RGBA float32 image in [0,1] with w=1, as ppm.h:309-333 builds it."""
        out = np.ones((self.H, self.W, 4), np.float32)
        out[..., :3] = self.image.astype(np.float32) / np.float32(255.0)
        return out

    def rhs(self) -> np.ndarray:
        return (self.gamma * self.s).astype(np.float32)


def _bilinear_field(rng: np.random.Generator, W: int, H: int) -> np.ndarray:
    g = rng.uniform(0.0, 255.0, size=(8, 8, 3))
    ys = np.linspace(0.0, 7.0, H)
    xs = np.linspace(0.0, 7.0, W)
    y0 = np.clip(np.floor(ys).astype(np.int64), 0, 6)
    x0 = np.clip(np.floor(xs).astype(np.int64), 0, 6)
    fy = (ys - y0)[:, None, None]
    fx = (xs - x0)[None, :, None]
    a = g[y0][:, x0]
    b = g[y0][:, x0 + 1]
    c = g[y0 + 1][:, x0]
    d = g[y0 + 1][:, x0 + 1]
    return a * (1 - fx) * (1 - fy) + b * fx * (1 - fy) + c * (1 - fx) * fy + d * fx * fy


def _strokes(rng: np.random.Generator, W: int, H: int, eligible: np.ndarray,
             scrib_frac: float, n_strokes: int = 20, width: int = 7) -> np.ndarray:
    """Boolean mask of ``n_strokes`` smooth random strokes ``width`` px wide.

    The stroke length is set in two passes: a first guess from the eligible
    fraction, then one rescale by the marked fraction the guess produced.
    """
    import scipy.ndimage as ndi

    starts = rng.uniform(0.0, 1.0, size=(n_strokes, 2)) * np.array([W, H])
    ang0 = rng.uniform(0.0, 2.0 * np.pi, size=n_strokes)
    bend = rng.normal(0.0, 1.0, size=n_strokes)
    r = width // 2
    struct = np.ones((2 * r + 1, 2 * r + 1), bool)

    def draw(length: int) -> np.ndarray:
        centre = np.zeros((H, W), bool)
        t = np.arange(length)
        for s in range(n_strokes):
            a = ang0[s] + bend[s] * 2.0 * t / length
            px = np.mod(starts[s, 0] + np.cumsum(np.cos(a)), W).astype(np.int64)
            py = np.mod(starts[s, 1] + np.cumsum(np.sin(a)), H).astype(np.int64)
            centre[np.clip(py, 0, H - 1), np.clip(px, 0, W - 1)] = True
        return ndi.binary_dilation(centre, structure=struct)

    e = max(float(eligible.mean()), 1e-3)
    length = max(8, int(scrib_frac * W * H / (n_strokes * width * e)))
    got = float((draw(length) & eligible).mean())
    length = max(8, int(length * scrib_frac / max(got, 1e-6)))
    return draw(length)


def make_problem(W: int, H: int, seed: int = 0, *, sigma: float | None = None,
                 scrib_frac: float | None = None, eps: float | None = None,
                 gamma_value: float = 100.0) -> Problem:
    """Build the seeded synthetic problem of size W x H.

    Defaults follow the workload family: sigma 6 px, 10% scribbles and
    eps 1e-5, except for images of 4096x4096 and larger, which use sigma 24,
    5% scribbles and eps 1e-7.
    """
    import scipy.ndimage as ndi

    large = W * H >= 4096 * 4096
    if sigma is None:
        sigma = 24.0 if large else 6.0
    if scrib_frac is None:
        scrib_frac = 0.05 if large else 0.10
    if eps is None:
        eps = 1e-7 if large else 1e-5
    rng = np.random.default_rng(seed)
    F = _bilinear_field(rng, W, H)
    B = _bilinear_field(rng, W, H)
    z = ndi.gaussian_filter(rng.uniform(-1.0, 1.0, size=(H, W)), sigma, mode="reflect")
    z = (z - z.mean()) / max(float(z.std()), 1e-12)
    alpha = 1.0 / (1.0 + np.exp(-8.0 * z))
    img = alpha[..., None] * F + (1.0 - alpha[..., None]) * B + rng.normal(0.0, 4.0, size=(H, W, 3))
    img = np.clip(np.rint(img), 0, 255).astype(np.uint8)
    fg = alpha > 0.98
    bg = alpha < 0.02
    mask = _strokes(rng, W, H, fg | bg, scrib_frac)
    scr = np.full((H, W), 128, np.uint8)
    scr[mask & bg] = 0
    scr[mask & fg] = 255
    gamma = np.where(scr != 128, np.float32(gamma_value), np.float32(0.0)).astype(np.float32)
    s = (scr == 255).astype(np.float32)
    return Problem(W, H, img, scr, alpha, gamma, s, float(eps), seed)


def batch_sizes(count: int = 64, lo: int = 256, hi: int = 1024, seed: int = 0) -> list[tuple[int, int]]:
    """Seeded (W, H) pairs with W and H uniform in [lo, hi]."""
    rng = np.random.default_rng(seed)
    wh = rng.integers(lo, hi + 1, size=(count, 2))
    return [(int(w), int(h)) for w, h in wh]
