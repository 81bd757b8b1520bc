"""Generates the golden fixtures in tests/golden/ by running the reference's
own CPU code (oracle/_ref/libgmref.so, compiled by `make -C oracle ref`
from the reference tree).

Fixtures:
  levin_ref_<case>.npz   inputs (im4 float4 image, scribbles, lambda) and the
                         reference hostLevinLaplacian outputs (25 bands, b),
                         Matting.cu:39-219 with its hard-coded gamma = 1.
  solve_host_<case>.npz  gaussSeidel_host / jacobi_host iterates
                         (Solve.cpp:3-85) from x0 = 0.5 on one of those
                         matrices.

The data05 case is a crop of the reference's sample image data/05.ppm and
its scribbles data/05_scribs.pgm.  Run from the repository root:
    python tests/golden/make_golden.py
"""
from __future__ import annotations

import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from gpumatting_b200.synth import make_problem  # noqa: E402
from oracle import oracle as O  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))
REF = O.REF_TREE


def read_pnm(path: str) -> np.ndarray:
    with open(path, "rb") as f:
        data = f.read()
    tokens = []
    pos = 0
    while len(tokens) < 4:
        while data[pos:pos + 1].isspace():
            pos += 1
        if data[pos:pos + 1] == b"#":
            while data[pos:pos + 1] not in (b"\n", b""):
                pos += 1
            continue
        start = pos
        while not data[pos:pos + 1].isspace():
            pos += 1
        tokens.append(data[start:pos])
    pos += 1
    magic, w, h, _ = tokens[0], int(tokens[1]), int(tokens[2]), int(tokens[3])
    ch = 3 if magic == b"P6" else 1
    arr = np.frombuffer(data[pos:pos + w * h * ch], np.uint8)
    return arr.reshape(h, w, ch) if ch == 3 else arr.reshape(h, w)


def im4_from_rgb(rgb: np.ndarray) -> np.ndarray:
    out = np.ones(rgb.shape[:2] + (4,), np.float32)
    out[..., :3] = rgb.astype(np.float32) / np.float32(255.0)
    return out


def cases():
    for name, (W, H, seed, lam) in {
        "s16x12": (16, 12, 3, 1e-5),
        "s37x29": (37, 29, 4, 1e-2),
        "s64x48": (64, 48, 5, 1e-5),
        "s3x3": (3, 3, 6, 1e-5),
        "s8x2": (8, 2, 7, 1e-5),
        "s5x7": (5, 7, 8, 1e-3),
    }.items():
        p = make_problem(W, H, seed)
        yield name, p.image_float4(), p.scribbles, lam
    img = os.path.join(REF, "data", "05.ppm")
    scr = os.path.join(REF, "data", "05_scribs.pgm")
    if os.path.exists(img):
        rgb = read_pnm(img)
        sc = read_pnm(scr)
        # the 64x48 window with the most scribbled and unknown pixels (no
        # window of that size holds both scribble values in this sample)
        best = None
        for v0 in range(0, sc.shape[0] - 48, 8):
            for u0 in range(0, sc.shape[1] - 64, 8):
                w = sc[v0:v0 + 48, u0:u0 + 64]
                score = min((w != 128).sum(), (w == 128).sum())
                if best is None or score > best[0]:
                    best = (score, u0, v0)
        _, u0, v0 = best
        yield "data05", im4_from_rgb(rgb[v0:v0 + 48, u0:u0 + 64]), np.ascontiguousarray(sc[v0:v0 + 48, u0:u0 + 64]), 1e-2


def main():
    O.build(ref=True)
    if not O.ref_available():
        raise SystemExit("oracle/_ref/libgmref.so was not built (reference tree missing?)")
    for name, im4, sc, lam in cases():
        a, b = O.ref_levin(im4, sc, lam)
        np.savez_compressed(os.path.join(OUT, f"levin_ref_{name}.npz"), im4=im4, scribbles=sc, lam=np.float32(lam),
                            a=a, b=b)
        print("wrote", name, a.shape)
        if name == "s37x29":
            H, W = sc.shape
            offs = O.levin_offsets(W)
            x0 = np.full(W * H, 0.5, np.float32)
            gs = O.gs_host(a, offs, b, x0, 10, use_ref=True)
            jac = O.jacobi_host(a, offs, b, x0, 10, use_ref=True)
            np.savez_compressed(os.path.join(OUT, f"solve_host_{name}.npz"), x0=x0, iters=np.int32(10), gs=gs,
                                jacobi=jac, omega=np.float32(2.0 / 3.0))
            print("wrote solve_host", name)


if __name__ == "__main__":
    main()
