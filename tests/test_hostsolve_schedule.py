"""The level schedule behind the gaussSeidel_host drop-in (host code only, no
GPU): levels follow level(i) = 1 + max level(i + o) over the backward
offsets o < 0 whose coefficient is non-zero, restated here in Python."""
import numpy as np

from conftest import load_golden


def py_levels(a: np.ndarray, offs: np.ndarray) -> int:
    nb, n = a.shape
    mid = nb // 2
    lev = np.zeros(n, np.int64)
    back = [j for j in range(nb) if j != mid and offs[j] < 0]
    for i in range(n):
        best = 0
        for j in back:
            k = i + int(offs[j])
            if k >= 0 and a[j, i] != 0.0:
                best = max(best, lev[k] + 1)
        lev[i] = best
    return int(lev.max()) + 1 if n else 0


def test_levels_of_the_levin_fixture():
    from gpumatting_b200 import api
    from oracle import oracle as O

    g = load_golden("s37x29")
    H, W = g["scribbles"].shape
    offs = O.levin_offsets(W)
    got = api.gs_host_levels(g["a"], offs)
    assert got == py_levels(g["a"], offs)
    # the anti-diagonals u + 3v, a little fewer at the right edge
    assert W + 3 * H - 6 <= got <= W + 3 * H - 3


def test_levels_of_other_patterns():
    from gpumatting_b200 import api

    n = 500
    tri = np.ones((3, n), np.float32)
    assert api.gs_host_levels(tri, [-1, 0, 1]) == n  # one chain
    # zero couplings do not count: every other row decoupled from its predecessor
    tri[0, 1::2] = 0.0
    assert api.gs_host_levels(tri, [-1, 0, 1]) == 2
    rng = np.random.default_rng(3)
    offs = np.array([-9, -4, -1, 0, 2, 7], np.int32)
    a = (rng.random((6, n)) < 0.6).astype(np.float32) * rng.random((6, n)).astype(np.float32)
    assert api.gs_host_levels(a, offs) == py_levels(a, offs)
