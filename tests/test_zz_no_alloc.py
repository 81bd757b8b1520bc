"""Allocation-free dot product against the allocating entry point.

gm_inner_prod_f64_noalloc keeps its partial sums in a fixed device array in
the library; it must give exactly the bits gm_inner_prod_f64 gives, on two
calls in a row (the second call reuses the array the first one wrote).  The
file name sorts last so the check also runs after every other GPU test has
used the library.
"""
import numpy as np
import pytest

from gpumatting_b200 import api
from tests.gpu_util import torch_cuda

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n", [1, 1000, 2_073_600, 16_777_216])
def test_noalloc_matches_allocating_dot_twice(n):
    torch = torch_cuda()
    g = torch.Generator(device="cuda").manual_seed(n)
    xs = [torch.rand(n, device="cuda", generator=g) - 0.5 for _ in range(2)]
    ys = [torch.rand(n, device="cuda", generator=g) - 0.5 for _ in range(2)]
    out = torch.empty(1, dtype=torch.float64, device="cuda")
    for x, y in zip(xs, ys):  # two calls in a row, different data
        want = api.inner_prod(x, y, f64=True).item()
        got = api.inner_prod_noalloc(x, y, out).item()
        assert got == want
        exact = float(np.dot(x.cpu().numpy().astype(np.float64), y.cpu().numpy().astype(np.float64)))
        assert abs(got - exact) <= 1e-12 * max(1.0, float(torch.sum(torch.abs(x * y)).item()))


def test_noalloc_back_to_back_on_one_stream():
    torch = torch_cuda()
    x = torch.full((4096,), 0.5, device="cuda")
    y = torch.full((4096,), 2.0, device="cuda")
    z = torch.full((100_000,), 3.0, device="cuda")
    out1 = torch.empty(1, dtype=torch.float64, device="cuda")
    out2 = torch.empty(1, dtype=torch.float64, device="cuda")
    api.inner_prod_noalloc(x, y, out1)
    api.inner_prod_noalloc(z, z, out2)  # queued behind the first; same array
    torch.cuda.synchronize()
    assert out1.item() == 4096.0
    assert out2.item() == 900_000.0


def test_noalloc_empty_and_bad_arguments():
    torch = torch_cuda()
    x = torch.ones(0, device="cuda")
    out = torch.full((1,), 7.0, dtype=torch.float64, device="cuda")
    api.inner_prod_noalloc(x, x, out)
    assert out.item() == 0.0
    from gpumatting_b200 import _lib as L

    rc = L.load().gm_inner_prod_f64_noalloc(None, None, None, 10, None)
    assert rc == L.GM_ERR_INVALID
