"""Row-slab split of one image (gpumatting_b200/slab.py) on CPU: slab rows,
halos and rank assignment; the distributed CG over 1, 2 and 4 slabs, in one
process and over two gloo ranks (one and two slabs per rank), against the
single-domain FP64 oracle CG; and a rank that leaves makes the other's
exchange fail instead of hang.

Each slab's operator here is a CPU stand-in built from the FP64 oracle: the
oracle's Levin assembly of the image rows around the slab (the rows whose
3x3 windows touch it), applied to the slab's extended vector -- the same
construction as the GPU slab operator (LevinSlab), in FP64."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from gpumatting_b200 import slab as S

W, H, SEED = 48, 41, 3


class OracleSlab:
    """FP64 CPU stand-in for a slab operator (test infrastructure)."""

    def __init__(self, image, gamma, r0, r1, pitched=False):
        from oracle import oracle as O

        Hh, Ww = gamma.shape
        self.R, self.r0 = r1 - r0, r0
        self.above, self.below = S.slab_halo(Hh, r0, r1)
        c0, c1 = max(0, r0 - self.above - S.HALO), min(Hh, r1 + self.below + S.HALO)
        self.skip, self.rows, self.W = r0 - self.above - c0, c1 - c0, Ww
        w = O.levin_sym64(image[c0:c1].astype(np.float64) / 255.0, 1e-5)
        self.op = O.Operator(W=Ww, H=c1 - c0, w=w, gamma=gamma[c0:c1].ravel().astype(np.float64))

        import torch

        n = self.above + self.R + self.below
        # pitched: a view into rows wider than W, as the GPU slab's buffer is
        # when W is not a multiple of 4 (its halo rows are not contiguous)
        self.ext = (torch.zeros((n, Ww + 3), dtype=torch.float64)[:, :Ww] if pitched
                    else torch.zeros((n, Ww), dtype=torch.float64))

    def apply_ext(self):
        import torch

        n = self.above + self.R + self.below
        xc = np.zeros((self.rows, self.W))
        xc[self.skip:self.skip + n] = self.ext.numpy()
        y = self.op.apply(xc.ravel()).reshape(self.rows, self.W)
        o = self.skip + self.above
        return torch.from_numpy(y[o:o + self.R].copy())


def _problem():
    from gpumatting_b200.synth import make_problem

    p = make_problem(W, H, SEED)
    return p, p.gamma.astype(np.float64), (p.gamma * p.s).astype(np.float64)


def _single_domain(rtol):
    from oracle import oracle as O

    p, g, b = _problem()
    w = O.levin_sym64(p.image.astype(np.float64) / 255.0, p.eps)
    op = O.Operator(W=W, H=H, w=w, gamma=g.ravel())
    x, it, rel = op.cg(b.ravel(), np.full(W * H, 0.5), rtol=rtol, maxit=100000)
    return x.reshape(H, W), it, op


def _solve_slabs(nslabs, first, count, rtol=1e-11, pitched=False):
    import torch

    p, g, b = _problem()
    assert p.eps == 1e-5
    slabs, xs, bs = [], [], []
    for k in range(first, first + count):
        r0, r1 = S.slab_bounds(H, nslabs, k)
        slabs.append(OracleSlab(p.image, g, r0, r1, pitched))
        xs.append(torch.full((r1 - r0, W), 0.5, dtype=torch.float64))
        bs.append(torch.from_numpy(b[r0:r1].copy()))
    comm = S.SlabComm(nslabs, first, count)
    res = S.slab_cg(slabs, comm, xs, bs, rtol=rtol, max_iters=20000)
    return res, [x.numpy() for x in xs]


def test_slab_rows_halos_and_ranks():
    rows = [S.slab_bounds(61, 4, k) for k in range(4)]
    assert rows[0][0] == 0 and rows[-1][1] == 61
    assert all(a[1] == b[0] for a, b in zip(rows, rows[1:]))
    assert all(r1 - r0 >= S.HALO for r0, r1 in rows)
    assert S.slab_halo(61, 0, 15) == (0, 2) and S.slab_halo(61, 45, 61) == (2, 0)
    assert [S.rank_slabs(5, 2, r) for r in range(2)] == [(0, 2), (2, 3)]
    with pytest.raises(ValueError):
        S.slab_bounds(5, 3, 0)  # a slab of one row would need a neighbour's neighbour
    with pytest.raises(ValueError):
        S.SlabComm(4, 1, 2)     # other ranks' slabs without a process group


@pytest.mark.parametrize("nslabs", [1, 2, 4])
def test_slab_cg_in_one_process_matches_single_domain(nslabs):
    """All slabs in one process (halos copied locally): the solution and
    the iteration count match the single-domain FP64 CG."""
    x64, it64, op = _single_domain(1e-11)
    res, xs = _solve_slabs(nslabs, 0, nslabs)
    assert res.status == 0 and res.rel_residual <= 1e-11, res
    x = np.concatenate(xs)
    b = _problem()[2].ravel()
    assert np.linalg.norm(b - op.apply(x.ravel())) / np.linalg.norm(b) <= 1.1e-11
    assert np.linalg.norm(x - x64) / np.linalg.norm(x64) <= 1e-6
    assert abs(res.iters - it64) <= 0.02 * it64 + 2, (res.iters, it64)


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, q, nslabs, mode, pitched=False):
    import datetime

    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=10))
    try:
        first, count = S.rank_slabs(nslabs, world, rank)
        if mode == "leave" and rank == 1:
            q.put((rank, "left"))
            return
        try:
            res, xs = _solve_slabs(nslabs, first, count, pitched=pitched)
            q.put((rank, res, first, xs))
        except Exception as e:  # noqa: BLE001 - a failed exchange is the expected outcome of "leave"
            q.put((rank, "error", type(e).__name__))
    finally:
        if mode == "ok":
            dist.destroy_process_group()


def _run(nslabs, mode="ok", pitched=False):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q, nslabs, mode, pitched)) for r in range(2)]
    for p in procs:
        p.start()
    out = [q.get(timeout=300) for _ in range(2)]
    for p in procs:
        p.join(timeout=60)
        if p.is_alive():
            p.kill()
    return sorted(out, key=lambda o: o[0])


@pytest.mark.parametrize("nslabs,pitched", [(2, False), (4, False), (2, True)])
def test_two_gloo_ranks_solve_one_image(nslabs, pitched):
    """Two ranks (one or two slabs each), halo rows over gloo send/recv and
    one all-reduce per iteration: the gathered solution matches the
    single-domain FP64 CG within 1e-6 relative, and both ranks agree on the
    iteration count and residual.  pitched: the halo rows travel through
    contiguous staging tensors."""
    x64, it64, op = _single_domain(1e-11)
    out = _run(nslabs, pitched=pitched)
    (_, r0, f0, xs0), (_, r1, f1, xs1) = out
    assert r0 == r1 and r0.status == 0 and r0.rel_residual <= 1e-11, (r0, r1)
    x = np.concatenate(xs0 + xs1)
    assert x.shape == (H, W)
    assert np.linalg.norm(x - x64) / np.linalg.norm(x64) <= 1e-6
    assert abs(r0.iters - it64) <= 0.02 * it64 + 2, (r0.iters, it64)


def test_rank_leaving_makes_the_exchange_fail():
    out = _run(2, mode="leave")
    assert out[1][1] == "left"
    assert out[0][1] == "error"
