"""Row-slab split of ONE image over several ranks (one process per GPU).

The Levin operator couples pixels at most two rows apart (the 5x5 stencil of
the 25-band store, main.cu:164-190), so an image cut into horizontal slabs
needs, per matrix product, only the two rows either side of each slab from
its neighbours, and CG needs its dot products summed over all slabs.  This
module is the host side of that split; the compute stays in libgpumat.

Slabs.  slab_bounds() cuts H rows into `nslabs` near-equal runs.  Slab k owns
rows [r0, r1) and keeps `above` = min(2, r0) halo rows above and `below` =
min(2, H - r1) below, so its vectors are (above + R + below) x W, own rows
in the middle.  A slab's operator must give exact rows of the whole image's
operator for its own rows from such an extended vector:

* LevinSlab (GPU): assembles a symmetric band store from the image rows
  [r0 - above - 2, r1 + below + 2) clipped to the image -- the 3x3 windows
  that touch an own row or a halo row lie inside them -- and applies its true
  FP32 operator (gm_levin_apply) to the extended vector; the own rows of the
  result are exact, the halo rows are not used.
* Any object with the same attributes (the tests use the FP64 oracle
  operator on CPU tensors as a stand-in).

Exchange.  SlabComm moves halo rows between neighbouring slabs: a plain
tensor copy between slabs of the same rank, torch.distributed point-to-point
send/recv into a LOCAL halo buffer between ranks (NCCL over NVLink on GPUs,
gloo on CPU), and sums the FP64 partials of each CG iteration with one
all_reduce.  No kernel reads another GPU's memory; nothing here waits inside
a kernel for another rank.

Solve.  slab_cg() runs CG with the single-reduction recurrence of the fused
solver: each iteration applies the operator once (after one halo exchange of
p) and all-reduces four FP64 sums (r.r, p.q, r.q, q.q); alpha = r.r / p.q
and the next r.r = r.r - 2 alpha r.q + alpha^2 q.q give beta without a second
reduction.  Every `replace_every` iterations, and before it stops, the true
residual b - A x (one more exchange and reduction) replaces the recurrence;
convergence is declared on the true residual only.  With one slab and no
process group it is an ordinary single-domain CG.  The reference solves one
image per process (main.cu:458-526); it has no multi-GPU path.
"""
from __future__ import annotations

from dataclasses import dataclass

HALO = 2


def slab_bounds(H: int, nslabs: int, k: int) -> tuple[int, int]:
    """Rows [r0, r1) of slab k of nslabs (near-equal runs).  Every slab has
    at least HALO rows, so a halo never reaches past a neighbour."""
    if not (0 <= k < nslabs) or nslabs * HALO > H:
        raise ValueError(f"slab {k} of {nslabs} for {H} rows (at most {H // HALO} slabs)")
    return H * k // nslabs, H * (k + 1) // nslabs


def slab_halo(H: int, r0: int, r1: int) -> tuple[int, int]:
    """Halo rows kept above and below a slab: two, or fewer at the image edge."""
    return min(HALO, r0), min(HALO, H - r1)


def rank_slabs(nslabs: int, world: int, rank: int) -> tuple[int, int]:
    """Slabs [first, first + count) of a rank: near-equal contiguous runs."""
    if nslabs < world:
        raise ValueError("fewer slabs than ranks")
    return nslabs * rank // world, nslabs * (rank + 1) // world - nslabs * rank // world


class SlabComm:
    """Halo exchange and scalar reduction for the slabs [first, first+count)
    of `nslabs` that this rank holds; the other ranks hold the others in
    rank order.  `group` is a torch.distributed process group (None: the
    default group when one is initialised, else this process is alone)."""

    def __init__(self, nslabs: int, first: int, count: int, group=None):
        self.nslabs, self.first, self.count = nslabs, first, count
        self.group = group
        import torch.distributed as dist

        self._dist = dist if (dist.is_available() and dist.is_initialized()) else None
        if self._dist is None and (first != 0 or count != nslabs):
            raise ValueError("slabs on other ranks need an initialised process group")

    def _rank_of(self, slab: int) -> int:
        """Rank holding a slab (the contiguous runs of rank_slabs)."""
        world = self._dist.get_world_size(self.group)
        for r in range(world):
            f, c = rank_slabs(self.nslabs, world, r)
            if f <= slab < f + c:
                return r
        raise ValueError(slab)

    def exchange(self, slabs, vecs) -> None:
        """Fill the halo rows of every local slab's extended vector vecs[i]
        from its neighbours' own rows."""
        for i in range(self.count - 1):
            a, b = slabs[i], slabs[i + 1]
            # bottom own rows of a -> top halo of b, top own rows of b -> bottom halo of a
            vecs[i + 1][:b.above] = vecs[i][a.above + a.R - b.above:a.above + a.R]
            vecs[i][a.above + a.R:] = vecs[i + 1][b.above:b.above + a.below]
        if self._dist is None:
            return
        dist = self._dist
        ops = []
        first, last = slabs[0], slabs[-1]
        # whole rows of a contiguous [rows, W] tensor: contiguous views, so the
        # received rows land in the vector itself
        if self.first > 0:
            peer = self._rank_of(self.first - 1)
            ops.append(dist.P2POp(dist.isend, vecs[0][first.above:2 * first.above], peer, self.group))
            ops.append(dist.P2POp(dist.irecv, vecs[0][:first.above], peer, self.group))
        if self.first + self.count < self.nslabs:
            peer = self._rank_of(self.first + self.count)
            lo = last.above + last.R
            ops.append(dist.P2POp(dist.isend, vecs[-1][lo - last.below:lo], peer, self.group))
            ops.append(dist.P2POp(dist.irecv, vecs[-1][lo:lo + last.below], peer, self.group))
        if ops:
            for req in dist.batch_isend_irecv(ops):
                req.wait()

    def allreduce(self, t):
        """Sum of an FP64 tensor over all slabs (in place)."""
        if self._dist is not None and self._dist.get_world_size(self.group) > 1:
            self._dist.all_reduce(t, group=self.group)
        return t


@dataclass
class SlabResult:
    status: int          # 0 converged, 6 not converged, 5 breakdown (the library's GM_* codes)
    iters: int
    replacements: int
    rel_residual: float  # true relative residual over the whole image


def slab_cg(slabs, comm: SlabComm, x, b, rtol: float = 1e-6, max_iters: int = 5000,
            replace_every: int = 50) -> SlabResult:
    """CG on the whole image from its local slabs.  x[i], b[i]: own-row
    tensors (R_i x W) of local slab i; x holds the initial guess and receives
    the solution.  Every slab object has .R, .above, .below and
    .apply(x_ext) -> y_ext on extended (above + R + below) x W tensors."""
    import torch

    n = len(slabs)
    ext = [torch.zeros((s.above + s.R + s.below,) + tuple(x[i].shape[1:]), dtype=x[i].dtype, device=x[i].device)
           for i, s in enumerate(slabs)]
    dev = x[0].device

    def own(i, t):
        s = slabs[i]
        return t[s.above:s.above + s.R]

    def apply_all(src):
        """q_i = own rows of A_i (src with halos)."""
        for i in range(n):
            own(i, ext[i]).copy_(src[i])
        comm.exchange(slabs, ext)
        # (the operator may return a view of its own buffer: copy out)
        return [own(i, slabs[i].apply(ext[i])).clone() for i in range(n)]

    def dots(pairs):
        """FP64 sums over all slabs of the products of each pair."""
        acc = torch.zeros(len(pairs), dtype=torch.float64, device=dev)
        for k, (u, v) in enumerate(pairs):
            for i in range(n):
                acc[k] += torch.sum(u[i].double() * v[i].double())
        comm.allreduce(acc)
        return [float(a) for a in acc.tolist()]

    def true_residual():
        ax = apply_all(x)
        return [b[i] - ax[i] for i in range(n)]

    r = true_residual()
    bb, rr = dots([(b, b), (r, r)])
    if not bb > 0.0:
        bb = rr if rr > 0.0 else 1.0
    rel = (rr / bb) ** 0.5
    it = nrep = 0
    status = 0
    p = [torch.zeros_like(r[i]) for i in range(n)]
    beta = 0.0
    while not (rtol > 0.0 and rel <= rtol) and it < max_iters:
        for i in range(n):
            p[i].mul_(beta).add_(r[i])
        q = apply_all(p)
        rr_, pq, rq, qq = dots([(r, r), (p, q), (r, q), (q, q)])
        if not (pq > 0.0) or pq != pq or rr_ != rr_:
            status = 5
            break
        alpha = rr_ / pq
        for i in range(n):
            x[i].add_(p[i], alpha=alpha)
            r[i].sub_(q[i], alpha=alpha)
        it += 1
        rr_next = max(rr_ - 2.0 * alpha * rq + alpha * alpha * qq, 0.0)
        due = replace_every > 0 and it % replace_every == 0
        if due or (rtol > 0.0 and rr_next <= rtol * rtol * bb) or it >= max_iters:
            r = true_residual()
            (rr_true,) = dots([(r, r)])
            nrep += 1
            rel = (rr_true / bb) ** 0.5
            beta = rr_true / rr_ if rr_ > 0.0 else 0.0
        else:
            rel = (rr_next / bb) ** 0.5
            beta = rr_next / rr_
    if status == 0 and rtol > 0.0 and not rel <= rtol:
        status = 6
    return SlabResult(status, it, nrep, rel)


class LevinSlab:
    """GPU operator of one slab: the true FP32 operator of a symmetric band
    store assembled from the image rows around the slab (see the module
    comment).  image: [H, W, 3] uint8 RGB on the device; scribbles: [H, W]
    uint8 map (0 background, 255 foreground)."""

    def __init__(self, image, scribbles, eps: float, gamma_value: float, r0: int, r1: int):
        from . import api

        H, W = int(image.shape[0]), int(image.shape[1])
        self.W, self.r0, self.r1, self.R = W, r0, r1, r1 - r0
        self.above, self.below = slab_halo(H, r0, r1)
        c0, c1 = max(0, r0 - self.above - HALO), min(H, r1 + self.below + HALO)
        self.skip = r0 - self.above - c0  # crop rows above the extended vector
        self.crop_rows = c1 - c0
        self.store = api.LevinStore(W, c1 - c0, "fp32").assemble(image[c0:c1].contiguous(),
                                                                  scribbles[c0:c1].contiguous(), eps=eps,
                                                                  gamma_value=gamma_value)
        import torch

        pitch = (W + 3) // 4 * 4
        self._x = torch.zeros((self.crop_rows, pitch), dtype=torch.float32, device=image.device)
        self._y = torch.empty((self.crop_rows, pitch), dtype=torch.float32, device=image.device)

    def rhs(self):
        """b = gamma s of the own rows (R x W)."""
        rows = self.store.planes("b")
        return rows[self.skip + self.above:self.skip + self.above + self.R, :self.W].clone()

    def apply(self, x_ext):
        n = self.above + self.R + self.below
        self._x[self.skip:self.skip + n, :self.W].copy_(x_ext)
        self.store.apply(self._x[:, :self.W], self._y[:, :self.W], true_op=True)
        return self._y[self.skip:self.skip + n, :self.W]
