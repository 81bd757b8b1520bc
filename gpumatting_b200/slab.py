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
convergence is declared on the true residual only.  p lives in the slab's
extended input buffer, so on the GPU one iteration is the halo exchange, one
gm_levin_apply, one gm_cg_dots4 (two launches) and one gm_cg_update_dev per
slab, the sum and all-reduce of four doubles, and one gm_cg_scalars launch
that turns them into alpha and beta on the device; no vector is copied and
the host reads the iteration state once per chunk of iterations.  With every
slab on one rank the chunk is a CUDA graph.  With one slab and no process
group it is an ordinary single-domain CG.  The reference solves one
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
        ops, back = [], []
        first, last = slabs[0], slabs[-1]

        def send(t):
            return t if t.is_contiguous() else t.contiguous()

        def recv(t):
            # a pitched view (a slab buffer wider than W) receives through a
            # contiguous staging tensor, copied in after the wait
            if t.is_contiguous():
                return t
            tmp = t.new_empty(t.shape)
            back.append((t, tmp))
            return tmp

        if self.first > 0:
            peer = self._rank_of(self.first - 1)
            ops.append(dist.P2POp(dist.isend, send(vecs[0][first.above:2 * first.above]), peer, self.group))
            ops.append(dist.P2POp(dist.irecv, recv(vecs[0][:first.above]), peer, self.group))
        if self.first + self.count < self.nslabs:
            peer = self._rank_of(self.first + self.count)
            lo = last.above + last.R
            ops.append(dist.P2POp(dist.isend, send(vecs[-1][lo - last.below:lo]), peer, self.group))
            ops.append(dist.P2POp(dist.irecv, recv(vecs[-1][lo:lo + last.below]), peer, self.group))
        if ops:
            for req in dist.batch_isend_irecv(ops):
                req.wait()
        for t, tmp in back:
            t.copy_(tmp)

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


def _is_cuda(t) -> bool:
    return bool(getattr(t, "is_cuda", False))


def _dots4(r, p, q, out):
    """out[:] = FP64 [r.r, p.q, r.q, q.q] of one slab's own rows."""
    if _is_cuda(r):
        from . import api

        api.cg_dots4(r, p, q, out=out)
    else:
        import torch

        rd, pd, qd = r.double(), p.double(), q.double()
        out.copy_(torch.stack([(rd * rd).sum(), (pd * qd).sum(), (rd * qd).sum(), (qd * qd).sum()]))


def _update(x, r, p, q, alpha: float, beta: float, update_p: bool) -> None:
    """x += alpha p; r -= alpha q; then p = r + beta p when update_p."""
    if _is_cuda(x):
        from . import api

        api.cg_update(x, r, p, q, alpha, beta, update_p)
    else:
        x.add_(p, alpha=alpha)
        r.sub_(q, alpha=alpha)
        if update_p:
            p.mul_(beta).add_(r)


# Device iteration state (6 doubles, the layout gm_cg_scalars keeps).
_THR, _RR, _RR_NEXT, _ITERS, _STOP, _STOP_AT = range(6)


def _scalars(coef, state, sums) -> None:
    """coef = [alpha, beta, mode] from the summed sums, advancing state:
    gm_cg_scalars on CUDA tensors, the same rule in Python on CPU ones."""
    if _is_cuda(sums):
        from . import api

        api.cg_scalars(coef, state, sums)
        return
    st = state.tolist()
    rr, pq, rq, qq = sums.tolist()
    alpha = beta = mode = 0.0
    if st[_STOP] == 0.0:
        if not (pq > 0.0) or rr != rr:
            st[_STOP] = 2.0
        else:
            alpha = rr / pq
            nx = max(rr - 2.0 * alpha * rq + alpha * alpha * qq, 0.0)
            st[_RR], st[_RR_NEXT], st[_ITERS] = rr, nx, st[_ITERS] + 1.0
            if (st[_THR] >= 0.0 and nx <= st[_THR]) or st[_ITERS] >= st[_STOP_AT]:
                st[_STOP], mode = 1.0, 1.0
            else:
                beta, mode = nx / rr, 2.0
        state.copy_(state.new_tensor(st))
    coef.copy_(coef.new_tensor([alpha, beta, mode]))


def _update_dev(x, r, p, q, coef) -> None:
    """The update with [alpha, beta, mode] read from coef."""
    if _is_cuda(x):
        from . import api

        api.cg_update_dev(x, r, p, q, coef)
        return
    alpha, beta, mode = coef.tolist()
    if mode != 0.0:
        _update(x, r, p, q, alpha, beta, mode == 2.0)


def slab_cg(slabs, comm: SlabComm, x, b, rtol: float = 1e-6, max_iters: int = 5000,
            replace_every: int = 50, chunk: int = 10, graph: bool | None = None) -> SlabResult:
    """CG on the whole image from its local slabs.  x[i], b[i]: own-row
    tensors (R_i x W) of local slab i; x holds the initial guess and receives
    the solution.  Every slab object has .R, .above, .below, .ext (its
    extended (above + R + below) x W input vector, which holds the search
    direction p) and .apply_ext() -> the own rows (R x W) of A ext, a view
    that stays valid until its next call.

    The scalars of each iteration stay on the device (gm_cg_scalars): the
    host queues `chunk` iterations and reads the 6-double state once per
    chunk.  An iteration after the stop (the recurrence met rtol, the next
    residual replacement is due, or a breakdown) changes nothing, so the
    iteration count is exact.  graph (CUDA tensors, all slabs on this rank
    only; None = whenever that holds): the chunk is captured once as a CUDA
    graph and replayed."""
    import torch

    n = len(slabs)
    dev = x[0].device
    cuda = _is_cuda(x[0])
    ext = [s.ext for s in slabs]
    p = [e[s.above:s.above + s.R] for s, e in zip(slabs, ext)]  # own rows of the extended vectors
    r = [torch.empty_like(b[i]) for i in range(n)]
    parts = torch.zeros((n, 4), dtype=torch.float64, device=dev)
    sums = torch.zeros(4, dtype=torch.float64, device=dev)
    coef = torch.zeros(3, dtype=torch.float64, device=dev)
    state = torch.zeros(6, dtype=torch.float64, device=dev)
    local = comm._dist is None or comm._dist.get_world_size(comm.group) == 1
    if graph is None:
        graph = cuda and local
    if graph and not (cuda and local):
        raise ValueError("graph capture needs CUDA tensors and every slab on this rank")

    def apply_p():
        """q_i = own rows of A_i p (halos exchanged first)."""
        comm.exchange(slabs, ext)
        return [s.apply_ext() for s in slabs]

    def reduce4(rs, ps, qs):
        """sums = FP64 [r.r, p.q, r.q, q.q] over all slabs (on the device)."""
        if n == 1:
            _dots4(rs[0], ps[0], qs[0], sums)
        else:
            for i in range(n):
                _dots4(rs[i], ps[i], qs[i], parts[i])
            torch.sum(parts, dim=0, out=sums)
        comm.allreduce(sums)

    def iteration():
        q = apply_p()
        reduce4(r, p, q)
        _scalars(coef, state, sums)
        for i in range(n):
            _update_dev(x[i], r[i], p[i], q[i], coef)

    def true_residual():
        """r = b - A x, through the extended vectors (p is kept)."""
        keep = [t.clone() for t in p]
        for i in range(n):
            p[i].copy_(x[i])
        ax = apply_p()
        for i in range(n):
            torch.sub(b[i], ax[i], out=r[i])
            p[i].copy_(keep[i])

    true_residual()
    for i in range(n):
        p[i].copy_(r[i])
    reduce4(b, r, r)
    bb, rr = sums.tolist()[:2]
    if not bb > 0.0:
        bb = rr if rr > 0.0 else 1.0
    rel = (rr / bb) ** 0.5
    thr = rtol * rtol * bb if rtol > 0.0 else -1.0
    it = nrep = 0
    status = 0
    chunk = max(1, int(chunk))
    g, warm = None, False
    while not (rtol > 0.0 and rel <= rtol) and it < max_iters:
        stop_at = max_iters if replace_every <= 0 else min(max_iters, (it // replace_every + 1) * replace_every)
        state.copy_(torch.tensor([thr, 0.0, 0.0, float(it), 0.0, float(stop_at)], dtype=torch.float64))
        while True:
            # the first chunk runs eagerly (kernels loaded, scratch pools made)
            if graph and warm and stop_at - it >= chunk:
                if g is None:
                    g = torch.cuda.CUDAGraph()
                    with torch.cuda.graph(g):
                        for _ in range(chunk):
                            iteration()
                g.replay()
            else:
                for _ in range(min(chunk, stop_at - it)):
                    iteration()
                warm = True
            st = state.tolist()
            it = int(st[_ITERS])
            if st[_STOP] != 0.0:
                break
        if st[_STOP] == 2.0:
            status = 5
            break
        # stop 1: x and r were updated, p kept -- replace r by the true residual
        rr_ = st[_RR]
        true_residual()
        reduce4(r, r, r)
        rr_true = sums.tolist()[0]
        nrep += 1
        rel = (rr_true / bb) ** 0.5
        if (rtol > 0.0 and rel <= rtol) or it >= max_iters:
            break
        beta = rr_true / rr_ if rr_ > 0.0 else 0.0
        for i in range(n):
            p[i].mul_(beta).add_(r[i])
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

    @property
    def ext(self):
        """The extended input vector ((above + R + below) x W): a view of the
        operator's input buffer, so nothing is copied before a product."""
        n = self.above + self.R + self.below
        return self._x[self.skip:self.skip + n, :self.W]

    def apply_ext(self):
        """Own rows (R x W) of the true FP32 operator applied to ext: a view
        of the output buffer, valid until the next call."""
        self.store.apply(self._x[:, :self.W], self._y[:, :self.W], true_op=True)
        o = self.skip + self.above
        return self._y[o:o + self.R, :self.W]

    def apply(self, x_ext):
        """Extended result (above + R + below) x W of the operator on x_ext
        (own rows exact, halo rows not)."""
        self.ext.copy_(x_ext)
        self.store.apply(self._x[:, :self.W], self._y[:, :self.W], true_op=True)
        n = self.above + self.R + self.below
        return self._y[self.skip:self.skip + n, :self.W]
