"""Distributed NTF over a one-dimensional slab partition of the tensor.

The reference's distributed loop (distntf/distauntf.hpp) block-partitions
every mode over a processor grid. On NVLink/NVSwitch the simplest mapping is
a 1-D grid: mode p of the tensor is cut into contiguous slabs, one per rank
(one GPU each), and every other mode's factor is replicated. Per mode n of an
outer iteration (the AUNTF order, ntf/auntf.hpp:128-177):

  * the leave-one-out Gram from the N global k x k Grams (identical on every
    rank: they are all-reduced when formed);
  * the rank's partial MTTKRP of its slab (the dimension tree on the local
    tensor); for n != p the partials are summed and scattered by rows
    (reduce-scatter, distauntf.hpp:305-315), for n = p they are already the
    rank's rows;
  * the update of the rank's rows (the updates are row-separable given the
    Gram: MU, HALS, ANLS/BPP);
  * the Gram of the updated rows, all-reduced (distauntf.hpp:92-115), which
    gives the global column norms lambda and the normalised Gram at once
    (NCPFactors::distributed_normalize); the rows are normalised;
  * for n != p the normalised rows are all-gathered into the replicated
    factor (distauntf.hpp:164-234).

The relative error is the Gram form ||X||^2 - 2 <X, model> + ||model||^2
(distauntf.hpp:685-727): <X, model> from the rank's rows of the last mode's
MTTKRP and factor, all-reduced; ||model||^2 from the global Grams.

The local compute goes through `ops` (GpuOps: the library's device entry
points on a Context holding the rank's slab) and the collectives through
`comm` (TorchComm over torch.distributed: NCCL between GPUs; with the gloo
backend on CPU ranks, as the tests run it, reduce-scatter is an all-reduce of
the padded buffer and the rank's slice of it).
"""
import numpy as np

ALGOS = ("mu", "hals", "anlsbpp")


def slab_bounds(I, world):
    """Contiguous, balanced slabs of I rows over `world` ranks (the first
    I % world ranks take one extra row)."""
    base, extra = divmod(I, world)
    bounds, lo = [], 0
    for r in range(world):
        hi = lo + base + (1 if r < extra else 0)
        bounds.append((lo, hi))
        lo = hi
    return bounds


class TorchComm:
    """Sum-collectives of the distributed loop over torch.distributed: NCCL's
    reduce-scatter / all-gather / all-reduce on device tensors; with the gloo
    backend (CPU ranks, or ranks whose device buffers are staged through host
    memory) reduce-scatter is an all-reduce and the rank's slice."""

    def __init__(self, dist, group=None):
        self.dist = dist
        self.group = group
        self.rank = dist.get_rank(group)
        self.world = dist.get_world_size(group)
        self.gloo = dist.get_backend(group) == "gloo"

    def _host(self, t):
        return t.cpu() if t.is_cuda else t

    def all_reduce(self, t):
        if self.gloo and t.is_cuda:
            h = t.cpu()
            self.dist.all_reduce(h, group=self.group)
            t.copy_(h)
        else:
            self.dist.all_reduce(t, group=self.group)

    def reduce_scatter(self, full, out):
        """out = rows [rank*c, (rank+1)*c) of the sum over ranks of `full`
        (world*c rows)."""
        if self.gloo:
            self.all_reduce(full)
            c = out.shape[0]
            out.copy_(full[self.rank * c:(self.rank + 1) * c])
        else:
            self.dist.reduce_scatter_tensor(out, full, group=self.group)

    def all_gather(self, part, full):
        """full (world*c rows) = every rank's `part` (c rows) in rank order."""
        if self.gloo:
            h = self._host(full).contiguous()
            chunks = list(h.chunk(self.world))
            self.dist.all_gather(chunks, self._host(part).contiguous(), group=self.group)
            if full.is_cuda:
                full.copy_(h)
        else:
            self.dist.all_gather_into_tensor(full, part.contiguous(), group=self.group)


class GpuOps:
    """Local compute of one rank on its GPU: the library's device entry points
    on a Context that holds the rank's slab of the tensor."""

    def __init__(self, ctx, torch, device):
        self.ctx = ctx
        self.torch = torch
        self.device = device
        self.stream = torch.cuda.ExternalStream(ctx.stream, device=device)

    def zeros(self, *shape):
        return self.torch.zeros(*shape, dtype=self.torch.float64, device=self.device)

    def scope(self):
        """Makes the context's stream current, so that torch's collectives are
        ordered with the library's kernels."""
        return self.torch.cuda.stream(self.stream)

    def mttkrp(self, n, F, out, reuse):
        self.ctx.mttkrp_device(n, [f.data_ptr() for f in F], out.data_ptr(), dimtree=True,
                               reuse=reuse)

    def update(self, algo, H, M, G, rows):
        self.ctx.update_device(algo, H.data_ptr(), M.data_ptr(), G.data_ptr(), rows, H.shape[1])

    def gram(self, F, rows, G):
        self.ctx.gram_device(F.data_ptr(), rows, F.shape[1], G.data_ptr())

    def normalize(self, F, rows, Gin, lam, Gout):
        self.ctx.normalize_device(F.data_ptr() if rows else 0, rows, Gin.shape[0], Gin.data_ptr(),
                                  lam.data_ptr(), Gout.data_ptr())

    def coldot(self, A, B, rows, out):
        self.ctx.coldot_device(A.data_ptr() if rows else 0, B.data_ptr() if rows else 0, rows,
                               out.shape[0], out.data_ptr())

    def sync(self):
        self.ctx.sync()


class DistNTF:
    """AUNTF over a 1-D slab partition of mode `part_mode`.

    dims: the global tensor's mode sizes; the rank's slab of mode part_mode
    (rows slab_bounds(dims[p], world)[rank]) is already in `ops`. F_init: the
    global initial factors (numpy, I_n x k), identical on every rank; they are
    normalised mode by mode as AUNTF::reset does."""

    def __init__(self, ops, comm, dims, k, part_mode, F_init, normX2_local):
        torch = ops.torch
        self.ops, self.comm, self.torch = ops, comm, torch
        self.dims = tuple(int(d) for d in dims)
        self.N = len(self.dims)
        self.k = int(k)
        self.p = int(part_mode)
        if self.dims[self.p] < comm.world:
            raise ValueError("the partitioned mode needs at least one row per rank")
        self.slab = slab_bounds(self.dims[self.p], comm.world)[comm.rank]
        self.chunk = [-(-d // comm.world) for d in self.dims]
        with ops.scope():
            self.F, self.M, self.Mfull, self.Fpad, self.Fblk = [], [], [], [], []
            for n, d in enumerate(self.dims):
                if n == self.p:
                    lo, hi = self.slab
                    f = torch.tensor(np.ascontiguousarray(F_init[n][lo:hi]), dtype=torch.float64)
                    self.F.append(f.to(ops.zeros(1).device))
                    self.M.append(ops.zeros(hi - lo, k))
                    self.Mfull.append(None)
                    self.Fpad.append(None)
                    self.Fblk.append(None)
                else:
                    c = self.chunk[n]
                    pad = ops.zeros(comm.world * c, k)
                    pad[:d] = torch.tensor(np.ascontiguousarray(F_init[n]), dtype=torch.float64)
                    self.Fpad.append(pad)
                    self.F.append(pad[:d])
                    self.Mfull.append(ops.zeros(comm.world * c, k))
                    self.M.append(ops.zeros(c, k))
                    self.Fblk.append(ops.zeros(c, k))
            self.G = [ops.zeros(k, k) for _ in range(self.N)]
            self.Gtmp = ops.zeros(k, k)
            self.lam = ops.zeros(k)
            self.dot = ops.zeros(k)
            nx = ops.zeros(1)
            nx[0] = float(normX2_local)
            comm.all_reduce(nx)
            self.normX2 = float(nx.cpu()[0])
            for n in range(self.N):
                lo, hi = self._rows(n)
                self._normalize(n, self._block(n, lo, hi), hi - lo)

    # rows of mode n this rank updates: its slab for the partitioned mode,
    # else its chunk of the reduce-scatter (clipped to the mode's size)
    def _rows(self, n):
        if n == self.p:
            return 0, self.slab[1] - self.slab[0]
        c = self.chunk[n]
        lo = min(self.comm.rank * c, self.dims[n])
        hi = min(lo + c, self.dims[n])
        return lo, hi

    def _block(self, n, lo, hi):
        """The rank's rows of F_n as a contiguous buffer it updates in place."""
        if n == self.p:
            return self.F[n]
        blk = self.Fblk[n]
        blk.zero_()
        blk[:hi - lo] = self.F[n][lo:hi]
        return blk

    def _normalize(self, n, blk, rows):
        ops, comm = self.ops, self.comm
        ops.gram(blk, rows, self.Gtmp)
        comm.all_reduce(self.Gtmp)
        ops.normalize(blk, rows, self.Gtmp, self.lam, self.G[n])
        if n != self.p:
            comm.all_gather(blk, self.Fpad[n])

    def _gram_loo(self, n):
        g = None
        for m in range(self.N):
            if m != n:
                g = self.G[m].clone() if g is None else g * self.G[m]
        return g

    def run(self, algo, iters, compute_error=True):
        """`iters` outer iterations; returns the relative error of each."""
        if algo not in ALGOS:
            raise ValueError("distributed updates: %s" % ", ".join(ALGOS))
        ops, comm = self.ops, self.comm
        errs = []
        with ops.scope():
            for _ in range(iters):
                for n in range(self.N):
                    Gloo = self._gram_loo(n)
                    lo, hi = self._rows(n)
                    rows = hi - lo
                    if n == self.p:
                        ops.mttkrp(n, self.F, self.M[n], reuse=n != 0)
                    else:
                        full = self.Mfull[n]
                        full.zero_()
                        ops.mttkrp(n, self.F, full[:self.dims[n]], reuse=n != 0)
                        comm.reduce_scatter(full, self.M[n])
                    blk = self._block(n, lo, hi)
                    ops.update(algo, blk, self.M[n], Gloo, rows)
                    self._normalize(n, blk, rows)
                if compute_error:
                    errs.append(self._error())
            ops.sync()
        return np.array(errs)

    def _error(self):
        last = self.N - 1
        lo, hi = self._rows(last)
        blk = self.F[last] if last == self.p else self.F[last][lo:hi]
        self.ops.coldot(self.M[last], blk.contiguous(), hi - lo, self.dot)
        self.comm.all_reduce(self.dot)
        lam = self.lam.double().cpu().numpy()
        inner = float(np.dot(self.dot.cpu().numpy(), lam))
        H = np.ones((self.k, self.k))
        for g in self.G:
            H = H * g.cpu().numpy()
        mn = float(lam @ H @ lam)
        e2 = self.normX2 - 2.0 * inner + mn
        return float(np.sqrt(abs(e2) / self.normX2))

    def factors(self):
        """The global factors (numpy, I_n x k; the partitioned mode gathered
        from every rank) and lambda."""
        torch, comm = self.torch, self.comm
        out = []
        with self.ops.scope():
            for n in range(self.N):
                if n != self.p:
                    out.append(self.F[n].cpu().numpy().copy())
                    continue
                bounds = slab_bounds(self.dims[n], comm.world)
                c = max(h - l for l, h in bounds)
                part = self.ops.zeros(c, self.k)
                part[:self.slab[1] - self.slab[0]] = self.F[n]
                full = self.ops.zeros(comm.world * c, self.k)
                comm.all_gather(part, full)
                fn = full.cpu().numpy()
                out.append(np.concatenate([fn[r * c:r * c + (h - l)] for r, (l, h) in enumerate(bounds)]))
        return out, self.lam.cpu().numpy().copy()


def slab_of(X, part_mode, rank, world):
    """The rank's slab of a global tensor X (numpy, Fortran order, mode 0
    fastest) along mode part_mode, as a Fortran-order array."""
    lo, hi = slab_bounds(X.shape[part_mode], world)[rank]
    idx = [slice(None)] * X.ndim
    idx[part_mode] = slice(lo, hi)
    return np.asfortranarray(X[tuple(idx)])


def gpu_dist_ntf(comm, X_slab, dims, k, part_mode, F_init, precision="fp64", device=0):
    """A DistNTF on this rank's GPU: a library Context holding the rank's slab
    (X_slab, numpy Fortran-order), its local factors set from F_init (the
    partitioned mode's slab rows)."""
    import torch

    from . import Context
    ctx = Context(device, precision)
    ctx.set_tensor(X_slab if precision == "fp64" else X_slab.astype(np.float32))
    lo, hi = slab_bounds(dims[part_mode], comm.world)[comm.rank]
    F_local = [f[lo:hi] if n == part_mode else f for n, f in enumerate(F_init)]
    ctx.set_factors(F_local)  # sizes the context's buffers; its own factors are not used
    ops = GpuOps(ctx, torch, "cuda:%d" % device)
    return DistNTF(ops, comm, dims, k, part_mode, F_init, ctx.tensor_norm2())
