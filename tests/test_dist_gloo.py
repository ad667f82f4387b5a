"""The distributed NTF schedule (planc_b200/dist.py: slab partition,
reduce-scatter of the partial MTTKRPs, all-reduced Grams, all-gathered
factors, Gram-form error) on world_size-2 gloo ranks on CPU, against the
single-process oracle. The local compute of each rank is a CPU stand-in over
the oracle (test infrastructure); the partition and every collective are the
product's own code."""
import contextlib
import os
import socket

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp


class CpuOps:
    """One rank's local compute on CPU: the oracle's MTTKRP and updates on the
    rank's slab (same interface as planc_b200.dist.GpuOps)."""

    def __init__(self, X_slab):
        import oracle
        self.oracle = oracle
        self.torch = torch
        self.X = X_slab

    def zeros(self, *shape):
        return torch.zeros(*shape, dtype=torch.float64)

    def scope(self):
        return contextlib.nullcontext()

    def mttkrp(self, n, F, out, reuse):
        out.copy_(torch.from_numpy(self.oracle.mttkrp_direct(self.X, [f.numpy() for f in F], n)))

    def update(self, algo, H, M, G, rows):
        h, m, g = H[:rows].numpy(), M[:rows].numpy(), G.numpy()
        if algo == "hals":
            new = self.oracle.hals_update(h, m, g)
        elif algo == "mu":
            new = self.oracle.mu_update(h, m, g)
        else:
            new = self.oracle.bpp_update(m, g)[0]
        H[:rows] = torch.from_numpy(new)

    def gram(self, F, rows, G):
        f = F[:rows]
        G.copy_(f.T @ f)

    def normalize(self, F, rows, Gin, lam, Gout):
        lam.copy_(torch.sqrt(torch.diagonal(Gin)))
        pos = lam > 0
        scale = torch.where(pos, lam, torch.ones_like(lam))
        both = pos[:, None] & pos[None, :]
        Gout.copy_(torch.where(both, Gin / (scale[:, None] * scale[None, :]), Gin))
        if rows:
            F[:rows] = F[:rows] / scale

    def coldot(self, A, B, rows, out):
        out.copy_((A[:rows] * B[:rows]).sum(0))

    def sync(self):
        pass


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, case, q):
    import datetime
    import sys
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    sys.path.insert(0, os.path.join(root, "tests"))
    import torch.distributed as dist

    from helpers import cp_tensor
    from planc_b200.dist import DistNTF, TorchComm, slab_of
    dims, k, part, algo, iters = case
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=120))
    try:
        X, _ = cp_tensor(dims, k, noise=0.02, seed=71)
        rng = np.random.default_rng(72)
        F0 = [rng.random((d, k)) for d in dims]
        comm = TorchComm(dist)
        Xs = slab_of(X, part, rank, world)
        ops = CpuOps(Xs)
        d = DistNTF(ops, comm, dims, k, part, F0, float(np.sum(Xs * Xs)))
        errs = d.run(algo, iters)
        F, lam = d.factors()
        q.put((rank, errs, F, lam))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("case", [((12, 10, 9), 4, 2, "hals", 5), ((12, 10, 9), 4, 0, "mu", 5),
                                  ((11, 7, 9, 6), 3, 1, "anlsbpp", 4),
                                  ((9, 13, 8), 5, 2, "anlsbpp", 4)])
def test_dist_ntf_two_gloo_ranks_matches_oracle(oracle_lib, case):
    from helpers import cp_tensor, rel
    dims, k, part, algo, iters = case
    world = 2
    port = _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, world, port, case, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = sorted([q.get(timeout=300) for _ in range(world)], key=lambda t: t[0])
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    X, _ = cp_tensor(dims, k, noise=0.02, seed=71)
    rng = np.random.default_rng(72)
    F0 = [rng.random((d, k)) for d in dims]
    Fo, lamo, eo = oracle_lib.ntf_run(X, F0, algo, iters, dimtree=False)
    for rank, errs, F, lam in res:
        assert np.max(np.abs(errs - eo) / eo) < 1e-10, (errs, eo)
        for a, b in zip(F, Fo):
            assert rel(a, b) < 1e-10
        assert rel(lam, lamo) < 1e-10


def test_slab_bounds_cover_and_balance():
    from planc_b200.dist import slab_bounds
    for I in (1, 5, 8, 13):
        for world in range(1, min(I, 6) + 1):
            b = slab_bounds(I, world)
            assert b[0][0] == 0 and b[-1][1] == I
            assert all(b[i][1] == b[i + 1][0] for i in range(world - 1))
            sizes = [h - l for l, h in b]
            assert max(sizes) - min(sizes) <= 1 and min(sizes) >= 1
