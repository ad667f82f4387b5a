"""The distributed NTF (planc_b200/dist.py) with its GPU local compute (the
library's device entry points on a Context per rank), against the FP64 oracle:
one NCCL rank, and two ranks sharing the one GPU over gloo (each rank's
kernels run on their own; the collectives run on the host, so no kernel waits
on another rank)."""
import os
import socket

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, backend, case, q):
    import datetime
    import sys
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    sys.path.insert(0, os.path.join(root, "tests"))
    import torch
    import torch.distributed as dist

    from helpers import cp_tensor
    from planc_b200.dist import TorchComm, gpu_dist_ntf, slab_of
    dims, k, part, algo, iters = case
    torch.cuda.set_device(0)
    kw = {"device_id": torch.device("cuda:0")} if backend == "nccl" else {}
    dist.init_process_group(backend, rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=120), **kw)
    try:
        X, _ = cp_tensor(dims, k, noise=0.02, seed=81)
        rng = np.random.default_rng(82)
        F0 = [rng.random((d, k)) for d in dims]
        comm = TorchComm(dist)
        d = gpu_dist_ntf(comm, slab_of(X, part, rank, world), dims, k, part, F0)
        errs = d.run(algo, iters)
        F, lam = d.factors()
        d.ops.ctx.close()
        q.put((rank, errs, F, lam))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world,backend,case", [
    (1, "nccl", ((40, 30, 24), 6, 2, "hals", 6)),
    (2, "gloo", ((40, 30, 24), 6, 2, "hals", 6)),
    (2, "gloo", ((36, 28, 20, 12), 5, 0, "anlsbpp", 4)),
    (2, "gloo", ((33, 29, 31), 8, 1, "mu", 5)),
])
def test_gpu_dist_ntf_matches_oracle(gpu, oracle_lib, world, backend, case):
    import torch.multiprocessing as mp

    from helpers import cp_tensor, rel
    dims, k, part, algo, iters = case
    port = _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, world, port, backend, case, q))
             for r in range(world)]
    for p in procs:
        p.start()
    res = sorted([q.get(timeout=300) for _ in range(world)], key=lambda t: t[0])
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    X, _ = cp_tensor(dims, k, noise=0.02, seed=81)
    rng = np.random.default_rng(82)
    F0 = [rng.random((d, k)) for d in dims]
    Fo, lamo, eo = oracle_lib.ntf_run(X, F0, algo, iters, dimtree=True)
    for rank, errs, F, lam in res:
        assert np.max(np.abs(errs - eo) / eo) < 1e-10, (errs, eo)
        for a, b in zip(F, Fo):
            assert rel(a, b) < 1e-10
        assert rel(lam, lamo) < 1e-10
