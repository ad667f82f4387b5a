"""The N > 1 bench logic on CPU: world_size-2 gloo ranks (127.0.0.1), each
with its own replica time; the job's time is the slowest rank's and the value
counts every rank's iterations."""
import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    local_ms = 100.0 + 50.0 * rank  # rank 1 is the slowest
    value, ms = bench.replica_value(local_ms, steps=10, world=world, dist=dist, device="cpu")
    q.put((rank, value, ms))
    dist.barrier()
    dist.destroy_process_group()


def test_replica_value_max_over_two_gloo_ranks():
    world = 2
    port = _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    res = sorted(q.get(timeout=10) for _ in range(world))
    for rank, value, ms in res:
        assert ms == pytest.approx(150.0)
        assert value == pytest.approx(world * 10 / 0.150)


def test_replica_value_single_process():
    import bench
    value, ms = bench.replica_value(200.0, steps=20, world=1)
    assert ms == 200.0 and value == pytest.approx(100.0)
