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


def _bench(args, env_extra=None):
    import json
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    env = dict(os.environ, **(env_extra or {}))
    r = subprocess.run([sys.executable, os.path.join(root, "bench.py")] + args, cwd=root,
                       env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    return [json.loads(l) for l in lines]


def test_reference_arm_line_on_cpu():
    # --impl reference runs the reference's CPU implementation (or the
    # oracle's restatement) on the host only: one JSON line with the
    # contract's keys, the e2e key repeating the value with no copies
    out = _bench(["--impl", "reference", "--dims", "24,20,16", "--rank", "4", "--steps", "3",
                  "--warmup", "1"], {"CUDA_VISIBLE_DEVICES": ""})
    assert len(out) == 1
    line = out[0]
    assert line["impl"] == "reference" and line["unit"] == "iters/s" and line["steps"] == 3
    assert line["value"] > 0 and line["higher_is_better"] is True
    assert line["e2e"] == {"value": line["value"], "unit": "iters/s", "h2d_bytes_per_step": 0,
                           "d2h_bytes_per_step": 0}
    assert line["cpu_baseline"]["kind"] in ("reference", "port")
    assert line["cpu_baseline"]["value"] == line["value"]
    assert 0 < line["final_rel_error"] < 1


def test_reference_arm_other_ranks_exit_without_output():
    out = _bench(["--impl", "reference", "--dims", "12,10,8", "--rank", "3", "--steps", "1",
                  "--warmup", "0"], {"RANK": "1", "WORLD_SIZE": "2", "CUDA_VISIBLE_DEVICES": ""})
    assert out == []


@pytest.mark.parametrize("dims,k,prec,env,expect", [
    # factored left contraction, cp.async instance: one 128-row tile a CTA,
    # 1024 / 128 = 8 row groups, 148 // 8 = 18 splits
    ((1024, 1024, 1024), 32, "bf16", {}, 18),
    # TMA instance (two tiles a CTA): 4 row groups, 37 splits
    ((1024, 1024, 1024), 32, "bf16", {"PLANC_GPU_TC_LOADS": "tma"}, 37),
    # bf16x2 has no cp.async instance of the factored left contraction
    ((1024, 1024, 1024), 32, "bf16x2", {}, 37),
    # I0 % 64 != 0: the long-K kernel over a Khatri-Rao image, 4 row groups
    ((1000, 1000, 1000), 32, "bf16", {}, 37),
    # ... or the producer-warp kernel
    ((1000, 1000, 1000), 32, "bf16", {"PLANC_GPU_LEFT_FORM": "producers"}, 37),
    # small K: at most one split per K group of two 64-wide blocks (L = 1320:
    # 21 blocks, 11 groups)
    ((40, 33, 96), 16, "bf16", {}, 11),
])
def test_bench_left_split_estimate(monkeypatch, dims, k, prec, env, expect):
    # bench.py's algorithmic bytes of the left contraction count the split-K
    # partials the library writes; its estimate follows the library's plans
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    import bench
    for name in ("PLANC_GPU_TC_LOADS", "PLANC_GPU_LEFT_FORM", "PLANC_GPU_LEFT_PARTS"):
        monkeypatch.delenv(name, raising=False)
    for name, v in env.items():
        monkeypatch.setenv(name, v)
    L = dims[0] * dims[1]
    assert bench.left_splits(L, dims[2], dims[0], k, 148, prec) == expect
