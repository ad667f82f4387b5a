#!/usr/bin/env python
"""Benchmark: NTF outer iterations/s on the dense 1024^3 rank-32 workload.

Workload (one step = one AUNTF outer iteration, ntf/auntf.hpp:129-176): a
1024 x 1024 x 1024 FP32 tensor (4.3 GB, larger than L2) built on the device as
a rank-32 CP model with U[0,1) factors plus 1 % Gaussian noise, clipped at 0;
HALS (default) at rank 32 with the dimension-tree MTTKRP, FP64 Gram/update/
error, mixed-precision (BF16 tensor-core) MTTKRP. The same GPU's FP64 plain
path, the final relative error of both after 50 iterations (HALS and MU), the
end-to-end rate through the C ABI with host buffers, the dominant kernel's
roofline and a CPU baseline are reported on the same JSON line.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

With N > 1 (torchrun) every rank runs an independent replica ("replicas
only": a single tensor's factorisation does not shard here), the time is the
max over ranks, and value = all ranks' iterations / that time.
"""
import argparse
import json
import os
import subprocess
import sys
import time

# the CPU legs use every host core: set before the BLAS is loaded
_CORES = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else os.cpu_count()
os.environ.setdefault("OPENBLAS_NUM_THREADS", str(_CORES))
os.environ.setdefault("OMP_NUM_THREADS", str(_CORES))

import numpy as np  # noqa: E402

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "NTF iters/s + MTTKRP TFLOP/s, mixed vs FP64 plain on same GPU, equal rel-error"
EB = {"bf16": 2, "bf16x2": 4, "fp64": 8}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=300)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", default="bf16", choices=["bf16", "bf16x2"])
    ap.add_argument("--algo", default="hals", choices=["hals", "mu", "anlsbpp"])
    ap.add_argument("--dims", default="1024,1024,1024")
    ap.add_argument("--rank", type=int, default=32)
    ap.add_argument("--quality-iters", type=int, default=50)
    ap.add_argument("--no-fp64", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--workload", default="cfg2",
                    choices=["cfg1", "cfg2", "cfg3", "cfg4", "cfg5", "updates", "nmf"],
                    help="cfg2 (default) is the metric's workload; the others are the remaining "
                         "synthetic configurations, measured with the same JSON contract")
    return ap.parse_args()


def workload(dims, k, seed=2024):
    rng = np.random.default_rng(seed)
    A = [rng.random((d, k)) for d in dims]
    G = np.ones((k, k))
    for a in A:
        G *= a.T @ a
    sigma = 0.01 * np.sqrt(G.sum() / float(np.prod(dims)))  # rho * ||M|| / sqrt(numel)
    F0 = [np.random.default_rng(seed + 1).random((d, k)) for d in dims]
    return A, sigma, F0


class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.path = os.path.join("/tmp", "planc_clocks_%d_%d.csv" % (os.getpid(), device))

    def start(self):
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), "--query-gpu=" + self.FIELDS,
                 "--format=csv,noheader,nounits", "-lms", "50"], stdout=self.f,
                stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(5)
        except Exception:
            self.proc.kill()
        self.f.close()
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            p = [x.strip() for x in line.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                mx.append(float(p[2]))
            except ValueError:
                continue
            for nm, v in zip(names, p[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        os.unlink(self.path)
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": float(max(mx)) if mx else None,
                "samples": len(sm), "reasons": sorted(reasons)}


def max_over_ranks(x, dist=None, device="cpu"):
    """Max of a per-rank scalar over all ranks (the job's time is the slowest
    rank's); identity without a process group."""
    if dist is None:
        return x
    import torch
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_value(local_ms, steps, world, dist=None, device="cpu"):
    """Whole-job iterations/s of `world` independent replicas that each ran
    `steps` iterations: all ranks' iterations / the slowest rank's time."""
    ms = max_over_ranks(local_ms, dist, device)
    return world * steps / (ms * 1e-3), ms


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def traffic_from_profiles(precision, dims, k, which):
    """Per-launch DRAM traffic of a partial MTTKRP kernel from the committed ncu
    summary (a line `traffic_per_launch_bytes <which> <prec> <dims> <k>: <n>`)."""
    path = os.path.join(ROOT, "profiles", "mttkrp_tc_1024cube_k32.md")
    if not os.path.exists(path):
        return None
    key = "traffic_per_launch_bytes %s %s %s %d:" % (which, precision, "x".join(map(str, dims)), k)
    for line in open(path):
        if line.strip().startswith(key):
            try:
                return float(line.split(":", 1)[1].strip().split()[0])
            except ValueError:
                return None
    return None


def left_splits(L, R, I0, k, sm_count):
    """Split-K count of the 3-way left contraction, as the library plans it
    (tc_left_plan: 128-row tiles, two per CTA when R > 128 and k <= 32, the
    SMs shared among the row groups, at most one split per run of I_0 rows)."""
    mt = 2 if (R > 128 and k <= 32) else 1
    groups = -(-R // (mt * 128))
    ns = max(1, sm_count // groups)
    units = L // I0 if I0 % 64 == 0 else -(-L // 64)
    return min(ns, units)


def cpu_sample(gpu, torch, dev, dims, A, sigma, F0, algo, iters=3):
    """The reference algorithm on the host cores over a bounded slice of the
    workload: dims[0] x dims[1] x 128 (1/8 of the tensor for 1024^3), same rank
    and noise model; iters/s scaled to the full tensor by the element ratio
    (the per-iteration cost is linear in the element count)."""
    import oracle
    from oracle import cpu_ntf
    sdims = (dims[0], dims[1], min(dims[2], 128))
    As = [A[0], A[1], A[2][:sdims[2]]]
    n = int(np.prod(sdims))
    x = torch.empty(n, dtype=torch.float64, device="cuda:%d" % dev)
    gpu.synth_cp_tensor(dev, x.data_ptr(), "f64", sdims, As, sigma, 7, clip=True)
    X = x.cpu().numpy().reshape(sdims, order="F")
    del x
    Fs = [F0[0], F0[1], F0[2][:sdims[2]]]
    oracle.lib()
    sec, _ = cpu_ntf.run_timed(X, Fs, algo, iters, _CORES, use_ref=True)
    scale = n / float(np.prod(dims))
    return {"value": (1.0 / sec) * scale, "unit": "iters/s", "cores": _CORES,
            "kind": "port",
            "sample": "%d outer %s iterations on a %dx%dx%d slice (same rank/noise), "
                      "iters/s scaled by the element ratio %.4f; MTTKRP through the reference's "
                      "own dimension-tree sources (oracle/_ref, OpenBLAS dgemm, %d threads) when "
                      "built, updates by the oracle restatement" % (iters, algo, *sdims, scale,
                                                                     _CORES)}


def reference_arm(args, rank, world):
    if rank != 0:
        return
    import oracle
    from oracle import cpu_ntf
    import torch
    import planc_b200 as gpu
    dims = tuple(int(x) for x in args.dims.split(","))
    k = args.rank
    A, sigma, F0 = workload(dims, k)
    sdims = (dims[0], dims[1], min(dims[2], 128))
    As = [A[0], A[1], A[2][:sdims[2]]]
    n = int(np.prod(sdims))
    dev = 0
    if torch.cuda.is_available():
        x = torch.empty(n, dtype=torch.float64, device="cuda:0")
        gpu.synth_cp_tensor(dev, x.data_ptr(), "f64", sdims, As, sigma, 7, clip=True)
        X = x.cpu().numpy().reshape(sdims, order="F")
        del x
    else:
        rng = np.random.default_rng(7)
        M = np.einsum("az,bz,cz->abc", *As)
        X = np.asfortranarray(np.maximum(M + sigma * rng.standard_normal(M.shape), 0))
    Fs = [F0[0], F0[1], F0[2][:sdims[2]]]
    oracle.lib()
    cpu_ntf.run_timed(X, Fs, args.algo, max(args.warmup, 0), _CORES, use_ref=True)
    t0 = time.perf_counter()
    sec, _ = cpu_ntf.run_timed(X, Fs, args.algo, args.steps, _CORES, use_ref=True)
    wall = time.perf_counter() - t0
    scale = n / float(np.prod(dims))
    value = (1.0 / sec) * scale
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "iters/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 / value, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": "%s FP32 tensor, rank %d, %s, dimension tree (CPU sample %s)"
                   % ("x".join(map(str, dims)), k, args.algo.upper(), "x".join(map(str, sdims))),
                   "dims": list(dims), "rank": k, "algo": args.algo},
        "cpu_baseline": {"value": value, "unit": "iters/s", "cores": _CORES, "kind": "port",
                         "sample": "each step one outer iteration on a %s slice, iters/s scaled by "
                                   "%.4f; MTTKRP via the reference's dimension-tree sources "
                                   "(oracle/_ref) when built" % ("x".join(map(str, sdims)), scale)},
        "e2e": {"value": value, "unit": "iters/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
        "wall_s": wall,
    }
    print(json.dumps(line))


def main():
    args = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        reference_arm(args, rank, world)
        return
    if args.workload != "cfg2":
        import bench_configs
        bench_configs.run(args, rank, world, local)
        return
    import torch
    import planc_b200 as gpu
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    dev = local
    torch.cuda.set_device(dev)
    dims = tuple(int(x) for x in args.dims.split(","))
    k = args.rank
    numel = int(np.prod(dims))
    A, sigma, F0 = workload(dims, k)
    X = torch.empty(numel, dtype=torch.float32, device="cuda:%d" % dev)
    gpu.synth_cp_tensor(dev, X.data_ptr(), "f32", dims, A, sigma, 7, clip=True)
    torch.cuda.synchronize(dev)

    def barrier():
        torch.cuda.synchronize(dev)
        if dist is not None:
            dist.barrier()

    devname = "cuda:%d" % dev

    # ---------------- mixed precision, tensor resident in HBM
    ctx = gpu.Context(dev, args.precision)
    ctx.set_tensor(X.data_ptr(), dims=dims, dtype="f32")
    ctx.set_factors(F0)
    stream = torch.cuda.ExternalStream(ctx.stream, device="cuda:%d" % dev)
    ctx.run(args.algo, args.warmup)
    sampler = ClockSampler(dev)
    sampler.start()
    time.sleep(0.2)
    barrier()
    # timed region: one CUDA graph per outer iteration, as a user's run executes
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    ctx.run(args.algo, args.steps, compute_error=True)
    e1.record(stream)
    barrier()
    clocks = sampler.stop()
    value, ms = replica_value(e0.elapsed_time(e1), args.steps, world, dist, devname)
    # per-kernel durations: a second region of the same steps with CUDA events
    # around every launch on the library's stream (graphs off while timing)
    ctx.set_timing(True)
    ctx.kernel_times()
    barrier()
    ek0, ek1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    n1 = ctx.launch_count()
    ek0.record(stream)
    ctx.run(args.algo, args.steps, compute_error=True)
    ek1.record(stream)
    barrier()
    # the graph-timed region replays exactly these kernels (launch() counts
    # each kernel launch; a graph replay is not counted by the library)
    launches = ctx.launch_count() - n1
    kt = ctx.kernel_times()
    ctx.set_timing(False)
    ms_event_timed = ek0.elapsed_time(ek1) / args.steps

    # dominant kernel: the partial MTTKRP contraction (right: P = X*F_last,
    # writes P in FP32; left: X^T*KRP, writes split-K FP64 partials)
    L = dims[0] * dims[1]
    R = numel // L
    nsplit_left = left_splits(L, R, dims[0], k, torch.cuda.get_device_properties(dev).multi_processor_count)
    kern = {
        "right": (kt["contract"], numel * EB[args.precision] + L * k * 4),
        "left": (kt["contract_left"], numel * EB[args.precision] + nsplit_left * R * k * 8),
    }
    peak, peak_kind = peaks()
    per_kernel = {}
    for name, ((kms, kn), kbytes) in kern.items():
        avg_s = (kms / max(kn, 1)) * 1e-3
        per_kernel[name] = {"launches": kn, "avg_launch_ms": avg_s * 1e3,
                            "algorithmic_bytes_per_launch": kbytes,
                            "achieved_gbs": kbytes / avg_s / 1e9 if avg_s > 0 else None}
    dom = max(per_kernel, key=lambda n: kern[n][0][0])
    d = per_kernel[dom]
    c_ms = kern["right"][0][0] + kern["left"][0][0]
    c_n = kern["right"][0][1] + kern["left"][0][1]
    mttkrp_tflops = (2.0 * numel * k * c_n) / (c_ms * 1e-3) / 1e12 if c_ms > 0 else None
    roofline = {"bound": "hbm", "achieved": d["achieved_gbs"], "peak": peak, "unit": "GB/s",
                "frac": d["achieved_gbs"] / peak if d["achieved_gbs"] else None,
                "traffic": traffic_from_profiles(args.precision, dims, k, dom),
                "peak_source": peak_kind,
                "kernel": "partial MTTKRP, %s contraction (k_tc_%s)" % (dom, dom),
                "algorithmic_bytes_per_launch": d["algorithmic_bytes_per_launch"],
                "avg_launch_ms": d["avg_launch_ms"], "launches": d["launches"],
                "per_kernel": per_kernel}
    kernel_share = {c: round(v[0] / max(sum(x[0] for x in kt.values()), 1e-9), 4)
                    for c, v in kt.items() if v[1]}

    # ---------------- FP64 plain path on the same GPU, same tensor
    fp64 = None
    quality = {}
    if not args.no_fp64:
        ctx64 = gpu.Context(dev, "fp64")
        ctx64.set_tensor(X.data_ptr(), dims=dims, dtype="f32")
        ctx64.set_factors(F0)
        ctx64.run(args.algo, 2, compute_error=False)
        k64 = max(3, min(args.steps, 20))
        s64 = torch.cuda.ExternalStream(ctx64.stream, device="cuda:%d" % dev)
        barrier()
        f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        f0.record(s64)
        ctx64.run(args.algo, k64, compute_error=True)
        f1.record(s64)
        barrier()
        ms64 = max_over_ranks(f0.elapsed_time(f1), dist, devname)
        fp64 = {"value": world * k64 / (ms64 * 1e-3), "unit": "iters/s",
                "ms_per_step": ms64 / k64, "steps": k64, "dtype": "f64"}
        # equal-iteration-count relative error, HALS and MU, both paths
        for algo in ("hals", "mu"):
            res = {}
            for name, c in (("mixed", ctx), ("fp64", ctx64)):
                c.set_factors(F0)
                res[name] = float(c.run(algo, args.quality_iters)[-1])
            res["abs_diff"] = abs(res["mixed"] - res["fp64"])
            quality[algo] = res
        ctx64.close()

    # ---------------- end to end through the C ABI with host buffers
    e2e = None
    if not args.no_e2e:
        xh = torch.empty(numel, dtype=torch.float32, pin_memory=True)
        xh.copy_(X)
        Xh = xh.numpy().reshape(dims, order="F")
        T = args.quality_iters
        ctx.set_tensor(Xh)  # warm-up of the path
        ctx.set_factors(F0)
        ctx.run(args.algo, 2)
        steps_e2e = 2
        barrier()
        g0, g1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        g0.record(stream)
        for _ in range(steps_e2e):
            ctx.set_tensor(Xh)
            ctx.set_factors(F0)
            ctx.run(args.algo, T, compute_error=True)
            ctx.get_factors()
        g1.record(stream)
        barrier()
        ms_e2e = max_over_ranks(g0.elapsed_time(g1), dist, devname)
        fbytes = sum(d * k * 8 for d in dims)
        e2e = {"value": world * steps_e2e * T / (ms_e2e * 1e-3), "unit": "iters/s",
               "h2d_bytes_per_step": numel * 4 + fbytes,
               "d2h_bytes_per_step": fbytes + k * 8 + T * 8,
               "step": "set_tensor(host) + set_factors + %d iterations + get_factors" % T}
        del xh

    cpu = None
    if not args.no_cpu and world == 1 and rank == 0:
        try:
            cpu = cpu_sample(gpu, torch, dev, dims, A, sigma, F0, args.algo)
        except Exception as ex:  # the baseline is reported, not required
            cpu = {"value": None, "error": str(ex)[:200]}
    ctx.close()
    del X

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "iters/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": args.precision,
            "data": "synthetic: rank-%d CP model, U[0,1) factors, 1%% Gaussian noise, clipped >= 0, "
                    "generated on the device (Philox)" % k,
            "config": {"workload": "%s FP32 tensor, rank %d, %s, dimension-tree MTTKRP on tensor "
                                   "cores (%s), FP64 Gram/update/error"
                                   % ("x".join(map(str, dims)), k, args.algo.upper(),
                                      args.precision),
                       "dims": list(dims), "rank": k, "algo": args.algo,
                       "precision": args.precision, "parallelism": "replicas x%d" % world,
                       "l2": "inputs larger than L2 (%.1f GB tensor)" % (numel * 4 / 1e9)},
            "mttkrp_tflops": mttkrp_tflops,
            "fp64_plain": fp64,
            "speedup_vs_fp64": (value / fp64["value"]) if fp64 else None,
            "rel_error": quality,
            "roofline": roofline,
            "kernel_time_share": kernel_share,
            "kernel_ms_per_iter": {c: round(v[0] / args.steps, 4) for c, v in kt.items() if v[1]},
            "ms_per_step_event_timed": ms_event_timed,
            "cpu_baseline": cpu,
            "e2e": e2e,
            "gpu_launches": launches,
            "clocks": clocks,
        }
        print(json.dumps(line))
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
