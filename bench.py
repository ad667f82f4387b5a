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


def left_splits(L, R, I0, k, sm_count, precision="bf16"):
    """Split-K count of the 3-way left contraction, as the library plans it
    (without the factored form, I_0 % 64 != 0: the long-K kernel's plan;
    tc_left_plan: 128-row tiles, two per CTA when R > 128 and k <= 32 except
    for the factored contraction's cp.async instance (I_0 % 64 == 0, rank <= 32,
    BF16, an even number of 64-wide chunks per work unit), which takes one;
    the SMs shared among the row groups, at most one split per work unit:
    a run of I_0 rows, or a part of one with PLANC_GPU_LEFT_PARTS)."""
    factored = I0 % 64 == 0
    hp = int(os.environ.get("PLANC_GPU_LEFT_PARTS", "1") or 1)
    if not factored or hp < 1 or (I0 // 64) % hp != 0:
        hp = 1
    kpad = 16 if k <= 16 else 32 if k <= 32 else 64
    cpa = (factored and kpad <= 32 and precision == "bf16" and (I0 // 64 // hp) % 2 == 0
           and os.environ.get("PLANC_GPU_TC_LOADS", "cpasync") != "tma")
    if not factored and os.environ.get("PLANC_GPU_LEFT_FORM", "image") != "producers":
        # the long-K kernel against a Khatri-Rao image (tc_long_plan): K groups
        # of two 64-wide blocks, one split per group at most
        mt = 2 if (R > 128 and kpad <= 32) else 1
        groups = -(-R // (mt * 128))
        ns = max(1, sm_count // groups)
        return min(ns, -(-(-(-L // 64)) // 2))
    mt = 1 if cpa else (2 if (R > 128 and k <= 32) else 1)
    groups = -(-R // (mt * 128))
    ns = max(1, sm_count // groups)
    units = L // I0 * hp if factored else -(-L // 64)
    return min(ns, units)


def cpu_model():
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def workload_name(dims, k, algo):
    """The workload both arms run, named without implementation details."""
    return ("%s FP32 tensor, rank-%d CP + 1%% noise, %s, rank %d, dimension-tree MTTKRP, "
            "relative error every iteration" % ("x".join(map(str, dims)), k, algo.upper(), k))


def reference_cpu(dims, k, algo, warmup, steps):
    """The reference's own NTF code on the host cores (oracle/_ref; the
    oracle's restatement when that build is absent) over the full workload:
    the same factors, noise and seed as the GPU arm, generated on the host.
    Returns (iters/s, details)."""
    import oracle
    from oracle import cpu_ntf
    A, sigma, F0 = workload(dims, k)
    oracle.lib()
    r = cpu_ntf.run(dims, A, sigma, 7, F0, algo, warmup, steps, compute_error=True)
    total = sum(r["step_s"])
    value = steps / total if total > 0 else None
    return value, r


def cpu_sample(dims, k, algo, warmup=1, steps=3):
    """cpu_baseline of the GPU arm: a bounded sample of the same workload,
    `steps` timed outer iterations (after `warmup`) of the reference's own
    code on the full tensor, all host cores."""
    value, r = reference_cpu(dims, k, algo, warmup, steps)
    return {"value": value, "unit": "iters/s", "cores": _CORES, "kind": r["kind"],
            "cpu": cpu_model(),
            "sample": "%d timed outer %s iterations (after %d untimed) of the full %s workload, "
                      "relative error every iteration; %s on %d host threads (OpenBLAS, "
                      "OpenMP)" % (steps, algo.upper(), warmup, "x".join(map(str, dims)),
                                   "the reference's own AUNTF + DenseDimensionTree compiled "
                                   "from its sources (oracle/_ref)" if r["kind"] == "reference"
                                   else "the oracle's restatement", _CORES),
            "final_rel_error": r["error"]}


def reference_arm(args, rank, world):
    """--impl reference: the reference's CPU implementation of the path on the
    host cores (no GPU, no library of this repository), on this bench's
    workload, metric and unit. Rank 0 alone runs; other ranks exit."""
    if rank != 0:
        return
    dims = tuple(int(x) for x in args.dims.split(","))
    k = args.rank
    t0 = time.perf_counter()
    value, r = reference_cpu(dims, k, args.algo, max(args.warmup, 0), args.steps)
    wall = time.perf_counter() - t0
    steps_ms = [1e3 * x for x in r["step_s"]]
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "iters/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": sum(steps_ms) / max(len(steps_ms), 1), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic: rank-%d CP model, U[0,1) factors, 1%% Gaussian noise, clipped >= 0, "
                "values rounded to FP32, generated on the host (Philox, the GPU arm's "
                "generator)" % k,
        "config": {"workload": workload_name(dims, k, args.algo), "dims": list(dims), "rank": k,
                   "algo": args.algo, "parallelism": "host cores x%d" % _CORES,
                   "l2": "inputs larger than L2 (%.1f GB FP64 tensor)" % (np.prod(dims) * 8 / 1e9)},
        "cpu_baseline": {"value": value, "unit": "iters/s", "cores": _CORES, "kind": r["kind"],
                         "cpu": cpu_model(),
                         "sample": "each step one outer iteration of the full workload through "
                                   "%s" % ("the reference's own AUNTF (NTF%s) with its "
                                           "DenseDimensionTree, compiled unmodified from its "
                                           "sources (oracle/_ref)" % args.algo.upper()
                                           if r["kind"] == "reference" else
                                           "the oracle's restatement")},
        "e2e": {"value": value, "unit": "iters/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
        "step_ms": {"min": min(steps_ms) if steps_ms else None,
                    "max": max(steps_ms) if steps_ms else None},
        "final_rel_error": r["error"],
        "setup_s": r["setup_s"],
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
    nsplit_left = left_splits(L, R, dims[0], k, torch.cuda.get_device_properties(dev).multi_processor_count,
                              args.precision)
    kern = {
        "right": (kt["contract"], numel * EB[args.precision] + L * k * 4),
        "left": (kt["contract_left"], numel * EB[args.precision] + nsplit_left * R * k * 8),
    }
    # the left contraction's kernel: the factored form when I0 is a multiple of 64
    kname = {"right": "k_tc_right", "left": "k_tc_left_fac" if dims[0] % 64 == 0 else "k_tc_left"}
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
                "kernel": "partial MTTKRP, %s contraction (%s)" % (dom, kname[dom]),
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
        ctx64.run(args.algo, 2, compute_error=True)  # captures the timed graph
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

    ctx.close()
    del X
    torch.cuda.empty_cache()
    cpu = None
    if not args.no_cpu and world == 1 and rank == 0:
        try:
            cpu = cpu_sample(dims, k, args.algo)
        except Exception as ex:  # the baseline is reported, not required
            cpu = {"value": None, "error": str(ex)[:200]}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "iters/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": args.precision,
            "data": "synthetic: rank-%d CP model, U[0,1) factors, 1%% Gaussian noise, clipped >= 0, "
                    "generated on the device (Philox)" % k,
            "config": {"workload": workload_name(dims, k, args.algo),
                       "mttkrp": "tcgen05 tensor cores (%s operands, FP32 accumulate); FP64 "
                                 "Grams, updates and error" % args.precision,
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
