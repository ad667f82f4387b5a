"""The synthetic configurations other than the headline one, measured with
the bench.py JSON contract (python bench.py --workload cfgN ...):

  cfg1  64x64x64 FP64 tensor, rank-8 CP + 1 % noise, HALS k=8, 20 iterations,
        FP64 plain path (latency-bound: one CUDA graph per iteration); parity
        against the CPU oracle on the same inputs is reported.
  cfg3  192x192x192x192 FP32 tensor from a rank-64 CP model with half of the
        factor entries zeroed, + 1 % noise; ANLS/BPP k=64, 30 iterations,
        BF16 tensor-core MTTKRP on the balanced 4-way tree, one batched BPP
        launch per mode; split-BF16 (bf16x2) and the FP64 plain path
        alongside.
  cfg4  256 independent 3-way FP32 tensors, mode sizes U{32..256}, ranks
        U{4,8,16,32}, CP + 1 % noise; HALS, one CUDA-graph launch per
        iteration for all 256 tensors, autotuned per-launch parallelism.
  cfg5  512^3 BF16 CP loss 1/2||X - [[A,B,C]]||^2 (rank 32, 5 % noise),
        torch.autograd with the MTTKRP kernels as backward, projected
        accelerated gradient steps on the factor leaves.
  nmf   shared-memory NMF of a dense 16384 x 16384 FP32 matrix (1.07 GB, rank-32
        nonnegative model + 1 % noise): MU, HALS and ANLS/BPP, 20 iterations
        each, A H and A^T W on tensor cores (BF16 copy of A) and on the FP64
        plain path, from the same start.
  updates  the headline tensor (1024^3 FP32, rank-32 CP + 1 % noise) under
        every update of the solver family -- MU, HALS, ANLS/BPP, AO-ADMM and
        Nesterov (with its extrapolation step) -- 20 iterations each, BF16
        tensor-core MTTKRP and the FP64 plain path, from the same start.

A step is one outer iteration (cfg1, cfg3), one batched iteration of all
256 tensors (cfg4) or one forward+backward+update (cfg5). Inputs are
generated on the device and stay resident; the timed region is bracketed by
synchronisation and timed with CUDA events on the launching stream.
"""
import json
import time

import numpy as np

METRIC = "NTF iters/s + MTTKRP TFLOP/s, mixed vs FP64 plain on same GPU, equal rel-error"


def _synth(gpu, torch, dev, dims, A, sigma, seed, dtype="f32"):
    n = int(np.prod(dims))
    X = torch.empty(n, dtype=torch.float32 if dtype == "f32" else torch.float64,
                    device="cuda:%d" % dev)
    gpu.synth_cp_tensor(dev, X.data_ptr(), dtype, dims, A, sigma, seed, clip=True)
    return X


def _sigma(A, rho):
    k = A[0].shape[1]
    G = np.ones((k, k))
    for a in A:
        G *= a.T @ a
    return rho * np.sqrt(G.sum() / float(np.prod([a.shape[0] for a in A])))


def _launches_per_run(ctx, algo, steps, err=True):
    """Kernel launches of one `steps`-iteration run, counted on an eager
    (graphs off) pass; a graph replay launches the same kernels."""
    ctx.set_timing(True)
    n0 = ctx.launch_count()
    ctx.run(algo, steps, compute_error=err)
    n = ctx.launch_count() - n0
    kt = ctx.kernel_times()
    ctx.set_timing(False)
    return n, kt


def _time_run(torch, ctx, algo, steps, err=True):
    stream = torch.cuda.ExternalStream(ctx.stream)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    n0 = ctx.launch_count()
    e0.record(stream)
    errs = ctx.run(algo, steps, compute_error=err)
    e1.record(stream)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1), errs, ctx.launch_count() - n0


def _line(args, world, value, unit, ms_per_step, dtype, config, **extra):
    line = {"metric": METRIC, "value": value, "unit": unit, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": dtype, "data": "synthetic",
            "config": config}
    line.update(extra)
    return line


def cfg1(args, gpu, torch, dev):
    import oracle
    dims, k, T = (64, 64, 64), 8, 20
    rng = np.random.default_rng(101)
    A = [rng.random((d, k)) for d in dims]
    Xd = _synth(gpu, torch, dev, dims, A, _sigma(A, 0.01), 11, dtype="f64")
    X = Xd.cpu().numpy().reshape(dims, order="F")
    F0 = [np.random.default_rng(102).random((d, k)) for d in dims]
    with gpu.Context(dev, "fp64") as c:
        c.set_tensor(X)
        c.set_factors(F0)
        c.run("hals", args.warmup)
        c.set_factors(F0)
        ms, errs, _ = _time_run(torch, c, "hals", T)
        Fg, lg = c.get_factors()
        launches, _ = _launches_per_run(c, "hals", T)
    t0 = time.perf_counter()
    Fo, lo, eo = oracle.ntf_run(X, F0, "hals", T)
    cpu_s = time.perf_counter() - t0
    par_err = float(np.max(np.abs(errs - eo) / eo))
    par_f = max(float(np.abs(a - b).max() / np.abs(b).max()) for a, b in zip(Fg, Fo))
    return _line(args, 1, T / (ms * 1e-3), "iters/s", ms / T, "f64",
                 {"workload": "64x64x64 FP64, rank-8 CP + 1% noise, HALS k=8, 20 iterations, "
                              "dimension tree, FP64 plain path", "dims": list(dims), "rank": k},
                 us_per_iter=1e3 * ms / T, gpu_launches=launches, launches_per_iter=launches / T,
                 parity_vs_oracle={"max_rel_err_diff": par_err, "max_rel_factor_diff": par_f,
                                   "bar": 1e-10},
                 cpu_baseline={"value": T / cpu_s, "unit": "iters/s", "cores": 1, "kind": "port",
                               "sample": "the whole 20-iteration run, oracle restatement"})


def cfg3(args, gpu, torch, dev):
    dims, k, T = (192, 192, 192, 192), 64, 30
    rng = np.random.default_rng(301)
    A = []
    for d in dims:
        a = rng.random((d, k))
        a[rng.random(a.shape) < 0.5] = 0.0
        A.append(a)
    X = _synth(gpu, torch, dev, dims, A, _sigma(A, 0.01), 31)
    F0 = [np.random.default_rng(302).random((d, k)) for d in dims]
    out = {}
    for prec in ("bf16x2", "bf16", "fp64"):
        with gpu.Context(dev, prec) as c:
            c.set_tensor(X.data_ptr(), dims=dims, dtype="f32")
            c.set_factors(F0)
            c.run("anlsbpp", max(args.warmup, 1), compute_error=False)
            c.set_factors(F0)
            ms, errs, _ = _time_run(torch, c, "anlsbpp", T)  # one CUDA graph per iteration
            # per-kernel breakdown and launch count from a separate run with
            # event timing (no graphs)
            c.set_factors(F0)
            c.kernel_times()
            launches, kt = _launches_per_run(c, "anlsbpp", T)
            out[prec] = (ms, errs, launches, kt)
    # headline: single BF16 (stochastically rounded tensor); the split-BF16
    # run is reported beside it
    ms, errs, launches, kt = out["bf16"]
    ms1, errs1, _, kt1 = out["bf16x2"]
    ms64, errs64, _, kt64 = out["fp64"]
    return _line(args, 1, T / (ms * 1e-3), "iters/s", ms / T, "bf16",
                 {"workload": "192^4 FP32 tensor, rank-64 sparse-factor CP + 1% noise, ANLS/BPP "
                              "k=64, 30 iterations, balanced dimension tree, BF16 tensor-core "
                              "MTTKRP", "dims": list(dims), "rank": k},
                 fp64_plain={"value": T / (ms64 * 1e-3), "unit": "iters/s", "ms_per_step": ms64 / T},
                 speedup_vs_fp64=ms64 / ms,
                 rel_error={"mixed": float(errs[-1]), "fp64": float(errs64[-1]),
                            "abs_diff": float(abs(errs[-1] - errs64[-1]))},
                 bf16x2={"value": T / (ms1 * 1e-3), "unit": "iters/s",
                              "speedup_vs_fp64": ms64 / ms1, "rel_error": float(errs1[-1]),
                              "abs_diff_vs_fp64": float(abs(errs1[-1] - errs64[-1])),
                              "kernel_ms_per_iter": {kk: round(v[0] / T, 4) for kk, v in kt1.items() if v[1]}},
                 kernel_ms_per_iter={kk: round(v[0] / T, 4) for kk, v in kt.items() if v[1]},
                 kernel_ms_per_iter_fp64={kk: round(v[0] / T, 4) for kk, v in kt64.items() if v[1]},
                 gpu_launches=launches)


def cfg4(args, gpu, torch, dev):
    T = 100
    rng = np.random.default_rng(401)
    specs = [(tuple(int(d) for d in rng.integers(32, 257, size=3)), int(rng.choice([4, 8, 16, 32])))
             for _ in range(256)]
    b = gpu.Batch(dev, "bf16", nstreams=64)
    total = 0
    for i, (dims, k) in enumerate(specs):
        r = np.random.default_rng(1000 + i)
        A = [r.random((d, k)) for d in dims]
        X = _synth(gpu, torch, dev, dims, A, _sigma(A, 0.01), 2000 + i)
        b.add(X.data_ptr(), [r.random((d, k)) for d in dims], dims=dims, dtype="f32")
        total += int(np.prod(dims))
        del X
    t0 = time.perf_counter()
    tuned_ms = b.autotune("hals", trials=2)
    tune_s = time.perf_counter() - t0
    b.run("hals", args.warmup, compute_error=False)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    errs = b.run("hals", T, compute_error=True)
    wall = time.perf_counter() - t0
    b.close()
    return _line(args, 1, T / wall, "batched iters/s (256 tensors)", 1e3 * wall / T, "bf16",
                 {"workload": "256 independent 3-way FP32 tensors, dims U{32..256}, ranks "
                              "U{4,8,16,32}, HALS, one CUDA-graph launch per batched iteration",
                  "tensors": 256, "total_elements": total},
                 timing="host wall clock around batch_run (its graph launches and the final "
                        "synchronisation), 100 iterations",
                 autotune={"best_ms_per_iter": tuned_ms, "tuning_seconds": tune_s},
                 final_rel_error={"median": float(np.median(errs[:, -1])),
                                  "max": float(np.max(errs[:, -1]))},
                 tensors_per_s=256 * T / wall)


def cfg5(args, gpu, torch, dev):
    from planc_b200.autograd import CPLoss, projected_accelerated_step
    dims, k, T = (512, 512, 512), 32, 200
    rng = np.random.default_rng(501)
    A = [rng.random((d, k)) for d in dims]
    X = _synth(gpu, torch, dev, dims, A, _sigma(A, 0.05), 51)
    lossf = CPLoss(X, dims=dims, rank=k, precision="bf16", device=dev)
    F = [torch.tensor(np.random.default_rng(502 + i).random((d, k)), device="cuda:%d" % dev,
                      dtype=torch.float64, requires_grad=True) for i, d in enumerate(dims)]
    Y = [f.detach().clone() for f in F]

    def step(F, Y, Fprev, t, eta):
        # projected accelerated gradient on all factors from one forward+backward
        for y in Y:
            y.requires_grad_(True)
            y.grad = None
        loss = lossf(*Y)
        loss.backward()
        t_next = 0.5 * (1 + (1 + 4 * t * t) ** 0.5)
        mom = (t - 1) / t_next
        with torch.no_grad():
            # F = max(Y - eta grad, 0), Y = F + mom (F - F_prev): one launch
            newF = [torch.empty_like(y) for y in Y]
            newY = [torch.empty_like(y) for y in Y]
            projected_accelerated_step(lossf, [y.detach() for y in Y], [y.grad for y in Y], Fprev,
                                       eta, mom, newF, newY)
        return newF, newY, t_next, loss.detach()

    with torch.no_grad():
        Lmax = max(float(torch.linalg.matrix_norm((F[1].T @ F[1]) * (F[2].T @ F[2]), 2)),
                   float(torch.linalg.matrix_norm((F[0].T @ F[0]) * (F[2].T @ F[2]), 2)),
                   float(torch.linalg.matrix_norm((F[0].T @ F[0]) * (F[1].T @ F[1]), 2)))
    eta = 1.0 / (3.0 * Lmax)
    Fc = [f.detach() for f in F]
    t = 1.0
    for _ in range(args.warmup):
        Fc, Y, t, l0 = step(Fc, Y, Fc, t, eta)
    Fc = [f.detach() for f in F]
    Y = [f.clone() for f in Fc]
    t = 1.0
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    losses = []
    for _ in range(T):
        Fn, Y, t, loss = step(Fc, Y, Fc, t, eta)
        Fc = Fn
        losses.append(loss)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    lv = [float(x) for x in losses]

    # The same 200 steps with forward + backward captured once as a CUDA graph
    # on the loss's stream (static factor inputs, static loss and gradient
    # outputs: PyTorch's whole-network capture, gradients set to None before
    # capture), each step one replay plus the one-launch step kernel.
    s = torch.cuda.ExternalStream(lossf.ctx.stream, device="cuda:%d" % dev)
    Ys = [f.detach().clone().requires_grad_(True) for f in F]
    bufs = [[f.detach().clone() for f in F], [torch.empty_like(f) for f in F]]
    with torch.cuda.stream(s):
        for _ in range(2):  # library buffers and the tree's state exist before capture
            for y in Ys:
                y.grad = None
            lossf(*Ys).backward()
    torch.cuda.synchronize()
    for y in Ys:
        y.grad = None
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph, stream=s, capture_error_mode="relaxed"):
        static_loss = lossf(*Ys)
        static_loss.backward()
    grads = [y.grad for y in Ys]
    with torch.no_grad():
        for y, f in zip(Ys, F):
            y.copy_(f.detach())
    torch.cuda.synchronize()
    t = 1.0
    gl = []
    g0, g1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with torch.cuda.stream(s), torch.no_grad():
        g0.record(s)
        for it in range(T):
            graph.replay()
            if it == 0 or it == T - 1:
                gl.append(static_loss.clone())
            t_next = 0.5 * (1 + (1 + 4 * t * t) ** 0.5)
            cur, nxt = bufs[it % 2], bufs[(it + 1) % 2]
            projected_accelerated_step(lossf, [y.detach() for y in Ys], grads, cur, eta,
                                       (t - 1) / t_next, nxt, [y.detach() for y in Ys])
            t = t_next
        g1.record(s)
    torch.cuda.synchronize()
    gms = g0.elapsed_time(g1)
    glv = [float(x) for x in gl]
    del graph
    lossf.close()
    return _line(args, 1, T / (gms * 1e-3), "steps/s", gms / T, "bf16",
                 {"workload": "512^3 BF16 CP loss (rank 32, 5% noise), autograd with MTTKRP "
                              "backward, 200 projected accelerated gradient steps; forward + backward "
                              "replayed as one CUDA graph per step, then the step kernel",
                  "dims": list(dims), "rank": k},
                 loss_first=glv[0], loss_last=glv[-1],
                 eager={"steps_per_s": T / (ms * 1e-3), "ms_per_step": ms / T,
                        "loss_first": lv[0], "loss_last": lv[-1]},
                 x_passes_per_step=2)


def updates(args, gpu, torch, dev):
    from bench import workload
    dims, k, T = (1024, 1024, 1024), 32, 20
    A, sigma, F0 = workload(dims, k)
    X = _synth(gpu, torch, dev, dims, A, sigma, 7)
    algos = {}
    for algo in ("mu", "hals", "anlsbpp", "aoadmm", "nesterov"):
        row = {}
        for prec in ("bf16", "fp64"):
            with gpu.Context(dev, prec) as c:
                c.set_tensor(X.data_ptr(), dims=dims, dtype="f32")
                c.set_factors(F0)
                # the warm-up captures the iteration graph the timed run replays;
                # both precisions then run T more iterations from the same state
                c.run(algo, max(args.warmup, 1), compute_error=True)
                ms, errs, _ = _time_run(torch, c, algo, T)
                r = {"iters_per_s": T / (ms * 1e-3), "ms_per_iter": ms / T,
                     "final_rel_error": float(errs[-1])}
                if prec == "bf16":
                    c.reset_update_state()
                    c.set_factors(F0)
                    c.kernel_times()
                    n, kt = _launches_per_run(c, algo, T)
                    r["launches_per_iter"] = n / T
                    r["kernel_ms_per_iter"] = {kk: round(v[0] / T, 4) for kk, v in kt.items()
                                               if v[1]}
                row[prec] = r
        row["speedup_vs_fp64"] = row["fp64"]["ms_per_iter"] / row["bf16"]["ms_per_iter"]
        row["final_error_abs_diff"] = abs(row["bf16"]["final_rel_error"] -
                                          row["fp64"]["final_rel_error"])
        algos[algo] = row
    slowest = min(algos, key=lambda a: algos[a]["bf16"]["iters_per_s"])
    v = algos[slowest]["bf16"]["iters_per_s"]
    return _line(args, 1, v, "iters/s", 1e3 / v, "bf16",
                 {"workload": "1024x1024x1024 FP32 tensor, rank-32 CP + 1% noise, 20 timed iterations "
                              "of each update (MU, HALS, ANLS/BPP, AO-ADMM, Nesterov) after the "
                              "warm-up ones, dimension tree, BF16 tensor-core MTTKRP vs the FP64 "
                              "plain path",
                  "dims": list(dims), "rank": k},
                 value_is="iters/s of the slowest update (%s), BF16" % slowest,
                 algorithms=algos)


def nmf(args, gpu, torch, dev):
    m, n, k, T = 16384, 16384, 32, 20
    rng = np.random.default_rng(601)
    A = [rng.random((m, k)), rng.random((n, k))]
    X = _synth(gpu, torch, dev, (m, n), A, _sigma(A, 0.01), 61)
    W0 = np.random.default_rng(602).random((m, k))
    H0 = np.random.default_rng(603).random((n, k))
    algos = {}
    for algo in ("mu", "hals", "anlsbpp"):
        row = {}
        for prec in ("bf16", "fp64"):
            with gpu.Context(dev, prec) as c:
                c.set_tensor(X.data_ptr(), dims=(m, n), dtype="f32")
                c.nmf_set_factors(W0, H0)
                c.nmf_run(algo, max(args.warmup, 1))
                c.nmf_set_factors(W0, H0)
                stream = torch.cuda.ExternalStream(c.stream)
                torch.cuda.synchronize()
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                _, rel = c.nmf_run(algo, T)
                e1.record(stream)
                torch.cuda.synchronize()
                ms = e0.elapsed_time(e1)
                r = {"iters_per_s": T / (ms * 1e-3), "ms_per_iter": ms / T,
                     "final_rel_error": float(rel[-1])}
                if prec == "bf16":
                    c.nmf_set_factors(W0, H0)
                    c.set_timing(True)
                    c.kernel_times()
                    n0 = c.launch_count()
                    c.nmf_run(algo, T)
                    r["launches_per_iter"] = (c.launch_count() - n0) / T
                    kt = c.kernel_times()
                    c.set_timing(False)
                    r["kernel_ms_per_iter"] = {kk: round(v[0] / T, 4) for kk, v in kt.items()
                                               if v[1]}
                    # A H (right, "contract") and A^T W (left, "contract_left"):
                    # one pass over the BF16 copy of A each
                    for cls in ("contract", "contract_left"):
                        if kt[cls][1]:
                            avg = kt[cls][0] / kt[cls][1] * 1e-3
                            r["%s_gbs" % cls] = (m * n * 2 + max(m, n) * k * 8) / avg / 1e9
                row[prec] = r
        row["speedup_vs_fp64"] = row["fp64"]["ms_per_iter"] / row["bf16"]["ms_per_iter"]
        row["final_error_abs_diff"] = abs(row["bf16"]["final_rel_error"] -
                                          row["fp64"]["final_rel_error"])
        algos[algo] = row
    v = algos["hals"]["bf16"]["iters_per_s"]
    return _line(args, 1, v, "iters/s", 1e3 / v, "bf16",
                 {"workload": "NMF of a dense 16384x16384 FP32 matrix (rank-32 nonnegative model "
                              "+ 1% noise), rank 32, 20 iterations of MU, HALS and ANLS/BPP, BF16 "
                              "tensor-core A H / A^T W vs the FP64 plain path",
                  "dims": [m, n], "rank": k},
                 value_is="HALS iters/s, BF16", algorithms=algos)


def run(args, rank, world, local):
    import torch
    import planc_b200 as gpu
    dev = local
    torch.cuda.set_device(dev)
    fn = {"cfg1": cfg1, "cfg3": cfg3, "cfg4": cfg4, "cfg5": cfg5, "updates": updates,
          "nmf": nmf}[args.workload]
    line = fn(args, gpu, torch, dev)
    if rank == 0:
        print(json.dumps(line))
