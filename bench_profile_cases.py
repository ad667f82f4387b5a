"""Small, fixed workloads for profiling single kernels of the library.

    python bench_profile_cases.py <case>

Each case builds its input on the device, runs the path a few times and
prints one line of timings. The cases are sized so that a profiler capture of
one launch holds a few GB of device memory at most while the tensors stay
larger than the 126 MB L2 (DRAM counters stay meaningful):

  f64     k_contract_f64 (FP64 path, DMMA): 512^3 tensor (FP64 copy), rank 32, HALS
  bpp     k_bpp / k_bpp_cta: ANLS/BPP normal equations of a 192-row mode at
          rank 64 taken from a 192 x 96 x 96 x 96 sparse-factor CP tensor
          after 10 iterations (passive sets of ~40, ~3 BPP steps per row),
          also repeated to 768 and 3072 right-hand sides, with either kernel
  tc3     k_tc_right / k_tc_left_fac: 512^3 FP32 tensor (BF16 copy), rank 32,
          HALS iterations
  tc4     k_tc_long (both sides) + the multi-TTVs of the balanced 4-way tree:
          128^4 FP32 tensor (BF16 copy), rank 64, HALS iterations
  cfg3it  three ANLS/BPP iterations of the 192^4 rank-64 workload (BF16), for
          a one-pass launch list at full size
  cfg4it  the 256-tensor batched HALS workload (dims U{32..256}, ranks
          U{4,8,16,32}, BF16 copies), 3 + 3 batched iterations, no autotuning
  cfg4small  the first 32 tensors of that workload (0.5 GB on the device),
          for captures of the grouped kernels
  nmf     shared-memory NMF of a dense 16384 x 16384 FP32 matrix (BF16 copy),
          rank 32: three iterations each of MU, HALS and ANLS/BPP
  upd     AO-ADMM and Nesterov NTF updates on the 1024^3 rank-32 headline
          tensor (BF16 copy): three iterations each (Nesterov's extrapolation
          runs from the sixth iteration of a call, so it is off here)
  nes     Nesterov NTF update on a 512^3 rank-32 tensor (BF16 copy): eight
          iterations in one call (the extrapolation runs from the sixth), for a
          capture of the register-resident inner kernel
  ttv     the multi-TTVs of the 3-way tensor-core path with the headline's
          intermediate: 1024 x 1024 x 64 FP32 tensor (BF16 copy), rank 32, so
          the FP32 partial MTTKRP P is 1024*1024 x 32 (134 MB > L2)
"""
import sys

import numpy as np


def _synth(gpu, torch, dims, k, seed, sparse=False):
    rng = np.random.default_rng(seed)
    A = []
    for d in dims:
        a = rng.random((d, k))
        if sparse:
            a[rng.random(a.shape) < 0.5] = 0.0
        A.append(a)
    G = np.ones((k, k))
    for a in A:
        G *= a.T @ a
    sigma = 0.01 * np.sqrt(G.sum() / float(np.prod(dims)))
    X = torch.empty(int(np.prod(dims)), dtype=torch.float32, device="cuda:0")
    gpu.synth_cp_tensor(0, X.data_ptr(), "f32", dims, A, sigma, seed + 1, clip=True)
    F0 = [np.random.default_rng(seed + 2).random((d, k)) for d in dims]
    return X, F0


def _timed(torch, ctx, fn, reps):
    stream = torch.cuda.ExternalStream(ctx.stream)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(reps):
        fn()
    e1.record(stream)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / reps


def case_bpp(gpu, torch):
    import os
    dims, k = (192, 96, 96, 96), 64
    X, F0 = _synth(gpu, torch, dims, k, 11, sparse=True)
    with gpu.Context(0, "bf16") as c:
        c.set_tensor(X.data_ptr(), dims=dims, dtype="f32")
        c.set_factors(F0)
        c.run("anlsbpp", 10, compute_error=False)
        G, M = c.mode_begin(0)
    res = {}
    # the mode's 192 right-hand sides, then the same rows repeated (more
    # right-hand sides per launch), with each batched BPP kernel
    for reps in (1, 4, 16):
        B = np.tile(M.T, (1, reps))
        for kern in ("warp", "cta"):
            os.environ["PLANC_GPU_BPP_KERNEL"] = kern
            with gpu.Context(0, "fp64") as c:
                for _ in range(3):
                    c.set_timing(True)
                    c.kernel_times()
                    Xs, P, its = c.bpp_solve(G, B)
                    ms = c.kernel_times()["bpp"][0]
                    c.set_timing(False)
            del os.environ["PLANC_GPU_BPP_KERNEL"]
            res[(reps, kern)] = (Xs, P)
            print("bpp: %d rows, k=64, %s kernel: %.1f us, BPP steps mean %.2f max %d, passive mean %.1f"
                  % (B.shape[1], kern, ms * 1e3, its.mean(), its.max(), P.sum(axis=0).mean()))
        (xw, pw), (xc, pc) = res[(reps, "warp")], res[(reps, "cta")]
        print("bpp: %d rows: masks differ in %d entries, max |X_warp - X_cta| / max |X| = %.2e"
              % (B.shape[1], int((pw != pc).sum()), np.abs(xw - xc).max() / max(np.abs(xw).max(), 1e-300)))
        if reps == 1:
            print("bpp: rows per BPP step count:", dict(enumerate(np.bincount(its).tolist())))


def case_f64(gpu, torch):
    # the FP64 path's DMMA contractions (right: P = X F_2, left: X^T KRP(F_0, F_1)):
    # 512^3 FP64 (1.07 GB), rank 32, HALS iterations
    dims, k = (512, 512, 512), 32
    X, F0 = _synth(gpu, torch, dims, k, 61)
    with gpu.Context(0, "fp64") as c:
        c.set_tensor(X.data_ptr(), dims=dims, dtype="f32")
        c.set_factors(F0)
        ms = _timed(torch, c, lambda: c.run("hals", 1, compute_error=False), 3)
    print("f64: 512^3 k=32 HALS FP64: %.3f ms per iteration" % ms)


def case_tc3(gpu, torch):
    dims, k = (512, 512, 512), 32
    X, F0 = _synth(gpu, torch, dims, k, 21)
    with gpu.Context(0, "bf16") as c:
        c.set_tensor(X.data_ptr(), dims=dims, dtype="f32")
        c.set_factors(F0)
        ms = _timed(torch, c, lambda: c.run("hals", 1, compute_error=False), 3)
    print("tc3: 512^3 k=32 HALS: %.3f ms per iteration" % ms)


def case_tc4(gpu, torch):
    dims, k = (128, 128, 128, 128), 64
    X, F0 = _synth(gpu, torch, dims, k, 31)
    with gpu.Context(0, "bf16") as c:
        c.set_tensor(X.data_ptr(), dims=dims, dtype="f32")
        c.set_factors(F0)
        ms = _timed(torch, c, lambda: c.run("hals", 1, compute_error=False), 3)
    print("tc4: 128^4 k=64 HALS: %.3f ms per iteration" % ms)


def case_cfg3it(gpu, torch):
    dims, k = (192, 192, 192, 192), 64
    X, F0 = _synth(gpu, torch, dims, k, 301, sparse=True)
    with gpu.Context(0, "bf16") as c:
        c.set_tensor(X.data_ptr(), dims=dims, dtype="f32")
        c.set_factors(F0)
        ms = _timed(torch, c, lambda: c.run("anlsbpp", 1, compute_error=True), 3)
    print("cfg3it: 192^4 k=64 ANLS/BPP: %.3f ms per iteration" % ms)


def case_ttv(gpu, torch):
    dims, k = (1024, 1024, 64), 32
    X, F0 = _synth(gpu, torch, dims, k, 41)
    with gpu.Context(0, "bf16") as c:
        c.set_tensor(X.data_ptr(), dims=dims, dtype="f32")
        c.set_factors(F0)
        c.run("hals", 2, compute_error=False)
        c.set_timing(True)
        c.kernel_times()
        c.run("hals", 3, compute_error=False)
        kt = c.kernel_times()
        c.set_timing(False)
    print("ttv: 1024x1024x64 k=32 HALS, per iteration: " +
          ", ".join("%s %.1f us" % (n, 1e3 * v[0] / 3) for n, v in kt.items() if v[1]))


def case_nmf(gpu, torch):
    m, n, k = 16384, 16384, 32
    rng = np.random.default_rng(601)
    A = [rng.random((m, k)), rng.random((n, k))]
    G = (A[0].T @ A[0]) * (A[1].T @ A[1])
    sigma = 0.01 * np.sqrt(G.sum() / float(m * n))
    X = torch.empty(m * n, dtype=torch.float32, device="cuda:0")
    gpu.synth_cp_tensor(0, X.data_ptr(), "f32", (m, n), A, sigma, 61, clip=True)
    W0 = np.random.default_rng(602).random((m, k))
    H0 = np.random.default_rng(603).random((n, k))
    out = []
    with gpu.Context(0, "bf16") as c:
        c.set_tensor(X.data_ptr(), dims=(m, n), dtype="f32")
        for algo in ("mu", "hals", "anlsbpp"):
            c.nmf_set_factors(W0, H0)
            ms = _timed(torch, c, lambda: c.nmf_run(algo, 1), 3)
            out.append("%s %.3f ms" % (algo, ms))
    print("nmf: 16384^2 k=32 per iteration: " + ", ".join(out))


def case_upd(gpu, torch):
    dims, k = (1024, 1024, 1024), 32
    X, F0 = _synth(gpu, torch, dims, k, 51)
    out = []
    with gpu.Context(0, "bf16") as c:
        c.set_tensor(X.data_ptr(), dims=dims, dtype="f32")
        for algo in ("aoadmm", "nesterov"):
            c.set_factors(F0)
            c.reset_update_state()
            ms = _timed(torch, c, lambda: c.run(algo, 1), 3)
            out.append("%s %.3f ms" % (algo, ms))
    print("upd: 1024^3 k=32 per iteration: " + ", ".join(out))


def case_nes(gpu, torch):
    dims, k = (512, 512, 512), 32
    X, F0 = _synth(gpu, torch, dims, k, 71)
    with gpu.Context(0, "bf16") as c:
        c.set_tensor(X.data_ptr(), dims=dims, dtype="f32")
        c.set_factors(F0)
        ms = _timed(torch, c, lambda: c.run("nesterov", 8), 1) / 8
    print("nes: 512^3 k=32 Nesterov: %.3f ms per iteration (8 in one call)" % ms)


def case_cfg4it(gpu, torch, members=256):
    # the batched workload of 256 uneven 3-way FP32 tensors (dims U{32..256},
    # ranks U{4,8,16,32}, BF16 copies), HALS iterations without the
    # autotuner: a launch list of one batched iteration's kernels
    import time
    rng = np.random.default_rng(401)
    specs = [(tuple(int(d) for d in rng.integers(32, 257, size=3)), int(rng.choice([4, 8, 16, 32])))
             for _ in range(members)]
    b = gpu.Batch(0, "bf16", nstreams=64)
    for i, (dims, k) in enumerate(specs):
        r = np.random.default_rng(1000 + i)
        A = [r.random((d, k)) for d in dims]
        G = np.ones((k, k))
        for a in A:
            G *= a.T @ a
        sigma = 0.01 * np.sqrt(G.sum() / float(np.prod(dims)))
        X = torch.empty(int(np.prod(dims)), dtype=torch.float32, device="cuda:0")
        gpu.synth_cp_tensor(0, X.data_ptr(), "f32", dims, A, sigma, 2000 + i, clip=True)
        b.add(X.data_ptr(), [r.random((d, k)) for d in dims], dims=dims, dtype="f32")
        del X
    b.run("hals", 3, compute_error=True)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    b.run("hals", 3, compute_error=True)
    torch.cuda.synchronize()
    print("cfg4it: %d tensors, HALS: %.3f ms per batched iteration (3 iterations, untuned)"
          % (members, (time.perf_counter() - t0) * 1e3 / 3))
    b.close()


def case_cfg4small(gpu, torch):
    case_cfg4it(gpu, torch, members=32)


CASES = {"bpp": case_bpp, "cfg4it": case_cfg4it, "cfg4small": case_cfg4small, "f64": case_f64, "nes": case_nes, "tc3": case_tc3, "tc4": case_tc4, "cfg3it": case_cfg3it,
         "ttv": case_ttv, "nmf": case_nmf, "upd": case_upd}


def main(argv):
    if len(argv) != 1 or argv[0] not in CASES:
        print("usage: python bench_profile_cases.py {%s}" % "|".join(CASES))
        return 2
    import torch

    import planc_b200 as gpu
    CASES[argv[0]](gpu, torch)
    return 0


if __name__ == "__main__":
    sys.exit(main(sys.argv[1:]))
