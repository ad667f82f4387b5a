"""GPU parity at the benchmark configurations' full sizes.

* The library's device generator and the oracle's host generator give the
  same tensor (both arms of the benchmark factorise the same data).
* FP64 GPU path vs the CPU oracle (itself pinned to the reference's own code
  by tests/test_oracle.py) for two outer iterations of the 1024^3 rank-32
  workload (HALS, MU) and of the 192^4 rank-64 sparse-factor workload
  (ANLS/BPP), to 1e-10 relative: factors, lambda and per-iteration errors.
* Batched BPP at one mode of the 192^4 rank-64 workload: the GPU solve of the
  mode's normal equations (G, M) against the reference's own BPPNNLS, passive
  sets identical outside near ties.
"""
import numpy as np
import pytest

from helpers import rel

pytestmark = pytest.mark.gpu


def _workload(dims, k, seed, zero_frac=0.0, noise=0.01):
    rng = np.random.default_rng(seed)
    A = [rng.random((d, k)) for d in dims]
    if zero_frac:
        for a in A:
            a[rng.random(a.shape) < zero_frac] = 0.0
    G = np.ones((k, k))
    for a in A:
        G *= a.T @ a
    sigma = noise * np.sqrt(G.sum() / float(np.prod(dims)))
    F0 = [np.random.default_rng(seed + 1).random((d, k)) for d in dims]
    return A, sigma, F0


def _device_tensor(gpu, dims, A, sigma, seed, dtype="f64"):
    import torch
    n = int(np.prod(dims))
    x = torch.empty(n, dtype=torch.float64 if dtype == "f64" else torch.float32, device="cuda:0")
    gpu.synth_cp_tensor(0, x.data_ptr(), dtype, dims, A, sigma, seed, clip=True)
    torch.cuda.synchronize()
    return x


def test_device_and_host_generators_agree(gpu, oracle_lib):
    dims, k = (37, 29, 23), 5
    A, sigma, _ = _workload(dims, k, 3, noise=0.05)
    xd = _device_tensor(gpu, dims, A, sigma, 11).cpu().numpy()
    xh = oracle_lib.synth_cp(dims, A, sigma, 11).ravel(order="F")
    assert np.max(np.abs(xd - xh)) <= 1e-13 * np.abs(xh).max()
    xf = _device_tensor(gpu, dims, A, sigma, 11, "f32").cpu().numpy().astype(np.float64)
    xr = oracle_lib.synth_cp(dims, A, sigma, 11, round_f32=True).ravel(order="F")
    # FP32 rounding of values equal to ~1e-15 can differ by one FP32 ulp
    ulp = np.spacing(np.abs(xr).astype(np.float32)).astype(np.float64)
    assert np.all(np.abs(xf - xr) <= ulp)
    assert np.mean(xf != xr) < 1e-3


def _fp64_run(gpu, x, dims, F0, algo, iters):
    with gpu.Context(0, "fp64") as c:
        c.set_tensor(x.data_ptr(), dims=dims, dtype="f64")
        c.set_factors(F0)
        errs = c.run(algo, iters)
        F, lam = c.get_factors()
    return F, lam, errs


@pytest.mark.parametrize("algo", ["hals", "mu"])
def test_fp64_1024cube_rank32_matches_oracle(gpu, oracle_lib, algo):
    dims, k, iters = (1024, 1024, 1024), 32, 2
    A, sigma, F0 = _workload(dims, k, 2024)
    x = _device_tensor(gpu, dims, A, sigma, 7)
    F, lam, errs = _fp64_run(gpu, x, dims, F0, algo, iters)
    X = x.cpu().numpy().reshape(dims, order="F")
    del x
    Fo, lamo, eo = oracle_lib.ntf_run(X, F0, algo, iters, dimtree=True)
    for a, b in zip(F, Fo):
        assert rel(a, b) < 1e-10
    assert rel(lam, lamo) < 1e-10
    assert np.max(np.abs(errs - eo) / eo) < 1e-10


def test_fp64_192x4_rank64_anlsbpp_matches_oracle(gpu, oracle_lib):
    dims, k, iters = (192, 192, 192, 192), 64, 2
    A, sigma, F0 = _workload(dims, k, 2025, zero_frac=0.5)
    x = _device_tensor(gpu, dims, A, sigma, 7)
    F, lam, errs = _fp64_run(gpu, x, dims, F0, "anlsbpp", iters)
    X = x.cpu().numpy().reshape(dims, order="F")
    del x
    Fo, lamo, eo = oracle_lib.ntf_run(X, F0, "anlsbpp", iters, dimtree=True)
    for a, b in zip(F, Fo):
        assert rel(a, b) < 1e-10
        # BPP's zeros are exact: the active sets agree entry by entry
        assert np.array_equal(a > 0, b > 0)
    assert rel(lam, lamo) < 1e-10
    assert np.max(np.abs(errs - eo) / eo) < 1e-10


@pytest.mark.skipif(not __import__("oracle").ref_available(), reason="reference build absent")
def test_bpp_config3_mode_masks_match_reference(gpu, oracle_lib):
    # one mode of the 192^4 rank-64 sparse-factor workload after one ANLS/BPP
    # iteration: (G, M) from the device, solved by the GPU's batched BPP and
    # by the reference's own BPPNNLS (nnls/bppnnls.hpp:67-191)
    dims, k = (192, 192, 192, 192), 64
    A, sigma, F0 = _workload(dims, k, 2025, zero_frac=0.5)
    x = _device_tensor(gpu, dims, A, sigma, 7)
    with gpu.Context(0, "fp64") as c:
        c.set_tensor(x.data_ptr(), dims=dims, dtype="f64")
        del x
        c.set_factors(F0)
        c.run("anlsbpp", 1)
        G, M = c.mode_begin(0)
        Xg, P, _ = c.bpp_solve(G, M.T)
    Xr, _ = oracle_lib.ref_bpp_solve(G, M.T)
    # near ties: entries whose value in either solution is below 1e-9 of the
    # column's largest are excluded from the mask comparison
    scale = np.maximum(np.abs(Xr).max(axis=0, keepdims=True), 1e-300)
    tie = (np.abs(Xr) < 1e-9 * scale) & (np.abs(Xg) < 1e-9 * scale)
    mg, mr = Xg > 0, Xr > 0
    assert np.array_equal(mg | tie, mr | tie)
    assert np.mean(mg != mr) < 1e-3
    assert rel(Xg, Xr) < 1e-9
