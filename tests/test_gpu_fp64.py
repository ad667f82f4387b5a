"""GPU parity of the FP64 plain path against the CPU oracle, through the C ABI.

Tolerance: the north-star bar for FP64, 1e-10 relative (max-abs error over
max-abs value) for factors, MTTKRPs, Grams and relative errors."""
import numpy as np
import pytest

from helpers import cp_tensor, einsum_mttkrp, init_factors, rel

pytestmark = pytest.mark.gpu
TOL = 1e-10


def _ctx(gpu, X, F, prec="fp64"):
    c = gpu.Context(0, prec)
    c.set_tensor(X)
    c.set_factors(F)
    return c


def _normalized(F):
    return [f / np.linalg.norm(f, axis=0) for f in F]


@pytest.mark.parametrize("dims,k", [((64, 64, 64), 8), ((17, 23, 9), 5), ((12, 10, 8, 6), 12),
                                    ((40, 33, 21), 32), ((9, 8, 7, 10), 64), ((30, 20, 10), 1)])
def test_mttkrp_and_gram(gpu, oracle_lib, dims, k):
    X, _ = cp_tensor(dims, 3, seed=1)
    F = init_factors(dims, k, seed=2)
    with _ctx(gpu, X, F) as c:
        Fn = _normalized(F)  # set_factors normalises like AUNTF::reset
        for n in range(len(dims)):
            ref = oracle_lib.mttkrp_direct(X, Fn, n)
            assert rel(c.mttkrp(n, dimtree=False), ref) < TOL
            if len(dims) in (3, 4):
                assert rel(c.mttkrp(n, dimtree=True), ref) < TOL
            assert rel(c.gram_loo(n), oracle_lib.gram_loo(Fn, n)) < TOL


def test_direct_mttkrp_five_modes(gpu, oracle_lib):
    dims, k = (5, 4, 6, 3, 4), 6
    X, _ = cp_tensor(dims, 2, seed=3)
    F = init_factors(dims, k, seed=4)
    with _ctx(gpu, X, F) as c:
        Fn = _normalized(F)
        for n in range(5):
            assert rel(c.mttkrp(n, dimtree=False), einsum_mttkrp(X, Fn, n)) < TOL


@pytest.mark.parametrize("algo", ["hals", "mu", "anlsbpp"])
# (5000, 7, 6): a factor above the one-cluster normalisation's 4096 rows
# (multi-CTA Gram partials, fixed-order finish, column scaling)
@pytest.mark.parametrize("dims,k,iters", [((64, 64, 64), 8, 20), ((20, 31, 17, 9), 6, 6),
                                          ((5000, 7, 6), 5, 6)])
def test_ntf_run_matches_oracle(gpu, oracle_lib, algo, dims, k, iters):
    X, _ = cp_tensor(dims, k, noise=0.01, seed=7)
    F0 = init_factors(dims, k, seed=8)
    Fo, lamo, eo = oracle_lib.ntf_run(X, F0, algo, iters, dimtree=True)
    for dimtree in (True, False):
        with _ctx(gpu, X, F0) as c:
            e = c.run(algo, iters, dimtree=dimtree, compute_error=True)
            F, lam = c.get_factors()
        assert rel(e, eo) < TOL, (e, eo)
        for a, b in zip(F, Fo):
            assert rel(a, b) < TOL
        assert rel(lam, lamo) < TOL


def test_run_in_pieces_equals_one_run(gpu, oracle_lib):
    X, _ = cp_tensor((30, 25, 20), 5, seed=9)
    F0 = init_factors(X.shape, 5, seed=10)
    # the second call needs a larger error buffer: the cached graph must be
    # rebuilt around it
    with _ctx(gpu, X, F0) as c:
        e1 = np.concatenate([c.run("hals", 3), c.run("hals", 9)])
        F1, _ = c.get_factors()
    with _ctx(gpu, X, F0) as c:
        e2 = c.run("hals", 12)
        F2, _ = c.get_factors()
    assert rel(e1, e2) < 1e-14
    assert all(rel(a, b) < 1e-14 for a, b in zip(F1, F2))


def test_objective_error_matches_explicit(gpu, oracle_lib):
    X, _ = cp_tensor((25, 20, 15), 4, seed=11)
    F0 = init_factors(X.shape, 4, seed=12)
    Fo, lamo, eo = oracle_lib.ntf_run(X, F0, "hals", 3)
    with _ctx(gpu, X, F0) as c:
        c.run("hals", 3, compute_error=False)
        err = c.objective_error()
    assert abs(err - eo[-1]) / eo[-1] < TOL


def test_host_update_extension_point(gpu, oracle_lib):
    # A host-side update (the reference's virtual AUNTF::update) driven by
    # mode_begin / mode_end reproduces the oracle's HALS iteration.
    X, _ = cp_tensor((16, 14, 12), 4, seed=13)
    F0 = init_factors(X.shape, 4, seed=14)
    Fo, lamo, eo = oracle_lib.ntf_run(X, F0, "hals", 2)
    with _ctx(gpu, X, F0) as c:
        F, _ = c.get_factors()
        for it in range(2):
            for n in range(3):
                G, M = c.mode_begin(n)
                H = oracle_lib.hals_update(F[n], M, G)
                c.mode_end(n, H)
                F, _ = c.get_factors()
        err = c.objective_error()
        F, lam = c.get_factors()
    assert all(rel(a, b) < TOL for a, b in zip(F, Fo))
    assert abs(err - eo[-1]) / eo[-1] < TOL


# the batched BPP kernels: a warp per right-hand side, a CTA per right-hand
# side (k > 16), and the library's choice by size
BPP_KERNELS = ["warp", "cta", None]


@pytest.mark.parametrize("kern", BPP_KERNELS)
@pytest.mark.parametrize("n", [3, 8, 17, 40, 64])
def test_bpp_solve_masks_and_values(gpu, oracle_lib, n, kern, monkeypatch):
    if kern:
        monkeypatch.setenv("PLANC_GPU_BPP_KERNEL", kern)
    rng = np.random.default_rng(100 + n)
    A = rng.random((2 * n, n))
    A[:, rng.random(n) < 0.3] *= 0.1
    AtA = A.T @ A
    B = rng.standard_normal((n, 300)) + 0.2
    Xo, Po, ito = oracle_lib.bpp_update(B.T.copy(), AtA)
    with gpu.Context(0, "fp64") as c:
        Xg, Pg, itg = c.bpp_solve(AtA, B)
    assert rel(Xg.T, Xo) < 1e-9
    assert np.array_equal(Pg.T, Po)
    assert itg.max() <= 5 * n


@pytest.mark.parametrize("kern", ["warp", "cta"])
def test_bpp_kernels_ntf_match_oracle(gpu, oracle_lib, kern, monkeypatch):
    # rank 36 (the CTA kernel's 64-column instance) with warm starts from the
    # second iteration on, against the oracle's cold-start run
    monkeypatch.setenv("PLANC_GPU_BPP_KERNEL", kern)
    dims, k, iters = (60, 50, 45), 36, 6
    rng = np.random.default_rng(81)
    A = [rng.random((d, k)) * (rng.random((d, k)) < 0.6) for d in dims]
    X = np.einsum("az,bz,cz->abc", *A)
    X = np.asfortranarray(np.maximum(X + 0.01 * X.std() * rng.standard_normal(dims), 0.0))
    F0 = init_factors(dims, k, seed=82)
    with gpu.Context(0, "fp64") as c:
        c.set_tensor(X)
        c.set_factors(F0)
        e = c.run("anlsbpp", iters)
        F, lam = c.get_factors()
    Fo, lo, eo = oracle_lib.ntf_run(X, F0, "anlsbpp", iters)
    assert all(rel(a, b) < 1e-10 for a, b in zip(F, Fo))
    assert np.max(np.abs(e - eo) / eo) < 1e-10


def test_bpp_warm_start_reaches_the_same_factors(gpu, oracle_lib):
    # the ANLS/BPP rows start from the replaced factor's passive set by
    # default; the unique NNLS optima, hence the factors, equal the cold-start
    # (reference, bppnnls.hpp:73-74) run and the oracle's
    dims, k, iters = (40, 36, 28, 24), 10, 12
    rng = np.random.default_rng(71)
    A = [rng.random((d, k)) * (rng.random((d, k)) < 0.5) for d in dims]
    X = np.einsum("az,bz,cz,dz->abcd", *A)
    X = np.asfortranarray(np.maximum(X + 0.01 * X.std() * rng.standard_normal(dims), 0.0))
    F0 = init_factors(dims, k, seed=72)
    res = {}
    for warm in (True, False):
        with gpu.Context(0, "fp64") as c:
            c.set_tensor(X)
            c.set_factors(F0)
            c.set_bpp_warm_start(warm)
            e = c.run("anlsbpp", iters)
            F, lam = c.get_factors()
            res[warm] = (F, lam, e)
    Fo, lo, eo = oracle_lib.ntf_run(X, F0, "anlsbpp", iters)
    for warm in (True, False):
        F, lam, e = res[warm]
        assert all(rel(a, b) < 1e-10 for a, b in zip(F, Fo)), warm
        assert np.max(np.abs(e - eo) / eo) < 1e-10, warm


@pytest.mark.parametrize("n,kern", [(4, None), (40, "warp"), (40, "cta")])
def test_bpp_singular_normal_equations_reports_status(gpu, n, kern, monkeypatch):
    # AtA with a zero row/column at an index that enters the passive set:
    # the solve has no pivot; the call returns ERR_SINGULAR and the context
    # stays usable.
    if kern:
        monkeypatch.setenv("PLANC_GPU_BPP_KERNEL", kern)
    AtA = np.eye(n)
    AtA[2, 2] = 0.0
    B = np.ones((n, 3))
    with gpu.Context(0, "fp64") as c:
        with pytest.raises(gpu.PlancGpuError) as ei:
            c.bpp_solve(AtA, B)
        assert ei.value.code == -9
        X, P, it = c.bpp_solve(np.eye(n), B)
        assert np.allclose(X, 1.0)


def test_argument_errors(gpu):
    X, _ = cp_tensor((8, 8, 8), 2, seed=1)
    with gpu.Context(0, "fp64") as c:
        with pytest.raises(gpu.PlancGpuError) as ei:
            c.run("hals", 1)
        assert ei.value.code == -3  # no tensor yet
        c.set_tensor(X)
        with pytest.raises(gpu.PlancGpuError) as ei:
            c.set_factors(init_factors(X.shape, 65))
        assert ei.value.code == -7
        c.set_factors(init_factors(X.shape, 4))
        with pytest.raises(gpu.PlancGpuError):
            c.mttkrp(-1)
        with pytest.raises(gpu.PlancGpuError):
            c.run(7, 1)
        c.run("hals", 1)


def test_synth_generator_matches_model(gpu):
    import torch
    dims, k = (20, 16, 12), 3
    A = init_factors(dims, k, seed=5)
    x = torch.empty(int(np.prod(dims)), dtype=torch.float64, device="cuda")
    gpu.synth_cp_tensor(0, x.data_ptr(), "f64", dims, A, 0.0, 1, clip=False)
    M = np.einsum("az,bz,cz->abc", *A).ravel(order="F")
    assert rel(x.cpu().numpy(), M) < 1e-14
    y = torch.empty_like(x)
    gpu.synth_cp_tensor(0, y.data_ptr(), "f64", dims, A, 0.5, 42, clip=False)
    z = (y - x).cpu().numpy() / 0.5
    assert abs(z.mean()) < 0.05 and abs(z.std() - 1) < 0.05


def _golden():
    import importlib.util
    import os
    gold = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
    spec = importlib.util.spec_from_file_location("make_golden", os.path.join(gold, "make_golden.py"))
    mg = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mg)
    return mg, np.load(os.path.join(gold, "ref_ntf_runs.npz"))


_MG, _G = _golden()


@pytest.mark.parametrize("name,algo", [(n, a) for n, _, _, _, _, al, _, _ in _MG.RUNS for a in al])
def test_ntf_run_matches_reference_golden(gpu, name, algo):
    # the FP64 GPU path against whole runs of the reference's own AUNTF
    # (tests/golden/ref_ntf_runs.npz; the 64^3 rank-8 HALS/MU/BPP runs of
    # 20 iterations are the benchmark's configuration 1)
    dims = tuple(int(d) for d in _G[name + "_dims"])
    k, iters, dt, seed = (int(v) for v in _G[name + "_meta"])
    X, F0 = _MG.run_inputs(dims, k, float(_G[name + "_noise"][0]), seed)
    with _ctx(gpu, X, F0) as c:
        e = c.run(algo, iters, dimtree=bool(dt), compute_error=True)
        F, lam = c.get_factors()
    pre = "%s_%s_" % (name, algo)
    for i in range(len(dims)):
        assert rel(F[i], _G[pre + "F%d" % i]) < TOL, i
    assert rel(lam, _G[pre + "lam"]) < TOL
    ref_err = _G[pre + "err"]
    if algo == "nesterov":
        assert abs(e[-1] - ref_err[-1]) <= TOL * ref_err[-1]
    else:
        assert np.max(np.abs(e - ref_err) / ref_err) < TOL


@pytest.mark.parametrize("prec,dtype", [("fp64", np.float64), ("fp64", np.float32),
                                        ("bf16", np.float32), ("bf16x2", np.float64)])
def test_set_tensor_host_and_device_sources_agree(gpu, prec, dtype):
    # a tensor of several upload chunks (64 MiB each), with a ragged last one:
    # host memory (through the staging buffer) and device memory (in place)
    # give the same resident copy bit for bit, and re-uploading a tensor of the
    # same shape into the same context reuses its buffers
    import torch
    dims, k = (301, 283, 203), 4
    rng = np.random.default_rng(91)
    X = np.asfortranarray(rng.random(dims).astype(dtype))
    F = init_factors(dims, k, seed=92)
    xd = torch.tensor(X.ravel(order="F"), device="cuda")
    with gpu.Context(0, prec) as a, gpu.Context(0, prec) as b:
        a.set_tensor(X)
        b.set_tensor(xd.data_ptr(), dims=dims, dtype="f64" if dtype == np.float64 else "f32")
        a.set_factors(F)
        b.set_factors(F)
        assert a.tensor_norm2() == b.tensor_norm2()
        assert abs(a.tensor_norm2() - float(np.sum(X.astype(np.float64) ** 2))) < 1e-12 * a.tensor_norm2()
        for n in range(3):
            assert np.array_equal(a.mttkrp(n), b.mttkrp(n))
        m0 = a.mttkrp(0)
        a.set_tensor(X)
        a.set_factors(F)
        assert np.array_equal(a.mttkrp(0), m0)
