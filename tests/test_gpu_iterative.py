"""GPU parity of the iterative updates -- AO-ADMM (ntf/ntfaoadmm.hpp) and the
Nesterov-accelerated update with its extrapolation step (ntf/ntfnes.hpp) --
against the CPU oracle, through the C ABI.

Bars: the FP64 path agrees with the oracle to 1e-10 relative (max-abs error
over max-abs value) in every reported error, factor and lambda, from the same
tensor and initial factors over the same iteration count. The runs are long
enough (20 iterations) for the Nesterov acceleration (from iteration 6 on) to
be both accepted and rejected. The tensor-core paths reach the FP64 path's
final error within the bounds of tests/test_gpu_tc.py (1e-3 for bf16 at 64^3,
1e-4 for bf16x2).

AO-ADMM normalises its dual variable column by column after every update
(ntf/ntfaoadmm.hpp:74). A dual column whose constraints all turn inactive
within the update is zero only up to rounding, (u + (x - u)) - x, and the
normalisation blows that residue up to a unit vector, so two implementations
whose x differ in the last bit can split there (the reference on two BLAS
libraries would too). The parity cases are ones where that does not happen
within the run: rank = data rank, or few more components than the data has.
Ranks far above the data's (40 components on rank-6 data) split this way."""
import numpy as np
import pytest

from helpers import cp_tensor, init_factors, rel

pytestmark = pytest.mark.gpu
TOL = 1e-10


def _run(gpu, X, F0, algo, iters, prec="fp64", dimtree=True):
    with gpu.Context(0, prec) as c:
        c.set_tensor(X if prec == "fp64" else X.astype(np.float32))
        c.set_factors(F0)
        e = c.run(algo, iters, dimtree=dimtree, compute_error=True)
        F, lam = c.get_factors()
    return F, lam, e


@pytest.mark.parametrize("algo", ["aoadmm", "nesterov"])
# the cases cover the row-per-warp forms of the cluster kernels (1, 4 and 8
# rows at rank <= 32; 1 and 4 at rank <= 64) and their global-memory forms
# beyond them (1100 rows)
@pytest.mark.parametrize("dims,k,rank", [((20, 18, 16), 5, 5), ((300, 40, 33), 8, 6),
                                         ((9, 8, 7, 10), 4, 4), ((50, 45, 40), 40, 40),
                                         ((800, 12, 10), 6, 6), ((1100, 12, 10), 6, 6),
                                         ((260, 48, 44), 40, 40)])
def test_iterative_update_matches_oracle(gpu, oracle_lib, algo, dims, k, rank):
    iters = 20
    X, _ = cp_tensor(dims, rank, noise=0.01, seed=51)
    F0 = init_factors(dims, k, seed=52)
    Fo, lamo, eo = oracle_lib.ntf_run(X, F0, algo, iters, dimtree=True)
    F, lam, e = _run(gpu, X, F0, algo, iters)
    assert rel(e, eo) < TOL, (e, eo)
    for a, b in zip(F, Fo):
        assert rel(a, b) < TOL
    assert rel(lam, lamo) < TOL


@pytest.mark.parametrize("algo", ["aoadmm", "nesterov"])
def test_iterative_update_direct_mttkrp(gpu, oracle_lib, algo):
    dims, k, iters = (16, 12, 14), 6, 12
    X, _ = cp_tensor(dims, k, noise=0.01, seed=53)
    F0 = init_factors(dims, k, seed=54)
    Fo, lamo, eo = oracle_lib.ntf_run(X, F0, algo, iters, dimtree=False)
    F, lam, e = _run(gpu, X, F0, algo, iters, dimtree=False)
    assert rel(e, eo) < TOL
    for a, b in zip(F, Fo):
        assert rel(a, b) < TOL


def test_nesterov_state_persists_and_resets(gpu):
    # the proximal iterate, previous iterate and acceleration counters live in
    # the context like the members of an NTFNES object: a second call continues
    # from them, planc_gpu_reset_update_state returns to a new object
    dims, k = (20, 18, 16), 5
    X, _ = cp_tensor(dims, k, noise=0.01, seed=55)
    F0 = init_factors(dims, k, seed=56)
    with gpu.Context(0, "fp64") as c:
        c.set_tensor(X)
        c.set_factors(F0)
        e1 = c.run("nesterov", 8)
        c.set_factors(F0)
        e2 = c.run("nesterov", 8)
        c.reset_update_state()
        c.set_factors(F0)
        e3 = c.run("nesterov", 8)
    assert rel(e3, e1) < 1e-14
    assert rel(e2, e1) > 1e-6


@pytest.mark.parametrize("prec", ["bf16", "bf16x2"])
@pytest.mark.parametrize("algo", ["aoadmm", "nesterov"])
def test_iterative_update_tensor_cores(gpu, prec, algo):
    dims, k, iters = (64, 64, 64), 8, 20
    X, _ = cp_tensor(dims, k, noise=0.01, seed=57)
    F0 = init_factors(dims, k, seed=58)
    _, _, e64 = _run(gpu, X, F0, algo, iters)
    _, _, e = _run(gpu, X, F0, algo, iters, prec=prec)
    assert np.all(np.isfinite(e))
    tol = 1e-4 if prec == "bf16x2" else 1e-3
    assert abs(e[-1] - e64[-1]) < tol, (e[-1], e64[-1])


def test_nesterov_4way_tensor_cores(gpu):
    # the balanced 4-way tree evaluates the extrapolation's error through the
    # last mode's MTTKRP of that tree
    dims, k, iters = (24, 20, 32, 28), 6, 12
    X, _ = cp_tensor(dims, k, noise=0.01, seed=59)
    F0 = init_factors(dims, k, seed=60)
    _, _, e64 = _run(gpu, X, F0, "nesterov", iters)
    _, _, e = _run(gpu, X, F0, "nesterov", iters, prec="bf16x2")
    assert abs(e[-1] - e64[-1]) < 1e-4, (e[-1], e64[-1])


def test_objective_error_balanced_4way(gpu, oracle_lib):
    # the Gram-form error of a 4-way tensor on the balanced tree takes <X, M>
    # from the tree's last-mode MTTKRP
    dims, k = (24, 20, 32, 28), 6
    X, _ = cp_tensor(dims, k, noise=0.01, seed=61)
    F0 = init_factors(dims, k, seed=62)
    Fn = [f / np.linalg.norm(f, axis=0) for f in F0]
    ref = oracle_lib.explicit_error(X, Fn, np.ones(k))
    with gpu.Context(0, "bf16x2") as c:
        c.set_tensor(X.astype(np.float32))
        c.set_factors(F0)
        assert abs(c.objective_error() - ref) < 1e-4


@pytest.mark.parametrize("dims", [(20, 18, 16), (1100, 12, 10)])
def test_nesterov_step_cap_reports_maxiter(gpu, monkeypatch, dims):
    # an inner loop that the step cap stops (here 2 steps, set for the
    # context through PLANC_GPU_NES_MAX_STEPS) ends with PLANC_GPU_ERR_MAXITER,
    # in the register-resident form and in the global-memory form (1100 rows);
    # a context created without the setting then runs normally
    k = 5
    X, _ = cp_tensor(dims, k, noise=0.01, seed=63)
    F0 = init_factors(dims, k, seed=64)
    monkeypatch.setenv("PLANC_GPU_NES_MAX_STEPS", "2")
    with gpu.Context(0, "fp64") as c:
        c.set_tensor(X)
        c.set_factors(F0)
        with pytest.raises(gpu.PlancGpuError) as ei:
            c.run("nesterov", 3)
        assert ei.value.code == -10
    monkeypatch.delenv("PLANC_GPU_NES_MAX_STEPS")
    with gpu.Context(0, "fp64") as c:
        c.set_tensor(X)
        c.set_factors(F0)
        e = c.run("nesterov", 3)
    assert np.all(np.isfinite(e))
