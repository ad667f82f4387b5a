"""GPU parity of the shared-memory NMF (common/nmf.hpp, nmf/hals.hpp,
nmf/mu.hpp, nmf/bppnmf.hpp) against the CPU oracle, through the C ABI.

Bars: the FP64 path agrees with the oracle to 1e-10 relative (max-abs error
over max-abs value) in the objective and relative error of every iteration
and in W and H, from the same matrix and initial factors, with and without
regularisation. The tensor-core paths (A in BF16, or split hi + lo) reach
the FP64 path's final relative error within 1e-3 (bf16) / 1e-4 (bf16x2), the
bounds of the NTF tensor-core tests."""
import numpy as np
import pytest

from helpers import rel

pytestmark = pytest.mark.gpu
TOL = 1e-10


def _problem(m, n, k, seed, noise=0.01):
    rng = np.random.default_rng(seed)
    A = rng.random((m, k)) @ rng.random((k, n))
    A = np.maximum(A + noise * A.std() * rng.standard_normal(A.shape), 0.0)
    return np.asfortranarray(A), rng.random((m, k)), rng.random((n, k))


def _gpu_nmf(gpu, A, W0, H0, algo, iters, prec="fp64", reg=None):
    with gpu.Context(0, prec) as c:
        c.set_tensor(A if prec == "fp64" else A.astype(np.float32))
        c.nmf_set_factors(W0, H0)
        if reg is not None:
            c.nmf_set_regularization(reg[0:2], reg[2:4], reg[4])
        obj, re = c.nmf_run(algo, iters)
        W, H = c.nmf_get_factors()
    return W, H, obj, re


@pytest.mark.parametrize("algo", ["hals", "mu", "anlsbpp"])
@pytest.mark.parametrize("m,n,k", [(60, 45, 6), (200, 130, 16), (3000, 70, 8), (90, 120, 40)])
def test_nmf_matches_oracle(gpu, oracle_lib, algo, m, n, k):
    iters = 15
    A, W0, H0 = _problem(m, n, k, 81)
    Wo, Ho, oo, ro = oracle_lib.nmf_run(A, W0, H0, algo, iters)
    W, H, obj, re = _gpu_nmf(gpu, A, W0, H0, algo, iters)
    assert rel(obj, oo) < TOL, (obj, oo)
    assert rel(re, ro) < TOL
    assert rel(W, Wo) < TOL and rel(H, Ho) < TOL


# HALS's W sweep runs as one cooperative launch with W's rows in shared
# memory: one row a thread (40 x 3000 rows: 12 CTAs), two rows a thread (40000
# rows over all SMs), and as k + 1 launches when W does not fit (130000 rows)
@pytest.mark.parametrize("m,n,k", [(3000, 70, 40), (40000, 12, 8), (130000, 6, 3)])
def test_nmf_hals_w_sweep_forms(gpu, oracle_lib, m, n, k):
    A, W0, H0 = _problem(m, n, k, 86)
    Wo, Ho, oo, ro = oracle_lib.nmf_run(A, W0, H0, "hals", 6)
    W, H, obj, re = _gpu_nmf(gpu, A, W0, H0, "hals", 6)
    assert rel(obj, oo) < TOL and rel(re, ro) < TOL
    assert rel(W, Wo) < TOL and rel(H, Ho) < TOL


@pytest.mark.parametrize("algo", ["hals", "mu", "anlsbpp"])
def test_nmf_regularized_matches_oracle(gpu, oracle_lib, algo):
    A, W0, H0 = _problem(70, 50, 5, 82)
    reg = (0.5, 0.1, 0.3, 0.2, 0.0)
    Wo, Ho, oo, ro = oracle_lib.nmf_run(A, W0, H0, algo, 10, reg=reg)
    W, H, obj, re = _gpu_nmf(gpu, A, W0, H0, algo, 10, reg=reg)
    assert rel(obj, oo) < TOL and rel(re, ro) < TOL
    assert rel(W, Wo) < TOL and rel(H, Ho) < TOL


def test_nmf_symmetric_bpp_matches_oracle(gpu, oracle_lib):
    # symmetric NMF of a square matrix (nmf/nmf.cpp:191-199 sets W = H and
    # symm_reg = max(A)^2): BPP with the shifted Gram and right-hand side
    rng = np.random.default_rng(83)
    B = rng.random((50, 5))
    A = np.asfortranarray(B @ B.T)
    H0 = 2 * np.sqrt(A.mean() / 5) * rng.random((50, 5))
    reg = (0.0, 0.0, 0.0, 0.0, float(A.max()) ** 2)
    Wo, Ho, oo, ro = oracle_lib.nmf_run(A, H0, H0, "anlsbpp", 8, reg=reg)
    W, H, obj, re = _gpu_nmf(gpu, A, H0, H0, "anlsbpp", 8, reg=reg)
    assert rel(obj, oo) < TOL and rel(re, ro) < TOL
    assert rel(W, Wo) < TOL and rel(H, Ho) < TOL


@pytest.mark.parametrize("prec", ["bf16", "bf16x2"])
@pytest.mark.parametrize("algo", ["hals", "mu", "anlsbpp"])
def test_nmf_tensor_cores(gpu, prec, algo):
    A, W0, H0 = _problem(700, 500, 16, 84)
    _, _, _, r64 = _gpu_nmf(gpu, A, W0, H0, algo, 20)
    _, _, _, r = _gpu_nmf(gpu, A, W0, H0, algo, 20, prec=prec)
    assert np.all(np.isfinite(r))
    tol = 1e-4 if prec == "bf16x2" else 1e-3
    assert abs(r[-1] - r64[-1]) < tol, (r[-1], r64[-1])


def test_nmf_runs_continue(gpu, oracle_lib):
    # two MU runs of 5 iterations continue from each other's factors (the
    # normalisation by W after a run leaves W H^T unchanged)
    A, W0, H0 = _problem(40, 30, 4, 85)
    with gpu.Context(0, "fp64") as c:
        c.set_tensor(A)
        c.nmf_set_factors(W0, H0)
        c.nmf_run("mu", 5)
        W1, H1 = c.nmf_get_factors()
        _, r2 = c.nmf_run("mu", 5)
    _, _, _, ro = oracle_lib.nmf_run(A, W1, H1, "mu", 5)
    assert rel(r2, ro) < TOL
