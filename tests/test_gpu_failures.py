"""Failure detection without a GPU fault: bounded device waits that run out,
the BPP iteration cap, non-finite inputs, bad shapes. Every failure comes back
as a status code and the context stays usable afterwards."""
import numpy as np
import pytest

from helpers import cp_tensor, init_factors

pytestmark = pytest.mark.gpu


def test_bounded_wait_times_out_and_reports(gpu):
    st = gpu.selftest_wait_timeout(0, 0.05)
    assert st == -6  # PLANC_GPU_ERR_TIMEOUT written by the kernel
    with gpu.Context(0, "fp64") as c:  # the device is still usable
        X, _ = cp_tensor((8, 8, 8), 2, seed=1)
        c.set_tensor(X)
        c.set_factors(init_factors(X.shape, 2))
        c.run("hals", 1)


def test_cooperative_sweep_wait_times_out_and_reports(gpu):
    # the cooperative NMF W sweep's per-column wait (the routine the sweep
    # runs) with one CTA that never stores its sum: the waits run out and
    # report the timeout; no fault, no hang, the device stays usable
    assert gpu.selftest_coop_timeout(0) == -6
    with gpu.Context(0, "fp64") as c:
        rng = np.random.default_rng(9)
        A = np.asfortranarray(rng.random((300, 40)))
        c.set_tensor(A)
        c.nmf_set_factors(rng.random((300, 4)), rng.random((40, 4)))
        obj, rel = c.nmf_run("hals", 2)
        assert np.all(np.isfinite(rel))


def test_bpp_iteration_cap_reports_failure_and_recovers(gpu):
    X, _ = cp_tensor((20, 18, 16), 6, seed=3)
    F0 = init_factors(X.shape, 6, seed=4)
    with gpu.Context(0, "fp64") as c:
        c.set_tensor(X)
        c.set_factors(F0)
        c.set_bpp_max_iter(1)  # "BPP failed" (nnls/bppnnls.hpp:185-188) as a status
        with pytest.raises(gpu.PlancGpuError) as ei:
            c.run("anlsbpp", 1)
        assert ei.value.code == -4
        c.set_bpp_max_iter(0)
        c.set_factors(F0)
        e = c.run("anlsbpp", 3)
        assert np.all(np.isfinite(e))


def test_nonfinite_tensor_rejected(gpu):
    X, _ = cp_tensor((8, 9, 10), 2, seed=5)
    X[3, 4, 5] = np.nan
    with gpu.Context(0, "fp64") as c:
        with pytest.raises(gpu.PlancGpuError) as ei:
            c.set_tensor(X)
        assert ei.value.code == -5
        X[3, 4, 5] = 1.0
        c.set_tensor(X)


def test_zero_factor_column_is_handled(gpu, oracle_lib):
    # a zero column keeps lambda = 0 and stays zero (ncpfactors.hpp:346-351)
    X, _ = cp_tensor((12, 10, 8), 3, seed=6)
    F0 = init_factors(X.shape, 3, seed=7)
    F0[1][:, 2] = 0.0
    Fo, lo, eo = oracle_lib.ntf_run(X, F0, "mu", 2)
    with gpu.Context(0, "fp64") as c:
        c.set_tensor(X)
        c.set_factors(F0)
        e = c.run("mu", 2)
    assert np.allclose(e, eo, rtol=1e-10, atol=0)
