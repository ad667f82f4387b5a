"""CPU timing harness for the reference algorithm (test / baseline
infrastructure only; used by bench.py's cpu_baseline and --impl reference legs).

Runs the AUNTF outer loop (ntf/auntf.hpp:128-177) on the host: the MTTKRPs go
through the reference's own dimension-tree kernels (oracle/_ref, compiled from
dimtree/dimtrees.hpp + dimtree/ddttensor.hpp) driven as DenseDimensionTree does
(set_factor after every update, ddt.hpp:93-98), when that build is present,
else through the oracle's restatement; the Gram, update and normalisation steps
are the oracle's restatement (OpenBLAS / plain C++).
"""
import ctypes
import time

import numpy as np

from . import (ALGO, _fptrs, _pd, gram_loo, hals_update, lib, mu_update, normalize, ref,
               ref_available, bpp_update)


def run_timed(X, F0, algo, iters, nthreads, use_ref=True):
    """Returns (seconds per outer iteration, final factors). X: Fortran-order
    float64. Timing excludes set-up (tensor norm, tree allocation)."""
    X = np.asfortranarray(X, dtype=np.float64)
    k = F0[0].shape[1]
    N = X.ndim
    F = []
    for f in F0:
        fn, _ = normalize(f)
        F.append(fn)
    use_ref = use_ref and ref_available() and N in (3, 4)
    h = None
    if use_ref:
        R = ref()
        dims = (ctypes.c_long * N)(*X.shape)
        h = R.ref_dimtree_create(_pd(X), dims, N, k, _fptrs(F), nthreads)
    try:
        t0 = time.perf_counter()
        for it in range(iters):
            for n in range(N):
                G = gram_loo(F, n)
                M = np.zeros((X.shape[n], k))
                if use_ref:
                    R.ref_dimtree_mttkrp(h, n, _pd(M))
                else:
                    from . import mttkrp_direct
                    M = mttkrp_direct(X, F, n)
                if algo == "hals":
                    H = hals_update(F[n], M, G)
                elif algo == "mu":
                    H = mu_update(F[n], M, G)
                else:
                    H, _, rc = bpp_update(M, G)
                    if rc < 0:
                        raise RuntimeError("BPP failed")
                H, lam = normalize(H)
                F[n] = H
                if use_ref:
                    R.ref_dimtree_set_factor(h, n, _pd(F[n]))
        dt = time.perf_counter() - t0
    finally:
        if h is not None:
            R.ref_dimtree_destroy(h)
    return dt / max(iters, 1), F
