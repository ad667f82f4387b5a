"""GPU test of the allocation-free last-mode MTTKRP entry point
(planc_gpu_mttkrp_last_mode_noalloc), called through the C ABI.

That entry point is for callers that cannot allocate device memory when they
call the library (pool-reserved GPU memory, latency-critical loops that must
not pay an allocation's implicit synchronisation); its split-K partials live
in a fixed device array shared by every call. The test compares it with the
existing MTTKRP entry point (planc_gpu_mttkrp, direct form, FP64) on two calls
in a row with different tensors, at the FP64 tolerance of the other tests
(1e-10 relative), and checks the size limit. This file is collected last."""
import ctypes

import numpy as np
import pytest

from helpers import cp_tensor, init_factors, rel

pytestmark = pytest.mark.gpu
TOL = 1e-10


def _noalloc(gpu, X, F, k):
    import torch
    lib = gpu.load()
    fn = lib.planc_gpu_mttkrp_last_mode_noalloc
    fn.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int64), ctypes.c_int,
                   ctypes.POINTER(ctypes.c_void_p), ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p]
    fn.restype = ctypes.c_int
    xd = torch.tensor(np.asfortranarray(X).ravel(order="F"), device="cuda", dtype=torch.float64)
    fd = [torch.tensor(np.ascontiguousarray(f), device="cuda", dtype=torch.float64) for f in F[:-1]]
    out = torch.full((X.shape[-1], k), float("nan"), device="cuda", dtype=torch.float64)
    dims = (ctypes.c_int64 * X.ndim)(*X.shape)
    ptrs = (ctypes.c_void_p * len(fd))(*[f.data_ptr() for f in fd])
    torch.cuda.synchronize()
    rc = fn(xd.data_ptr(), dims, X.ndim, ptrs, k, out.data_ptr(), None)
    torch.cuda.synchronize()
    return rc, out.cpu().numpy()


def _existing(gpu, X, F):
    with gpu.Context(0, "fp64") as c:
        c.set_tensor(X)
        c.set_factors(F)
        Fn, _ = c.get_factors()
        return c.mttkrp(X.ndim - 1, dimtree=False), Fn


def test_noalloc_matches_existing_entry_point_two_calls():
    import planc_b200 as gpu
    cases = [((40, 36, 30), 8, 1), ((24, 20, 16, 50), 32, 2)]
    for dims, k, seed in cases:  # two calls in a row, different tensors and ranks
        X, _ = cp_tensor(dims, 3, seed=seed)
        F = init_factors(dims, k, seed=seed + 10)
        ref, Fn = _existing(gpu, X, F)  # Fn: the normalised factors that call used
        rc, got = _noalloc(gpu, X, Fn, k)
        assert rc == 0, gpu.load().planc_gpu_last_error()
        assert rel(got, ref) < TOL
    # the same inputs again: the shared array's earlier contents do not leak in
    rc2, got2 = _noalloc(gpu, X, Fn, k)
    assert rc2 == 0 and rel(got2, ref) < TOL


def test_noalloc_rejects_sizes_beyond_its_scratch():
    import planc_b200 as gpu
    k = 64
    dims = (2, (1 << 20) // k + 1)
    X = np.ones(dims)
    F = [np.ones((dims[0], k)), np.ones((dims[1], k))]
    rc, _ = _noalloc(gpu, X, F, k)
    assert rc == -7
    assert b"exceeds the allocation-free scratch" in gpu.load().planc_gpu_last_error()
