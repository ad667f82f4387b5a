"""planc_b200 -- B200 (sm_100a) implementation of PLANC's shared-memory NTF.

Python binding of the C ABI in ``include/planc_gpu.h`` (``libplanc_gpu.so``,
built in-tree by ``planc_b200/build.py``). There is no CPU fallback: every
call goes to the CUDA library, and importing fails loudly if the library is
missing.

Conventions follow the reference (see ``include/planc_gpu.h``): tensors are
column-major with mode 0 fastest (numpy Fortran order), factors are C-order
``(I_n, k)`` float64 arrays.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libplanc_gpu.so")

OK = 0
ERR = {
    -1: "ERR_ARG", -2: "ERR_CUDA", -3: "ERR_STATE", -4: "ERR_BPP_MAXITER",
    -5: "ERR_NONFINITE", -6: "ERR_TIMEOUT", -7: "ERR_UNSUPPORTED", -8: "ERR_OOM",
    -9: "ERR_SINGULAR", -10: "ERR_MAXITER",
}
PREC = {"fp64": 0, "bf16": 1, "bf16x2": 2}
ALGO = {"mu": 0, "hals": 1, "anlsbpp": 2, "aoadmm": 4, "nesterov": 5}
F64, F32 = 0, 1
KERNEL_CLASSES = ["contract", "ttv", "update", "normgram", "error", "reduce", "bpp", "prep",
                  "contract_left"]

# Every symbol declared in include/planc_gpu.h.
EXPORTS = [
    "planc_gpu_abi_version", "planc_gpu_last_error", "planc_gpu_create", "planc_gpu_destroy",
    "planc_gpu_stream", "planc_gpu_set_tensor", "planc_gpu_set_factors", "planc_gpu_run",
    "planc_gpu_get_factors", "planc_gpu_mttkrp", "planc_gpu_gram_loo",
    "planc_gpu_objective_error", "planc_gpu_mode_begin", "planc_gpu_mode_end",
    "planc_gpu_bpp_solve", "planc_gpu_set_timing", "planc_gpu_get_kernel_times",
    "planc_gpu_launch_count", "planc_gpu_synth_cp_tensor", "planc_gpu_mttkrp_device",
    "planc_gpu_tensor_norm2", "planc_gpu_set_bpp_max_iter", "planc_gpu_set_bpp_warm_start",
    "planc_gpu_reset_update_state", "planc_gpu_selftest_wait_timeout",
    "planc_gpu_nmf_set_factors", "planc_gpu_nmf_set_regularization", "planc_gpu_nmf_run",
    "planc_gpu_nmf_get_factors",
    "planc_gpu_batch_create", "planc_gpu_batch_add", "planc_gpu_batch_count",
    "planc_gpu_batch_set_factors", "planc_gpu_batch_run", "planc_gpu_batch_get_factors",
    "planc_gpu_batch_autotune", "planc_gpu_batch_destroy", "planc_gpu_mttkrp_last_mode_noalloc",
    "planc_gpu_update_device", "planc_gpu_gram_device", "planc_gpu_normalize_device",
    "planc_gpu_coldot_device", "planc_gpu_sync", "planc_gpu_selftest_coop_timeout",
    "planc_gpu_cp_loss_device", "planc_gpu_cp_grads_device", "planc_gpu_cp_step_device",
]


class PlancGpuError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__("%s (%d): %s" % (ERR.get(code, "ERR"), code, msg))
        self.code = code


_lib = None


def load():
    """Load libplanc_gpu.so (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError("libplanc_gpu.so is not built; run `python -m planc_b200.build`")
    L = ctypes.CDLL(LIB_PATH)
    P = ctypes.POINTER
    i32, i64, d, vp = ctypes.c_int, ctypes.c_int64, ctypes.c_double, ctypes.c_void_p
    pd, pi64, pi32 = P(d), P(i64), P(ctypes.c_int32)
    L.planc_gpu_abi_version.restype = i32
    L.planc_gpu_last_error.restype = ctypes.c_char_p
    L.planc_gpu_create.argtypes = [P(vp), i32, i32, vp]
    L.planc_gpu_destroy.argtypes = [vp]
    L.planc_gpu_stream.argtypes = [vp]
    L.planc_gpu_stream.restype = vp
    L.planc_gpu_set_tensor.argtypes = [vp, vp, i32, pi64, i32, i32]
    L.planc_gpu_set_factors.argtypes = [vp, P(pd), pd, i32]
    L.planc_gpu_run.argtypes = [vp, i32, i32, i32, i32, pd]
    L.planc_gpu_get_factors.argtypes = [vp, P(pd), pd]
    L.planc_gpu_mttkrp.argtypes = [vp, i32, i32, pd]
    L.planc_gpu_gram_loo.argtypes = [vp, i32, pd]
    L.planc_gpu_objective_error.argtypes = [vp, pd]
    L.planc_gpu_mode_begin.argtypes = [vp, i32, i32, pd, pd]
    L.planc_gpu_mode_end.argtypes = [vp, i32, pd]
    L.planc_gpu_bpp_solve.argtypes = [vp, pd, pd, i32, i64, pd, pi32, pi32]
    L.planc_gpu_set_timing.argtypes = [vp, i32]
    L.planc_gpu_get_kernel_times.argtypes = [vp, pd, pi64, i32]
    L.planc_gpu_launch_count.argtypes = [vp]
    L.planc_gpu_launch_count.restype = i64
    L.planc_gpu_synth_cp_tensor.argtypes = [i32, vp, i32, pi64, i32, P(pd), i32, d, ctypes.c_uint64,
                                            i32, vp]
    L.planc_gpu_mttkrp_device.argtypes = [vp, i32, P(vp), vp, i32]
    L.planc_gpu_tensor_norm2.argtypes = [vp, pd]
    L.planc_gpu_set_bpp_max_iter.argtypes = [vp, i32]
    L.planc_gpu_set_bpp_warm_start.argtypes = [vp, i32]
    L.planc_gpu_reset_update_state.argtypes = [vp]
    L.planc_gpu_nmf_set_factors.argtypes = [vp, pd, pd, i32]
    L.planc_gpu_nmf_set_regularization.argtypes = [vp, pd, pd, ctypes.c_double]
    L.planc_gpu_nmf_run.argtypes = [vp, i32, i32, pd, pd]
    L.planc_gpu_nmf_get_factors.argtypes = [vp, pd, pd]
    L.planc_gpu_batch_create.argtypes = [P(vp), i32, i32, i32]
    L.planc_gpu_batch_add.argtypes = [vp, vp, i32, pi64, i32, i32, P(pd), i32, P(i32)]
    L.planc_gpu_batch_count.argtypes = [vp]
    L.planc_gpu_batch_set_factors.argtypes = [vp, i32, P(pd), i32]
    L.planc_gpu_batch_run.argtypes = [vp, i32, i32, i32, pd]
    L.planc_gpu_batch_get_factors.argtypes = [vp, i32, P(pd), pd]
    L.planc_gpu_batch_autotune.argtypes = [vp, i32, i32, pd]
    L.planc_gpu_batch_destroy.argtypes = [vp]
    L.planc_gpu_mttkrp_last_mode_noalloc.argtypes = [vp, pi64, i32, P(vp), i32, vp, vp]
    L.planc_gpu_selftest_wait_timeout.argtypes = [i32, d, P(i32)]
    L.planc_gpu_update_device.argtypes = [vp, i32, vp, vp, vp, i64, i32]
    L.planc_gpu_gram_device.argtypes = [vp, vp, i64, i32, vp]
    L.planc_gpu_normalize_device.argtypes = [vp, vp, i64, i32, vp, vp, vp]
    L.planc_gpu_coldot_device.argtypes = [vp, vp, vp, i64, i32, vp]
    L.planc_gpu_sync.argtypes = [vp]
    L.planc_gpu_selftest_coop_timeout.argtypes = [i32, P(i32)]
    L.planc_gpu_cp_loss_device.argtypes = [vp, P(vp), vp, vp, vp]
    L.planc_gpu_cp_grads_device.argtypes = [vp, P(vp), vp, P(vp), vp, P(vp)]
    L.planc_gpu_cp_step_device.argtypes = [vp, P(vp), P(vp), P(vp), d, d, P(vp), P(vp)]
    for name in EXPORTS:
        getattr(L, name).restype = getattr(L, name).restype or i32
    L.planc_gpu_last_error.restype = ctypes.c_char_p
    L.planc_gpu_stream.restype = vp
    L.planc_gpu_launch_count.restype = i64
    _lib = L
    return L


def _check(rc):
    if rc != OK:
        raise PlancGpuError(rc, load().planc_gpu_last_error().decode())


def _pd(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _fptrs(F):
    arr = (ctypes.POINTER(ctypes.c_double) * len(F))()
    for i, f in enumerate(F):
        arr[i] = _pd(f)
    return arr


def _vps(ptrs):
    return (ctypes.c_void_p * len(ptrs))(*[int(p) for p in ptrs])


def _c64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


class Context:
    """One device-resident tensor + CP factors + stream (planc_gpu_ctx)."""

    def __init__(self, device=0, precision="fp64", stream=None):
        L = load()
        h = ctypes.c_void_p()
        _check(L.planc_gpu_create(ctypes.byref(h), device, PREC[precision], stream))
        self.h = h
        self.precision = precision
        self.device = device
        self.dims = None
        self.k = None
        # bumped by every call that may leave new dimension-tree intermediates
        # in the context (a caller that wants to reuse them checks it)
        self.tree_epoch = 0

    def close(self):
        if self.h:
            load().planc_gpu_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    @property
    def stream(self):
        return load().planc_gpu_stream(self.h)

    def set_tensor(self, X, dims=None, dtype=None):
        """X: numpy array (any shape; Fortran order = mode 0 fastest), or a
        device pointer (int) with explicit dims and dtype ('f32'/'f64')."""
        self.tree_epoch += 1
        L = load()
        if isinstance(X, np.ndarray):
            dims = X.shape
            if X.dtype == np.float32:
                dt, arr = F32, np.asfortranarray(X)
            else:
                dt, arr = F64, np.asfortranarray(X, dtype=np.float64)
            ptr, on_dev = arr.ctypes.data_as(ctypes.c_void_p), 0
            self._keep = arr
        else:
            dt = F32 if dtype == "f32" else F64
            ptr, on_dev = ctypes.c_void_p(int(X)), 1
        d = (ctypes.c_int64 * len(dims))(*dims)
        _check(L.planc_gpu_set_tensor(self.h, ptr, dt, d, len(dims), on_dev))
        self._keep = None
        self.dims = tuple(int(x) for x in dims)

    def set_factors(self, F, lam=None):
        self.tree_epoch += 1
        F = [_c64(f) for f in F]
        k = F[0].shape[1]
        lamp = _pd(_c64(lam)) if lam is not None else None
        if lam is not None:
            lam_arr = _c64(lam)
            lamp = _pd(lam_arr)
        _check(load().planc_gpu_set_factors(self.h, _fptrs(F), lamp, k))
        self.k = k

    def run(self, algo, iters, dimtree=True, compute_error=True):
        self.tree_epoch += 1
        errs = np.zeros(max(iters, 1))
        _check(load().planc_gpu_run(self.h, ALGO[algo] if isinstance(algo, str) else int(algo),
                                    iters, int(dimtree), int(compute_error), _pd(errs)))
        return errs[:iters]

    def get_factors(self):
        F = [np.zeros((d, self.k)) for d in self.dims]
        lam = np.zeros(self.k)
        _check(load().planc_gpu_get_factors(self.h, _fptrs(F), _pd(lam)))
        return F, lam

    # ---- shared-memory NMF of a matrix A ~ W H^T (set_tensor(A) with a 2-D
    # Fortran-order array; W: (m, k), H: (n, k))
    def nmf_set_factors(self, W, H):
        W, H = _c64(W), _c64(H)
        _check(load().planc_gpu_nmf_set_factors(self.h, _pd(W), _pd(H), W.shape[1]))
        self.k = W.shape[1]

    def nmf_set_regularization(self, regW=(0.0, 0.0), regH=(0.0, 0.0), symm_reg=0.0):
        rw, rh = _c64(np.asarray(regW, dtype=np.float64)), _c64(np.asarray(regH, dtype=np.float64))
        _check(load().planc_gpu_nmf_set_regularization(self.h, _pd(rw), _pd(rh), float(symm_reg)))

    def nmf_run(self, algo, iters):
        """Returns (objective, relative error) per iteration."""
        self.tree_epoch += 1
        obj, rel = np.zeros(max(iters, 1)), np.zeros(max(iters, 1))
        _check(load().planc_gpu_nmf_run(self.h, ALGO[algo] if isinstance(algo, str) else int(algo),
                                        iters, _pd(obj), _pd(rel)))
        return obj[:iters], rel[:iters]

    def nmf_get_factors(self):
        W, H = np.zeros((self.dims[0], self.k)), np.zeros((self.dims[1], self.k))
        _check(load().planc_gpu_nmf_get_factors(self.h, _pd(W), _pd(H)))
        return W, H

    def mttkrp(self, mode, dimtree=True):
        self.tree_epoch += 1
        out = np.zeros((self.dims[mode], self.k))
        _check(load().planc_gpu_mttkrp(self.h, mode, int(dimtree), _pd(out)))
        return out

    def gram_loo(self, mode):
        out = np.zeros((self.k, self.k))
        _check(load().planc_gpu_gram_loo(self.h, mode, _pd(out)))
        return out

    def objective_error(self):
        self.tree_epoch += 1
        e = ctypes.c_double()
        _check(load().planc_gpu_objective_error(self.h, ctypes.byref(e)))
        return e.value

    def mode_begin(self, mode, dimtree=True):
        self.tree_epoch += 1
        G = np.zeros((self.k, self.k))
        M = np.zeros((self.dims[mode], self.k))
        _check(load().planc_gpu_mode_begin(self.h, mode, int(dimtree), _pd(G), _pd(M)))
        return G, M

    def mode_end(self, mode, factor):
        self.tree_epoch += 1
        f = _c64(factor)
        _check(load().planc_gpu_mode_end(self.h, mode, _pd(f)))

    def bpp_solve(self, AtA, AtB):
        """AtA n x n, AtB n x ncols -> (X n x ncols, passive n x ncols, iters)."""
        AtA = _c64(AtA)
        n, ncols = AtB.shape
        B = np.ascontiguousarray(np.asarray(AtB, dtype=np.float64).T)  # column-major n x ncols
        X = np.zeros((ncols, n))
        P = np.zeros((ncols, n), dtype=np.int32)
        it = np.zeros(ncols, dtype=np.int32)
        _check(load().planc_gpu_bpp_solve(
            self.h, _pd(AtA), _pd(B), n, ncols, _pd(X),
            P.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)),
            it.ctypes.data_as(ctypes.POINTER(ctypes.c_int32))))
        return X.T.copy(), P.T.copy(), it

    def mttkrp_device(self, mode, factor_ptrs, out_ptr, dimtree=True, reuse=False):
        """MTTKRP of `mode` for device factors (pointers to row-major (I_n, k)
        float64 buffers) into the device buffer out_ptr; stream-ordered."""
        arr = (ctypes.c_void_p * len(factor_ptrs))(*[int(p) for p in factor_ptrs])
        self.tree_epoch += 1
        _check(load().planc_gpu_mttkrp_device(self.h, mode, arr, ctypes.c_void_p(int(out_ptr)),
                                              int(dimtree) | (2 if reuse else 0)))

    # ---- device building blocks of the distributed iteration (device
    # pointers, row-major rows x k FP64 blocks; ordered on the context's stream)
    def update_device(self, algo, H_ptr, M_ptr, G_ptr, rows, k):
        _check(load().planc_gpu_update_device(self.h, ALGO[algo] if isinstance(algo, str) else int(algo),
                                              ctypes.c_void_p(int(H_ptr)), ctypes.c_void_p(int(M_ptr)),
                                              ctypes.c_void_p(int(G_ptr)), int(rows), int(k)))

    def gram_device(self, F_ptr, rows, k, G_ptr):
        _check(load().planc_gpu_gram_device(self.h, ctypes.c_void_p(int(F_ptr)), int(rows), int(k),
                                            ctypes.c_void_p(int(G_ptr))))

    def normalize_device(self, F_ptr, rows, k, Gin_ptr, lam_ptr, Gout_ptr):
        _check(load().planc_gpu_normalize_device(self.h, ctypes.c_void_p(int(F_ptr) if F_ptr else None),
                                                 int(rows), int(k), ctypes.c_void_p(int(Gin_ptr)),
                                                 ctypes.c_void_p(int(lam_ptr)),
                                                 ctypes.c_void_p(int(Gout_ptr))))

    def coldot_device(self, A_ptr, B_ptr, rows, k, out_ptr):
        _check(load().planc_gpu_coldot_device(self.h, ctypes.c_void_p(int(A_ptr) if A_ptr else None),
                                              ctypes.c_void_p(int(B_ptr) if B_ptr else None),
                                              int(rows), int(k), ctypes.c_void_p(int(out_ptr))))

    def sync(self):
        _check(load().planc_gpu_sync(self.h))

    # ---- differentiable CP loss on device factors (pointers)
    def cp_loss_device(self, F_ptrs, M0_ptr, G_ptr, loss_ptr):
        _check(load().planc_gpu_cp_loss_device(self.h, _vps(F_ptrs), ctypes.c_void_p(int(M0_ptr)),
                                               ctypes.c_void_p(int(G_ptr)),
                                               ctypes.c_void_p(int(loss_ptr))))

    def cp_grads_device(self, F_ptrs, G_ptr, M_ptrs, g_ptr, grad_ptrs):
        _check(load().planc_gpu_cp_grads_device(self.h, _vps(F_ptrs), ctypes.c_void_p(int(G_ptr)),
                                                _vps(M_ptrs), ctypes.c_void_p(int(g_ptr)),
                                                _vps(grad_ptrs)))

    def cp_step_device(self, Y_ptrs, grad_ptrs, Fprev_ptrs, eta, mom, Fnew_ptrs, Ynew_ptrs):
        _check(load().planc_gpu_cp_step_device(self.h, _vps(Y_ptrs), _vps(grad_ptrs), _vps(Fprev_ptrs),
                                               float(eta), float(mom), _vps(Fnew_ptrs),
                                               _vps(Ynew_ptrs)))

    def tensor_norm2(self):
        v = ctypes.c_double()
        _check(load().planc_gpu_tensor_norm2(self.h, ctypes.byref(v)))
        return v.value

    def set_bpp_max_iter(self, n):
        _check(load().planc_gpu_set_bpp_max_iter(self.h, int(n)))

    def set_bpp_warm_start(self, on):
        _check(load().planc_gpu_set_bpp_warm_start(self.h, int(bool(on))))

    def reset_update_state(self):
        """Fresh AO-ADMM / Nesterov solver state (as a new solver object)."""
        _check(load().planc_gpu_reset_update_state(self.h))

    def set_timing(self, on):
        _check(load().planc_gpu_set_timing(self.h, int(on)))

    def kernel_times(self):
        ms = np.zeros(len(KERNEL_CLASSES))
        n = np.zeros(len(KERNEL_CLASSES), dtype=np.int64)
        _check(load().planc_gpu_get_kernel_times(self.h, _pd(ms),
                                                 n.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)),
                                                 len(KERNEL_CLASSES)))
        return {c: (float(ms[i]), int(n[i])) for i, c in enumerate(KERNEL_CLASSES)}

    def launch_count(self):
        return int(load().planc_gpu_launch_count(self.h))


class Batch:
    """Many independent tensors factorised together (planc_gpu_batch)."""

    def __init__(self, device=0, precision="fp64", nstreams=16):
        h = ctypes.c_void_p()
        _check(load().planc_gpu_batch_create(ctypes.byref(h), device, PREC[precision], nstreams))
        self.h = h
        self.members = []  # (dims, k)

    def add(self, X, F, dims=None, dtype=None):
        F = [_c64(f) for f in F]
        k = F[0].shape[1]
        if isinstance(X, np.ndarray):
            dims = X.shape
            arr = np.asfortranarray(X) if X.dtype == np.float32 else np.asfortranarray(X, dtype=np.float64)
            dt, ptr, on_dev = (F32 if arr.dtype == np.float32 else F64), arr.ctypes.data_as(ctypes.c_void_p), 0
        else:
            dt, ptr, on_dev = (F32 if dtype == "f32" else F64), ctypes.c_void_p(int(X)), 1
        d = (ctypes.c_int64 * len(dims))(*dims)
        idx = ctypes.c_int()
        _check(load().planc_gpu_batch_add(self.h, ptr, dt, d, len(dims), on_dev, _fptrs(F), k,
                                          ctypes.byref(idx)))
        self.members.append((tuple(int(x) for x in dims), k))
        return idx.value

    def set_factors(self, index, F):
        F = [_c64(f) for f in F]
        _check(load().planc_gpu_batch_set_factors(self.h, index, _fptrs(F), F[0].shape[1]))

    def run(self, algo, iters, compute_error=True):
        errs = np.zeros((len(self.members), max(iters, 1)))
        _check(load().planc_gpu_batch_run(self.h, ALGO[algo], iters, int(compute_error), _pd(errs)))
        return errs[:, :iters]

    def get_factors(self, index):
        dims, k = self.members[index]
        F = [np.zeros((d, k)) for d in dims]
        lam = np.zeros(k)
        _check(load().planc_gpu_batch_get_factors(self.h, index, _fptrs(F), _pd(lam)))
        return F, lam

    def autotune(self, algo, trials=3):
        ms = ctypes.c_double()
        _check(load().planc_gpu_batch_autotune(self.h, ALGO[algo], trials, ctypes.byref(ms)))
        return ms.value

    def close(self):
        if self.h:
            load().planc_gpu_batch_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


def selftest_wait_timeout(device=0, seconds=0.05):
    """Runs the bounded-wait self-test; returns the status the kernel wrote."""
    st = ctypes.c_int32()
    _check(load().planc_gpu_selftest_wait_timeout(device, float(seconds), ctypes.byref(st)))
    return st.value


def selftest_coop_timeout(device=0):
    """Runs the cooperative NMF sweep's bounded wait with one CTA that never
    reports; returns the device status (-6, PLANC_GPU_ERR_TIMEOUT, expected)."""
    st = ctypes.c_int32(0)
    _check(load().planc_gpu_selftest_coop_timeout(device, ctypes.byref(st)))
    return st.value


def synth_cp_tensor(device, x_dev_ptr, dtype, dims, A, sigma, seed, clip=True, stream=None):
    """Fill device memory with a CP model + Gaussian noise (see planc_gpu.h)."""
    A = [_c64(a) for a in A]
    d = (ctypes.c_int64 * len(dims))(*dims)
    _check(load().planc_gpu_synth_cp_tensor(device, ctypes.c_void_p(int(x_dev_ptr)),
                                            F32 if dtype == "f32" else F64, d, len(dims),
                                            _fptrs(A), A[0].shape[1], float(sigma), int(seed),
                                            int(clip), stream))
