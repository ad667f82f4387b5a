"""ctypes binding of the CPU oracle (test infrastructure only).

Only tests/, ``__graft_entry__.smoke()`` and the CPU-baseline legs of
``bench.py`` import this package; the product path never does.

Two libraries are loaded:
  * ``liboracle.so``: the CPU restatement of the reference NTF path
    (``ntf_oracle.cpp``; every function cites the reference lines it follows);
  * ``_ref/libref_planc.so``: the reference's own shared-memory NTF code
    (``AUNTF`` and its updates, ``BPPNNLS``, ``NCPFactors``, ``Tensor``,
    ``DenseDimensionTree``) compiled unmodified by ``oracle/Makefile`` against
    the Armadillo-subset shim in ``ref_shim/``, driven by
    ``ref_planc_driver.cpp``.

Array conventions: tensors are numpy arrays in Fortran order (mode 0
fastest, ``common/tensor.hpp:22-28``); factors are C-order ``(I_n, k)``
float64 arrays (row-major, the layout of ``ncp_mttkrp_t`` and the dimension
tree's factors).
"""
import ctypes
import glob
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ALGO = {"mu": 0, "hals": 1, "anlsbpp": 2, "aoadmm": 4, "nesterov": 5}

_lib = None
_ref = None


def find_openblas():
    """Locate an LP64 OpenBLAS (with LAPACK) shipped inside the Python env."""
    import numpy  # noqa: F401  (only to find site-packages)
    site = os.path.dirname(os.path.dirname(np.__file__))
    cands = sorted(glob.glob(os.path.join(site, "opencv_python_headless.libs", "libopenblas*.so*")))
    if not cands:
        raise RuntimeError("no LP64 OpenBLAS found for the CPU oracle")
    return cands[0]


def build(reference_dir=None):
    """Compile liboracle.so (and _ref/libref_planc.so when the reference
    tree is present)."""
    cmd = ["make", "-s", "-C", HERE, "OPENBLAS=" + find_openblas()]
    if reference_dir and os.path.isdir(reference_dir):
        cmd.append("REFERENCE_DIR=" + reference_dir)
    subprocess.run(cmd, check=True)


def lib():
    global _lib
    if _lib is None:
        path = os.path.join(HERE, "liboracle.so")
        if not os.path.exists(path):
            build()
        L = ctypes.CDLL(path)
        P = ctypes.POINTER
        d, i64, i32 = ctypes.c_double, ctypes.c_int64, ctypes.c_int
        pd, pi64, pi = P(d), P(i64), P(i32)
        ppd = P(pd)
        L.orc_gram_loo.argtypes = [ppd, pi64, i32, i32, i32, pd]
        L.orc_krp_leave_out_one.argtypes = [ppd, pi64, i32, i32, i32, pd]
        L.orc_mttkrp_direct.argtypes = [pd, pi64, i32, ppd, i32, i32, pd]
        L.orc_mttkrp_dimtree_all.argtypes = [pd, pi64, i32, ppd, i32, ppd]
        L.orc_mttkrp_dimtree_all.restype = i32
        L.orc_normalize.argtypes = [pd, i64, i32, pd]
        L.orc_hals_update.argtypes = [pd, i64, i32, pd, pd]
        L.orc_mu_update.argtypes = [pd, i64, i32, pd, pd]
        L.orc_bpp_update.argtypes = [pd, i64, i32, pd, pd, pi]
        L.orc_bpp_update.restype = i32
        L.orc_bpp_solve.argtypes = [pd, pd, i32, i64, pd, pi]
        L.orc_bpp_solve.restype = i32
        L.orc_explicit_error.argtypes = [pd, pi64, i32, ppd, pd, i32]
        L.orc_explicit_error.restype = d
        L.orc_ntf_run.argtypes = [pd, pi64, i32, i32, ppd, pd, i32, i32, i32, i32, pd]
        L.orc_ntf_run.restype = i32
        L.orc_tensor_randu.argtypes = [i64, ctypes.c_uint, pd]
        L.orc_synth_cp.argtypes = [pi64, i32, ppd, i32, d, ctypes.c_uint64, i32, i32, pd]
        L.orc_admm_update.argtypes = [pd, pd, i64, i32, pd, pd, i32, d]
        L.orc_admm_update.restype = i32
        L.orc_nes_update.argtypes = [pd, pd, i64, i32, pd, pd, d, d, i32]
        L.orc_nes_update.restype = i32
        L.orc_sym_eig_minmax.argtypes = [pd, i32, pd, pd]
        L.orc_nmf_run.argtypes = [pd, i64, i64, i32, pd, pd, i32, i32, pd, pd, pd]
        L.orc_nmf_run.restype = i32
        _lib = L
    return _lib


REF_LIB = os.path.join(HERE, "_ref", "libref_planc.so")


def ref_available():
    """True when the reference's own code (oracle/_ref/libref_planc.so, built
    from the reference tree by oracle/Makefile) is present."""
    return os.path.exists(REF_LIB)


def ref():
    """ctypes handle of oracle/_ref/libref_planc.so: the reference's AUNTF,
    its updates, BPPNNLS, NCPFactors, Tensor and DenseDimensionTree compiled
    unmodified against the Armadillo-subset shim (ref_planc_driver.cpp)."""
    global _ref
    if _ref is None:
        R = ctypes.CDLL(REF_LIB)
        P = ctypes.POINTER
        d, vp, i32, li = ctypes.c_double, ctypes.c_void_p, ctypes.c_int, ctypes.c_long
        pd = P(d)
        ppd = P(pd)
        R.ref_tensor_new.argtypes = [P(li), i32, i32]
        R.ref_tensor_new.restype = vp
        R.ref_tensor_from.argtypes = [P(li), i32, pd]
        R.ref_tensor_from.restype = vp
        R.ref_tensor_data.argtypes = [vp]
        R.ref_tensor_data.restype = pd
        R.ref_tensor_norm.argtypes = [vp]
        R.ref_tensor_norm.restype = d
        R.ref_tensor_free.argtypes = [vp]
        R.ref_tensor_mttkrp.argtypes = [vp, ppd, i32, i32, pd]
        R.ref_gram_leave_out_one.argtypes = [P(li), i32, i32, ppd, i32, pd]
        R.ref_normalize_mode.argtypes = [pd, li, i32, pd]
        R.ref_update.argtypes = [i32, pd, pd, pd, li, i32, pd]
        R.ref_update.restype = i32
        R.ref_bpp_solve.argtypes = [pd, pd, i32, li, pd]
        R.ref_bpp_solve.restype = i32
        R.ref_ntf_create.argtypes = [vp, i32, i32, i32, ppd, i32, i32]
        R.ref_ntf_create.restype = vp
        R.ref_ntf_run.argtypes = [vp, i32]
        R.ref_ntf_run.restype = d
        R.ref_ntf_factors.argtypes = [vp, ppd, pd]
        R.ref_ntf_objective_error.argtypes = [vp]
        R.ref_ntf_objective_error.restype = d
        R.ref_ntf_destroy.argtypes = [vp]
        R.ref_dimtree_create.argtypes = [pd, P(li), i32, i32, ppd]
        R.ref_dimtree_create.restype = vp
        R.ref_dimtree_set_factor.argtypes = [vp, li, pd]
        R.ref_dimtree_mttkrp.argtypes = [vp, li, pd]
        R.ref_dimtree_destroy.argtypes = [vp]
        _ref = R
    return _ref


def _ldims(shape):
    return (ctypes.c_long * len(shape))(*shape)


class RefTensor:
    """planc::Tensor of the reference (common/tensor.hpp), owning its data."""

    def __init__(self, X=None, dims=None, serial=True):
        """From an array X (copied, Tensor(dims, data)), or Tensor(dims) with
        the reference's mt19937(103) fill (one OpenMP thread when serial)."""
        R = ref()
        if X is not None:
            X = _xf(X)
            self.dims = tuple(X.shape)
            self.h = R.ref_tensor_from(_ldims(X.shape), X.ndim, _pd(X))
        else:
            self.dims = tuple(int(x) for x in dims)
            self.h = R.ref_tensor_new(_ldims(self.dims), len(self.dims), int(serial))

    def data(self):
        """The tensor's m_data as a Fortran-order view (no copy)."""
        n = int(np.prod(self.dims))
        p = ref().ref_tensor_data(self.h)
        return np.ctypeslib.as_array(p, shape=(n,)).reshape(self.dims, order="F")

    def norm(self):
        """Tensor::norm(): the squared Frobenius norm (common/tensor.hpp:350-356)."""
        return ref().ref_tensor_norm(self.h)

    def mttkrp(self, F, n):
        """Tensor::mttkrp(n, krp_leave_out_one(n)) as row-major I_n x k."""
        F = [_c(f) for f in F]
        out = np.zeros((self.dims[n], F[0].shape[1]))
        ref().ref_tensor_mttkrp(self.h, _fptrs(F), F[0].shape[1], n, _pd(out))
        return out

    def close(self):
        if self.h:
            ref().ref_tensor_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class RefNTF:
    """The reference's AUNTF subclass for `algo` on a RefTensor, driven as a
    library user drives it: dim_tree() before reset(initial factors),
    compute_error(), then computeNTF() for a number of iterations."""

    def __init__(self, tensor, F0, algo, dimtree=True, compute_error=True, serial_setup=True):
        F0 = [_c(f) for f in F0]
        self.tensor = tensor
        self.k = F0[0].shape[1]
        self.h = ref().ref_ntf_create(tensor.h, self.k, ALGO[algo], int(dimtree), _fptrs(F0),
                                      int(compute_error), int(serial_setup))
        if not self.h:
            raise ValueError("unknown algorithm")

    def run(self, iters):
        """computeNTF() with num_it(iters); returns current_error()."""
        return ref().ref_ntf_run(self.h, iters)

    def factors(self):
        F = [np.zeros((d, self.k)) for d in self.tensor.dims]
        lam = np.zeros(self.k)
        ref().ref_ntf_factors(self.h, _fptrs(F), _pd(lam))
        return F, lam

    def objective_error(self):
        return ref().ref_ntf_objective_error(self.h)

    def close(self):
        if self.h:
            ref().ref_ntf_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def ref_ntf_run(X, F0, algo, iters, dimtree=True, compute_error=True):
    """The reference's own AUNTF run from injected factors. Returns (factors,
    lambda, per-iteration relative errors). Nesterov runs its iterations in
    one computeNTF() call (its acceleration counts iterations within a call)
    and reports the final error only; the other updates run one iteration per
    call so that every iteration's error is seen (the loop state carries over
    between calls)."""
    t = RefTensor(X)
    s = RefNTF(t, F0, algo, dimtree, compute_error)
    try:
        if algo == "nesterov":
            errs = np.array([s.run(iters)])
        else:
            errs = np.array([s.run(1) for _ in range(iters)])
        F, lam = s.factors()
    finally:
        s.close()
        t.close()
    return F, lam, errs


def ref_update(algo, H, M, G):
    """update(mode) of the reference's NTF class for `algo` with the given
    factor H (I x k), MTTKRP M (I x k) and leave-one-out Gram G; returns the
    new factor (I x k)."""
    H, M, G = _c(H), _c(M), _c(G)
    out = np.zeros_like(H)
    rc = ref().ref_update(ALGO[algo], _pd(H), _pd(M), _pd(G), H.shape[0], H.shape[1], _pd(out))
    if rc != 0:
        raise ValueError("unsupported algorithm for an isolated update")
    return out


def ref_bpp_solve(AtA, AtB):
    """BPPNNLS(AtA, AtB, true).solveNNLS(); returns (X, iterations)."""
    A = np.asfortranarray(AtA, dtype=np.float64)
    B = np.asfortranarray(AtB, dtype=np.float64)
    X = np.zeros(B.shape, order="F")
    it = ref().ref_bpp_solve(_pd(A), _pd(B), A.shape[0], B.shape[1], _pd(X))
    return X, it


def ref_normalize(H):
    """NCPFactors::normalize(mode) of H; returns (normalised H, lambda)."""
    H = _c(H).copy()
    lam = np.zeros(H.shape[1])
    ref().ref_normalize_mode(_pd(H), H.shape[0], H.shape[1], _pd(lam))
    return H, lam


def ref_gram_loo(F, n):
    """NCPFactors::gram_leave_out_one(n)."""
    F = [_c(f) for f in F]
    k = F[0].shape[1]
    G = np.zeros((k, k))
    ref().ref_gram_leave_out_one(_ldims([f.shape[0] for f in F]), len(F), k, _fptrs(F), n,
                                 _pd(G))
    return G.T.copy()


def _c(a):
    return np.ascontiguousarray(a, dtype=np.float64)


# ---------------------------------------------------------------- helpers
def _pd(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _dims(X):
    return (ctypes.c_int64 * X.ndim)(*X.shape)


def _fptrs(F):
    arr = (ctypes.POINTER(ctypes.c_double) * len(F))()
    for i, f in enumerate(F):
        assert f.dtype == np.float64 and f.flags.c_contiguous
        arr[i] = _pd(f)
    return arr


def _xf(X):
    X = np.asarray(X, dtype=np.float64)
    return np.asfortranarray(X)


def tensor_randu(dims, seed=103):
    """Tensor(dims) fill: std::mt19937(seed) + uniform_real_distribution<>(0,1)
    in linear order (common/tensor.hpp:86-93, 219-235, single-threaded)."""
    n = int(np.prod(dims))
    flat = np.empty(n, dtype=np.float64)
    lib().orc_tensor_randu(n, seed, _pd(flat))
    return flat.reshape(tuple(dims), order="F")


def synth_cp(dims, A, sigma, seed, clip=True, round_f32=False, out=None):
    """Synthetic CP tensor [[A]] + sigma N(0,1) (clipped at 0) on the host,
    the same function of (factors, sigma, seed) as the library's device
    generator; round_f32 rounds every value to FP32 (the device generator's
    FP32 output), stored as float64. `out`: a ctypes double pointer or a
    float64 array of numel elements to fill; returns the Fortran-order array
    when out is None."""
    A = [_c(a) for a in A]
    d = (ctypes.c_int64 * len(dims))(*dims)
    X = None
    if out is None:
        X = np.empty(int(np.prod(dims)), dtype=np.float64)
        out = X
    p = _pd(out) if isinstance(out, np.ndarray) else out
    lib().orc_synth_cp(d, len(dims), _fptrs(A), A[0].shape[1], float(sigma), int(seed),
                       int(clip), int(round_f32), p)
    return None if X is None else X.reshape(tuple(dims), order="F")


def gram_loo(F, n):
    k = F[0].shape[1]
    G = np.zeros((k, k))
    dims = (ctypes.c_int64 * len(F))(*[f.shape[0] for f in F])
    lib().orc_gram_loo(_fptrs(F), dims, len(F), k, n, _pd(G))
    return G


def mttkrp_direct(X, F, n):
    X = _xf(X)
    k = F[0].shape[1]
    out = np.zeros((X.shape[n], k))
    lib().orc_mttkrp_direct(_pd(X), _dims(X), X.ndim, _fptrs(F), k, n, _pd(out))
    return out


def mttkrp_dimtree_all(X, F):
    X = _xf(X)
    k = F[0].shape[1]
    outs = [np.zeros((X.shape[n], k)) for n in range(X.ndim)]
    rc = lib().orc_mttkrp_dimtree_all(_pd(X), _dims(X), X.ndim, _fptrs(F), k, _fptrs(outs))
    if rc != 0:
        raise ValueError("dimension tree needs N in {3,4}")
    return outs


def ref_mttkrp_dimtree_all(X, F):
    """All-mode MTTKRP through the reference's DenseDimensionTree, with fixed
    factors (the factor slot overwritten by each MTTKRP is restored as AUNTF's
    set_factor would, ntf/auntf.hpp:70-73)."""
    X = _xf(X)
    k = F[0].shape[1]
    R = ref()
    dims = (ctypes.c_long * X.ndim)(*X.shape)
    h = R.ref_dimtree_create(_pd(X), dims, X.ndim, k, _fptrs(F))
    outs = []
    try:
        for n in range(X.ndim):
            o = np.zeros((X.shape[n], k))
            R.ref_dimtree_mttkrp(h, n, _pd(o))
            R.ref_dimtree_set_factor(h, n, _pd(F[n]))
            outs.append(o)
    finally:
        R.ref_dimtree_destroy(h)
    return outs


def normalize(F):
    F = np.ascontiguousarray(F, dtype=np.float64).copy()
    lam = np.zeros(F.shape[1])
    lib().orc_normalize(_pd(F), F.shape[0], F.shape[1], _pd(lam))
    return F, lam


def hals_update(H, M, G):
    H = np.ascontiguousarray(H, dtype=np.float64).copy()
    M = np.ascontiguousarray(M, dtype=np.float64)
    G = np.ascontiguousarray(G, dtype=np.float64)
    lib().orc_hals_update(_pd(H), H.shape[0], H.shape[1], _pd(M), _pd(G))
    return H


def mu_update(H, M, G):
    H = np.ascontiguousarray(H, dtype=np.float64).copy()
    M = np.ascontiguousarray(M, dtype=np.float64)
    G = np.ascontiguousarray(G, dtype=np.float64)
    lib().orc_mu_update(_pd(H), H.shape[0], H.shape[1], _pd(M), _pd(G))
    return H


def bpp_update(M, G):
    """Returns (H row-major I x k, passive mask I x k, iterations)."""
    M = np.ascontiguousarray(M, dtype=np.float64)
    G = np.ascontiguousarray(G, dtype=np.float64)
    I, k = M.shape
    H = np.zeros((I, k))
    mask = np.zeros((I, k), dtype=np.int32)
    it = lib().orc_bpp_update(_pd(H), I, k, _pd(M), _pd(G),
                              mask.ctypes.data_as(ctypes.POINTER(ctypes.c_int)))
    return H, mask, it


def admm_update(H, U, M, G, admm_iter=5, tol=0.01):
    """One AO-ADMM mode update (ntf/ntfaoadmm.hpp:23-77). Returns
    (H_new unnormalised, U_new column-normalised, iterations)."""
    H = np.ascontiguousarray(H, dtype=np.float64).copy()
    U = np.ascontiguousarray(U, dtype=np.float64).copy()
    M = np.ascontiguousarray(M, dtype=np.float64)
    G = np.ascontiguousarray(G, dtype=np.float64)
    it = lib().orc_admm_update(_pd(H), _pd(U), H.shape[0], H.shape[1], _pd(M), _pd(G),
                               int(admm_iter), float(tol))
    if it < 0:
        raise RuntimeError("chol() failed")
    return H, U, it


def nes_update(H0, M, G, delta1=1e-2, delta2=1e-2, max_inner=20000):
    """One Nesterov mode update from the proximal point H0
    (ntf/ntfnes.hpp:100-151). Returns (H_new unnormalised, inner steps)."""
    H0 = np.ascontiguousarray(H0, dtype=np.float64)
    M = np.ascontiguousarray(M, dtype=np.float64)
    G = np.ascontiguousarray(G, dtype=np.float64)
    H = np.zeros_like(H0)
    it = lib().orc_nes_update(_pd(H0), _pd(H), H0.shape[0], H0.shape[1], _pd(M), _pd(G),
                              float(delta1), float(delta2), int(max_inner))
    if it < 0:
        raise RuntimeError("inner step cap reached")
    return H, it


def sym_eig_minmax(G):
    G = np.ascontiguousarray(G, dtype=np.float64)
    lo, hi = ctypes.c_double(), ctypes.c_double()
    lib().orc_sym_eig_minmax(_pd(G), G.shape[0], ctypes.byref(lo), ctypes.byref(hi))
    return lo.value, hi.value


def explicit_error(X, F, lam):
    X = _xf(X)
    return lib().orc_explicit_error(_pd(X), _dims(X), X.ndim, _fptrs(F),
                                    _pd(np.ascontiguousarray(lam, dtype=np.float64)), F[0].shape[1])


def ntf_run(X, F_init, algo, iters, dimtree=True, compute_error=True, lam=None):
    """The AUNTF loop (ntf/auntf.hpp:128-177) from injected initial factors.
    Returns (factors, lambda, errors)."""
    X = _xf(X)
    k = F_init[0].shape[1]
    F = [np.ascontiguousarray(f, dtype=np.float64).copy() for f in F_init]
    lam = np.ones(k) if lam is None else np.asarray(lam, dtype=np.float64).copy()
    errs = np.zeros(max(iters, 1))
    rc = lib().orc_ntf_run(_pd(X), _dims(X), X.ndim, k, _fptrs(F), _pd(lam),
                           ALGO[algo] if isinstance(algo, str) else int(algo),
                           iters, int(dimtree), int(compute_error), _pd(errs))
    if rc != 0:
        raise RuntimeError("oracle ntf_run failed with code %d" % rc)
    return F, lam, errs[:iters]


def nmf_run(A, W0, H0, algo, iters, reg=None):
    """Shared-memory NMF A ~ W H^T (nmf/hals.hpp, nmf/mu.hpp, nmf/bppnmf.hpp)
    from W0 (m x k) and H0 (n x k). reg = (regW L2, regW L1, regH L2, regH L1,
    symm_reg) or None. Returns (W, H, objective per iteration, relative error
    per iteration)."""
    A = np.asfortranarray(np.asarray(A, dtype=np.float64))
    m, n = A.shape
    W = np.ascontiguousarray(W0, dtype=np.float64).copy()
    H = np.ascontiguousarray(H0, dtype=np.float64).copy()
    k = W.shape[1]
    obj = np.zeros(max(iters, 1))
    rel = np.zeros(max(iters, 1))
    r = None if reg is None else np.ascontiguousarray(reg, dtype=np.float64)
    rc = lib().orc_nmf_run(_pd(A), m, n, k, _pd(W), _pd(H),
                           ALGO[algo] if isinstance(algo, str) else int(algo), iters,
                           _pd(r) if r is not None else None, _pd(obj), _pd(rel))
    if rc != 0:
        raise RuntimeError("oracle nmf_run failed with code %d" % rc)
    return W, H, obj[:iters], rel[:iters]
