"""CPU tests of the oracle: pinned against the reference's own compiled
dimension-tree kernels (golden fixtures, and live when oracle/_ref is built),
an independent mt19937 computation, and known-answer identities."""
import itertools
import os

import numpy as np
import pytest

from helpers import cp_tensor, einsum_mttkrp, init_factors, rel

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def test_tensor_randu_matches_mt19937_pin(oracle_lib):
    # Tensor(dims) data (common/tensor.hpp:86-93, 219-235) vs an independent
    # numpy computation of std::mt19937(103) + uniform_real_distribution.
    gold = np.load(os.path.join(GOLD, "mt19937_103.npz"))["values"]
    x = oracle_lib.tensor_randu((16, 16, 16), 103).ravel(order="F")
    assert np.array_equal(x, gold)


@pytest.mark.parametrize("case", ["n3", "n4", "n3b"])
def test_oracle_mttkrp_matches_reference_golden(oracle_lib, case):
    g = np.load(os.path.join(GOLD, "ref_dimtree_mttkrp.npz"))
    dims = tuple(int(d) for d in g[case + "_dims"])
    X = g[case + "_X"].reshape(dims, order="F")
    F = [g["%s_F%d" % (case, i)] for i in range(len(dims))]
    dt = oracle_lib.mttkrp_dimtree_all(X, F)
    for n in range(len(dims)):
        ref = g["%s_M%d" % (case, n)]
        assert rel(oracle_lib.mttkrp_direct(X, F, n), ref) < 1e-13
        assert rel(dt[n], ref) < 1e-13


@pytest.mark.skipif(not __import__("oracle").ref_available(), reason="reference build absent")
@pytest.mark.parametrize("dims,k", [((7, 6, 5), 4), ((4, 5, 6, 3), 5), ((3, 9, 2), 7)])
def test_oracle_mttkrp_matches_reference_live(oracle_lib, dims, k):
    X = oracle_lib.tensor_randu(dims, 103)
    F = init_factors(dims, k, seed=5)
    ref = oracle_lib.ref_mttkrp_dimtree_all(X, F)
    dt = oracle_lib.mttkrp_dimtree_all(X, F)
    for n in range(len(dims)):
        assert rel(dt[n], ref[n]) < 1e-13
        assert rel(oracle_lib.mttkrp_direct(X, F, n), ref[n]) < 1e-13


@pytest.mark.parametrize("dims", [(5, 6, 7), (3, 4, 5, 6), (2, 3, 4, 2, 3)])
def test_mttkrp_known_answer_exact_cp(oracle_lib, dims):
    # X = [[A_0..A_{N-1}]] exactly => MTTKRP_n = A_n (*_{m!=n} A_m^T A_m)
    k = 3
    A = init_factors(dims, k, seed=11)
    letters = "abcdefgh"[:len(dims)]
    X = np.asfortranarray(np.einsum(",".join(c + "z" for c in letters) + "->" + letters, *A))
    for n in range(len(dims)):
        H = np.ones((k, k))
        for m in range(len(dims)):
            if m != n:
                H *= A[m].T @ A[m]
        assert rel(oracle_lib.mttkrp_direct(X, A, n), A[n] @ H) < 1e-12
        assert rel(oracle_lib.gram_loo(A, n), H) < 1e-13


def test_krp_order_matches_einsum(oracle_lib):
    dims = (3, 4, 5)
    F = init_factors(dims, 2, seed=3)
    X = oracle_lib.tensor_randu(dims, 7)
    for n in range(3):
        assert rel(oracle_lib.mttkrp_direct(X, F, n), einsum_mttkrp(X, F, n)) < 1e-13


@pytest.mark.parametrize("algo", ["hals", "mu"])
def test_update_fixed_point_at_exact_factors(oracle_lib, algo):
    # At the exact (normalised) factors of a noise-free CP tensor, the HALS and
    # MU updates leave the factors unchanged (up to MU's 1e-6 regulariser).
    dims, k = (6, 5, 7), 3
    A = init_factors(dims, k, seed=4)
    lam = np.ones(k)
    An = []
    for a in A:
        nrm = np.linalg.norm(a, axis=0)
        An.append(a / nrm)
        lam *= nrm
    An[0] = An[0] * lam  # fold lambda into mode 0 (the updated mode)
    letters = "abc"
    X = np.asfortranarray(np.einsum("az,bz,cz->abc", *An))
    M = oracle_lib.mttkrp_direct(X, An, 0)
    G = oracle_lib.gram_loo(An, 0)
    upd = oracle_lib.hals_update(An[0], M, G) if algo == "hals" else oracle_lib.mu_update(An[0], M, G)
    assert rel(upd, An[0]) < (1e-12 if algo == "hals" else 1e-4)


def _nnls_exhaustive(AtA, b):
    """min 0.5 x'AtA x - b'x s.t. x >= 0 by enumerating passive sets."""
    n = len(b)
    best, bestx = np.inf, None
    for mask in itertools.product([0, 1], repeat=n):
        idx = [i for i in range(n) if mask[i]]
        x = np.zeros(n)
        if idx:
            x[idx] = np.linalg.solve(AtA[np.ix_(idx, idx)], b[idx])
            if (x[idx] < 0).any():
                continue
        f = 0.5 * x @ AtA @ x - b @ x
        if f < best - 1e-14:
            best, bestx = f, x
    return bestx


@pytest.mark.parametrize("n", [2, 5, 8])
def test_bpp_matches_exhaustive_active_set(oracle_lib, n):
    rng = np.random.default_rng(n)
    A = rng.random((3 * n, n))
    AtA = A.T @ A
    B = rng.standard_normal((n, 40)) * 2 + 0.3
    X, mask, it = oracle_lib.bpp_update(B.T.copy(), AtA)
    assert it >= 0
    for c in range(B.shape[1]):
        x_ex = _nnls_exhaustive(AtA, B[:, c])
        assert np.allclose(X[c], x_ex, atol=1e-10, rtol=1e-9)
        assert np.array_equal(mask[c].astype(bool), X[c] > 0)


def test_ntf_error_decreases_and_dimtree_equals_direct(oracle_lib):
    X, _ = cp_tensor((20, 18, 16), 4, noise=0.01, seed=2)
    F0 = init_factors(X.shape, 4, seed=3)
    for algo in ["hals", "mu", "anlsbpp"]:
        F, lam, e = oracle_lib.ntf_run(X, F0, algo, 8, dimtree=True)
        F2, lam2, e2 = oracle_lib.ntf_run(X, F0, algo, 8, dimtree=False)
        assert e[-1] < e[0]
        assert np.allclose(e, e2, rtol=1e-12, atol=0)
        for a, b in zip(F, F2):
            assert rel(a, b) < 1e-11


# ---- AO-ADMM and Nesterov updates (ntf/ntfaoadmm.hpp, ntf/ntfnes.hpp) ----

def _spd_problem(I, k, seed):
    rng = np.random.default_rng(seed)
    A = rng.random((3 * k, k))
    G = A.T @ A
    M = rng.random((I, k)) @ G  # right-hand sides with a mix of active and inactive bounds
    M -= 0.4 * M.mean()
    return np.ascontiguousarray(M), G


def test_oracle_sym_eig_matches_numpy(oracle_lib):
    _, G = _spd_problem(5, 12, 3)
    lo, hi = oracle_lib.sym_eig_minmax(G)
    w = np.linalg.eigvalsh(G)
    assert abs(lo - w[0]) < 1e-12 * w[-1] and abs(hi - w[-1]) < 1e-12 * w[-1]


def test_oracle_admm_reaches_nnls_optimum(oracle_lib):
    # with the iteration cap and tolerance opened up, the ADMM of
    # NTFAOADMM::update converges to the unique NNLS optimum that BPP finds
    M, G = _spd_problem(40, 8, 4)
    H0 = np.random.default_rng(5).random(M.shape)
    H, U, it = oracle_lib.admm_update(H0, np.zeros_like(H0), M, G, admm_iter=5000, tol=1e-13)
    ref, _, _ = oracle_lib.bpp_update(M, G)
    assert rel(H, ref) < 1e-8, rel(H, ref)
    # the dual variable leaves the call column-normalised (ntfaoadmm.hpp:74)
    nrm = np.linalg.norm(U, axis=0)
    assert np.allclose(nrm[nrm > 0], 1.0)


def test_oracle_admm_reference_defaults_stop_within_five(oracle_lib):
    M, G = _spd_problem(30, 6, 6)
    H0 = np.random.default_rng(7).random(M.shape)
    _, _, it = oracle_lib.admm_update(H0, np.zeros_like(H0), M, G)
    assert 1 <= it <= 5


def test_oracle_nes_reaches_proximal_nnls_optimum(oracle_lib):
    # from H0 = 0 the Nesterov inner loop minimises
    # 1/2 h^T (G + lambda I) h - m^T h over h >= 0 (ntfnes.hpp:113-145), whose
    # optimum BPP computes with AtA = G + lambda I
    M, G = _spd_problem(25, 6, 8)
    H, steps = oracle_lib.nes_update(np.zeros_like(M), M, G, delta1=1e-13, delta2=1e-13)
    w = np.linalg.eigvalsh(G)
    L, mu = w[-1], w[0]
    q = L / mu
    lam = 10 * mu if q > 1e6 else (mu if q > 1e3 else mu / 10)
    ref, _, _ = oracle_lib.bpp_update(M, G + lam * np.eye(G.shape[0]))
    assert steps > 0
    assert rel(H, ref) < 1e-6, rel(H, ref)


@pytest.mark.parametrize("algo", ["aoadmm", "nesterov"])
def test_oracle_ntf_run_new_algorithms_descend(oracle_lib, algo):
    dims, k = (14, 12, 10), 4
    X, _ = cp_tensor(dims, k, noise=0.01, seed=31)
    F0 = init_factors(dims, k, seed=32)
    F, lam, errs = oracle_lib.ntf_run(X, F0, algo, 15)
    assert np.all(np.isfinite(errs))
    assert errs[-1] < 0.7 * errs[0], errs
    # lambda and the factors describe the model whose error is reported; the
    # Nesterov acceleration that follows the last error keeps its extrapolated
    # factors only if they lower it (ntfnes.hpp:80-96)
    e = oracle_lib.explicit_error(X, F, lam)
    if algo == "nesterov":
        assert e < errs[-1] + 1e-12
    else:
        assert abs(e - errs[-1]) < 1e-12


# ---- shared-memory NMF (nmf/hals.hpp, nmf/mu.hpp, nmf/bppnmf.hpp) ----

def _nmf_problem(m, n, k, seed, noise=0.01):
    rng = np.random.default_rng(seed)
    A = rng.random((m, k)) @ rng.random((k, n))
    A = np.maximum(A + noise * A.std() * rng.standard_normal(A.shape), 0.0)
    return np.asfortranarray(A), rng.random((m, k)), rng.random((n, k))


@pytest.mark.parametrize("algo", ["hals", "mu", "anlsbpp"])
def test_oracle_nmf_error_is_the_fit(oracle_lib, algo):
    # the reported relative error is ||A - W H^T|| / ||A|| of the factors the
    # run returns (normalize_by_W rescales W and H without changing W H^T)
    A, W0, H0 = _nmf_problem(40, 30, 5, 71)
    W, H, obj, rel = oracle_lib.nmf_run(A, W0, H0, algo, 12)
    direct = np.linalg.norm(A - W @ H.T) / np.linalg.norm(A)
    assert abs(direct - rel[-1]) < 1e-10
    assert abs(obj[-1] - (rel[-1] * np.linalg.norm(A)) ** 2) < 1e-8 * obj[-1]
    assert rel[-1] < rel[0]
    # W leaves the run with unit columns
    assert np.allclose(np.linalg.norm(W, axis=0), 1.0)


def test_oracle_nmf_bpp_is_monotone_and_solves_nnls(oracle_lib):
    # ANLS: each half step is an exact NNLS solve, so the objective never
    # rises, and H is the NNLS optimum for the W it was solved with (the final
    # normalize_by_W scales W's columns by 1/s and H's by s, which maps one
    # NNLS optimum onto the other)
    from scipy.optimize import nnls
    A, W0, H0 = _nmf_problem(50, 35, 6, 72)
    W, H, obj, rel = oracle_lib.nmf_run(A, W0, H0, "anlsbpp", 10)
    assert np.all(np.diff(obj) <= 1e-9 * obj[0])
    for j in range(0, 35, 7):
        x, _ = nnls(W, A[:, j])
        assert np.allclose(x, H[j], atol=1e-8 * np.abs(H).max())


def test_oracle_nmf_regularized_objective(oracle_lib):
    # HALS normalises by W before each error, so the returned factors are the
    # ones the last objective was computed from (common/nmf.hpp:386-425)
    A, W0, H0 = _nmf_problem(30, 30, 4, 73)
    w2, w1, h2, h1 = 0.5, 0.1, 0.3, 0.2
    W, H, obj, rel = oracle_lib.nmf_run(A, W0, H0, "hals", 3, reg=(w2, w1, h2, h1, 0.0))
    fit = np.linalg.norm(A - W @ H.T) ** 2
    ref = (fit + w2 * np.sum(W * W) + h2 * np.sum(H * H) + w1 * np.sum(W.sum(1) ** 2)
           + h1 * np.sum(H.sum(1) ** 2))
    assert abs(obj[-1] - ref) < 1e-9 * ref


# ---------------------------------------------------------------------------
# The update, normalisation, BPP and AUNTF-loop steps of the oracle pinned to
# the reference's OWN code (ntf/auntf.hpp, ntf/ntf*.hpp, nnls/bppnnls.hpp,
# common/ncpfactors.hpp compiled unmodified against the Armadillo-subset shim
# in oracle/ref_shim/): committed fixtures made by tests/golden/make_golden.py,
# and the live library when oracle/_ref is built.

def _golden_runs():
    import importlib.util
    spec = importlib.util.spec_from_file_location("make_golden", os.path.join(GOLD, "make_golden.py"))
    mg = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mg)
    return mg


_MG = _golden_runs()
_RUN_CASES = [(name, a) for name, _, _, _, _, algos, _, _ in _MG.RUNS for a in algos]


@pytest.mark.parametrize("name,algo", _RUN_CASES)
def test_oracle_ntf_runs_match_reference_golden(oracle_lib, name, algo):
    g = np.load(os.path.join(GOLD, "ref_ntf_runs.npz"))
    dims = tuple(int(d) for d in g[name + "_dims"])
    k, iters, dt, seed = (int(v) for v in g[name + "_meta"])
    X, F0 = _MG.run_inputs(dims, k, float(g[name + "_noise"][0]), seed)
    xs = g[name + "_xsum"]
    assert abs(X.sum() - xs[0]) <= 1e-12 * xs[0] and X.ravel(order="F")[7] == xs[2]
    F, lam, errs = oracle_lib.ntf_run(X, F0, algo, iters, dimtree=bool(dt))
    pre = "%s_%s_" % (name, algo)
    for i in range(len(dims)):
        assert rel(F[i], g[pre + "F%d" % i]) < 1e-10, i
    assert rel(lam, g[pre + "lam"]) < 1e-10
    ref_err = g[pre + "err"]
    if algo == "nesterov":  # the reference run reports its final error only
        assert abs(errs[-1] - ref_err[-1]) <= 1e-10 * ref_err[-1]
    else:
        assert np.max(np.abs(errs - ref_err) / ref_err) < 1e-10


@pytest.mark.parametrize("case", [0, 1, 2])
def test_oracle_updates_match_reference_golden(oracle_lib, case):
    g = np.load(os.path.join(GOLD, "ref_updates.npz"))
    H, M, G = g["u%d_H" % case], g["u%d_M" % case], g["u%d_G" % case]
    assert rel(oracle_lib.hals_update(H, M, G), g["u%d_hals" % case]) < 1e-13
    assert rel(oracle_lib.mu_update(H, M, G), g["u%d_mu" % case]) < 1e-13
    Hb, mask, _ = oracle_lib.bpp_update(M, G)
    ref_b = g["u%d_anlsbpp" % case]
    assert rel(Hb, ref_b) < 1e-12
    assert np.array_equal(mask != 0, ref_b > 0)
    Ha, _, _ = oracle_lib.admm_update(H, np.zeros_like(H), M, G)
    assert rel(Ha, g["u%d_aoadmm" % case]) < 1e-12


@pytest.mark.parametrize("case", [0, 1, 2])
def test_oracle_bpp_matches_reference_golden(oracle_lib, case):
    # BPPNNLS (nnls/bppnnls.hpp:67-191) on normal equations; case 2 is one
    # mode of the 192^4 rank-64 workload in size (k = 64, 192 right-hand sides)
    g = np.load(os.path.join(GOLD, "ref_updates.npz"))
    AtA, AtB, Xr = g["b%d_AtA" % case], g["b%d_AtB" % case], g["b%d_X" % case]
    H, mask, it = oracle_lib.bpp_update(AtB.T, AtA)
    assert rel(H.T, Xr) < 1e-11
    assert np.array_equal(mask.T != 0, Xr > 0)
    assert it == int(g["b%d_iters" % case][0])


_live = pytest.mark.skipif(not __import__("oracle").ref_available(), reason="reference build absent")


@_live
@pytest.mark.parametrize("algo", ["mu", "hals", "anlsbpp", "aoadmm", "nesterov"])
@pytest.mark.parametrize("dims,k,dimtree", [((11, 9, 13), 4, True), ((6, 5, 7, 4), 3, True),
                                            ((10, 8, 7), 6, False), ((5, 6, 4, 3), 2, False)])
def test_oracle_ntf_run_matches_reference_live(oracle_lib, algo, dims, k, dimtree):
    X, _ = cp_tensor(dims, k, noise=0.05, seed=sum(dims) + k)
    F0 = init_factors(dims, k, seed=k + 40)
    iters = 7
    Fr, lr, er = oracle_lib.ref_ntf_run(X, F0, algo, iters, dimtree=dimtree)
    F, lam, errs = oracle_lib.ntf_run(X, F0, algo, iters, dimtree=dimtree)
    for a, b in zip(F, Fr):
        assert rel(a, b) < 1e-10
    assert rel(lam, lr) < 1e-10
    if algo == "nesterov":
        assert abs(errs[-1] - er[-1]) <= 1e-10 * er[-1]
    else:
        assert np.max(np.abs(errs - er) / er) < 1e-10


@_live
@pytest.mark.parametrize("seed", range(6))
def test_oracle_bpp_matches_reference_live(oracle_lib, seed):
    # random normal equations, rank-deficient data, single and many columns
    rng = np.random.default_rng(900 + seed)
    n = int(rng.integers(2, 40))
    ncols = [1, 3, 17, 120, 2, 64][seed]
    B = rng.random((2 * n, n))
    B[rng.random(B.shape) < 0.4] = 0.0
    AtA = B.T @ B + 1e-6 * np.eye(n)
    AtB = rng.standard_normal((n, ncols)) * np.abs(AtA).mean() * n
    Xr, it_r = oracle_lib.ref_bpp_solve(AtA, AtB)
    H, mask, it = oracle_lib.bpp_update(AtB.T, AtA)
    assert rel(H.T, Xr) < 1e-9
    assert np.array_equal(mask.T != 0, Xr > 0)
    assert it == it_r


@_live
def test_oracle_normalize_and_gram_match_reference_live(oracle_lib):
    rng = np.random.default_rng(5)
    F = [rng.random((d, 6)) for d in (9, 4, 7, 5)]
    F[1][:, 2] = 0.0  # a zero column keeps lambda 0 and the column unscaled
    for n in range(4):
        assert rel(oracle_lib.gram_loo(F, n), oracle_lib.ref_gram_loo(F, n)) < 1e-14
    Hn, lam = oracle_lib.normalize(F[1])
    Hr, lr = oracle_lib.ref_normalize(F[1])
    assert rel(Hn, Hr) < 1e-14 and rel(lam, lr) < 1e-14 and lr[2] == 0.0


@_live
def test_reference_tensor_fill_matches_mt19937_pin(oracle_lib):
    # the reference's own Tensor(dims) constructor fill (single-threaded)
    gold = np.load(os.path.join(GOLD, "mt19937_103.npz"))["values"]
    t = oracle_lib.RefTensor(dims=(16, 16, 16))
    assert np.array_equal(t.data().ravel(order="F"), gold)
    t.close()
