"""Generates the golden fixtures in tests/golden/ (run in a tree where the
reference sources are present, so oracle/_ref/libref_planc.so is built from
them: the reference's own NTF code compiled unmodified against the
Armadillo-subset shim, see oracle/Makefile).

  ref_dimtree_mttkrp.npz : MTTKRP of every mode computed by the REFERENCE's own
      DenseDimensionTree (dimtree/ddt.hpp over dimtree/dimtrees.hpp and
      dimtree/ddttensor.hpp) on Tensor(dims)-style inputs (std::mt19937(103)
      uniform data, common/tensor.hpp:86-93, 219-235) and fixed numpy
      factors, for N = 3 and N = 4.
  ref_ntf_runs.npz : whole runs of the reference's own AUNTF subclasses
      (ntf/auntf.hpp with ntf/ntf{mu,hals,anlsbpp,aoadmm,nes}.hpp) from
      injected initial factors: final factors, lambda and per-iteration
      relative errors. Inputs are CP tensors made by tests/helpers.py's
      cp_tensor (numpy, seeded); the fixture keeps their checksums.
  ref_updates.npz : one update(mode) of each reference NTF class from given
      (factor, MTTKRP, leave-one-out Gram), and BPPNNLS solutions with their
      iteration counts, including a rank-64 system with 192 right-hand sides
      (the size of one mode of the 192^4 rank-64 workload).
  mt19937_103.npz : the first values of std::mt19937(103) fed through
      libstdc++'s uniform_real_distribution<double>, computed independently
      from numpy's MT19937 with the reference's seeding (init_genrand).

    python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests"))
import oracle  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))


def mt19937_uniform(seed, n):
    """std::uniform_real_distribution<double>(0,1) over std::mt19937(seed) as
    libstdc++ implements it (generate_canonical: two 32-bit draws,
    (g1 + g2 * 2^32) / 2^64)."""
    bg = np.random.MT19937()
    bg._legacy_seeding(seed)
    raw = bg.random_raw(2 * n).astype(np.float64)
    g1, g2 = raw[0::2], raw[1::2]
    v = (g1 + g2 * 4294967296.0) / 18446744073709551616.0
    v[v >= 1.0] = np.nextafter(1.0, 0.0)
    return v


def main():
    np.savez(os.path.join(OUT, "mt19937_103.npz"), values=mt19937_uniform(103, 4096))
    if not oracle.ref_available():
        raise SystemExit("oracle/_ref/libref_planc.so missing: build it from the reference tree")
    cases = {}
    for name, dims, k in [("n3", (6, 5, 4), 3), ("n4", (5, 4, 3, 6), 3), ("n3b", (9, 7, 8), 5)]:
        X = oracle.tensor_randu(dims, 103)
        rng = np.random.default_rng(20240611 + len(dims))
        F = [rng.random((d, k)) for d in dims]
        outs = oracle.ref_mttkrp_dimtree_all(X, F)
        cases[name + "_dims"] = np.array(dims)
        cases[name + "_X"] = X.ravel(order="F")
        for i, f in enumerate(F):
            cases["%s_F%d" % (name, i)] = f
        for i, o in enumerate(outs):
            cases["%s_M%d" % (name, i)] = o
    np.savez(os.path.join(OUT, "ref_dimtree_mttkrp.npz"), **cases)
    np.savez_compressed(os.path.join(OUT, "ref_ntf_runs.npz"), **ntf_runs())
    np.savez_compressed(os.path.join(OUT, "ref_updates.npz"), **updates())
    print("wrote", sorted(os.listdir(OUT)))


# (name, dims, rank, iterations, dimtree, algorithms, noise, seed)
RUNS = [
    ("c1", (64, 64, 64), 8, 20, True, ("hals", "mu", "anlsbpp"), 0.01, 101),
    ("s3", (16, 14, 12), 4, 10, True, ("mu", "hals", "anlsbpp", "aoadmm", "nesterov"), 0.05, 102),
    ("s4", (8, 7, 6, 5), 3, 10, True, ("mu", "hals", "anlsbpp", "aoadmm", "nesterov"), 0.05, 103),
    ("d3", (12, 10, 9), 5, 8, False, ("mu", "hals", "anlsbpp"), 0.05, 104),
    ("d5", (5, 4, 3, 4, 3), 3, 6, False, ("hals", "anlsbpp"), 0.05, 105),
]


def run_inputs(dims, k, noise, seed):
    from helpers import cp_tensor
    X, _ = cp_tensor(dims, k, noise=noise, seed=seed)
    rng = np.random.default_rng(seed + 1000)
    F0 = [rng.random((d, k)) for d in dims]
    return X, F0


def ntf_runs():
    out = {}
    for name, dims, k, iters, dt, algos, noise, seed in RUNS:
        X, F0 = run_inputs(dims, k, noise, seed)
        out[name + "_dims"] = np.array(dims)
        out[name + "_meta"] = np.array([k, iters, int(dt), seed])
        out[name + "_noise"] = np.array([noise])
        out[name + "_xsum"] = np.array([X.sum(), (X * X).sum(), X.ravel(order="F")[7]])
        for a in algos:
            F, lam, errs = oracle.ref_ntf_run(X, F0, a, iters, dimtree=dt)
            for i, f in enumerate(F):
                out["%s_%s_F%d" % (name, a, i)] = f
            out["%s_%s_lam" % (name, a)] = lam
            out["%s_%s_err" % (name, a)] = errs
    return out


def updates():
    out = {}
    rng = np.random.default_rng(77)
    for i, (I, k) in enumerate([(40, 6), (25, 12), (9, 3)]):
        H = rng.random((I, k))
        A = rng.random((3 * k, k))
        G = A.T @ A
        M = rng.random((I, k)) * G.sum(1).mean() * 0.3
        out["u%d_H" % i], out["u%d_M" % i], out["u%d_G" % i] = H, M, G
        for a in ("mu", "hals", "anlsbpp", "aoadmm"):
            out["u%d_%s" % (i, a)] = oracle.ref_update(a, H, M, G)
    # BPP on normal equations: random systems and a rank-64, 192-column one
    for i, (n, ncols, zero_frac) in enumerate([(8, 30, 0.0), (20, 50, 0.3), (64, 192, 0.5)]):
        B = rng.random((3 * n, n))
        B[rng.random(B.shape) < zero_frac] = 0.0
        AtA = B.T @ B + 1e-3 * np.eye(n)
        W = rng.random((n, ncols))
        W[rng.random(W.shape) < 0.5] = 0.0
        AtB = AtA @ W + 0.05 * rng.standard_normal((n, ncols)) * np.abs(AtA @ W).mean()
        X, it = oracle.ref_bpp_solve(AtA, AtB)
        out["b%d_AtA" % i], out["b%d_AtB" % i], out["b%d_X" % i] = AtA, AtB, X
        out["b%d_iters" % i] = np.array([it])
    return out


if __name__ == "__main__":
    main()
