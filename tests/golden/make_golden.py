"""Generates the golden fixtures in tests/golden/ (run in a tree where the
reference sources are present, so oracle/_ref/libref_dimtree.so is built from
them).

  ref_dimtree_mttkrp.npz : MTTKRP of every mode computed by the REFERENCE's own
      dimension-tree kernels (dimtree/dimtrees.hpp, dimtree/ddttensor.hpp,
      compiled unmodified by oracle/Makefile) on Tensor(dims)-style inputs
      (std::mt19937(103) uniform data, common/tensor.hpp:86-93, 219-235) and
      fixed numpy factors, for N = 3 and N = 4.
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
        raise SystemExit("oracle/_ref/libref_dimtree.so missing: build it from the reference tree")
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
    print("wrote", sorted(os.listdir(OUT)))


if __name__ == "__main__":
    main()
