"""Seeded synthetic inputs shared by the tests (numpy, host side)."""
import numpy as np


def cp_tensor(dims, k, noise=0.01, seed=0, zero_frac=0.0):
    """Nonnegative CP model with U[0,1) factors (optionally a fraction of
    factor entries zeroed) + Gaussian noise of relative level `noise`
    (sigma = noise * ||M|| / sqrt(numel), dimtree/ddttensor.hpp:951-952),
    clipped at >= 0. Returns (X Fortran-order float64, true factors)."""
    rng = np.random.default_rng(seed)
    A = [rng.random((d, k)) for d in dims]
    if zero_frac > 0:
        for a in A:
            a[rng.random(a.shape) < zero_frac] = 0.0
    letters = "abcdefgh"[:len(dims)]
    M = np.einsum(",".join(c + "z" for c in letters) + "->" + letters, *A)
    sigma = noise * np.linalg.norm(M) / np.sqrt(M.size)
    X = np.maximum(M + sigma * rng.standard_normal(M.shape), 0.0)
    return np.asfortranarray(X), A


def init_factors(dims, k, seed=1):
    rng = np.random.default_rng(seed)
    return [rng.random((d, k)) for d in dims]


def einsum_mttkrp(X, F, n):
    letters = "abcdefgh"[:X.ndim]
    terms = [letters] + [letters[m] + "z" for m in range(X.ndim) if m != n]
    return np.einsum(",".join(terms) + "->" + letters[n] + "z", X,
                     *[F[m] for m in range(X.ndim) if m != n])


def rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))
