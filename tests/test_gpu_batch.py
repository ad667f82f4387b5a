"""Batched factorisation of many uneven tensors in one CUDA graph per
iteration (planc_gpu_batch_*), checked member by member against single
contexts and the CPU oracle."""
import numpy as np
import pytest

from helpers import cp_tensor, init_factors, rel

pytestmark = pytest.mark.gpu


def _members(n=6, seed=40):
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        dims = tuple(int(d) for d in rng.integers(20, 70, size=3))
        k = int(rng.choice([4, 8, 16]))
        X, _ = cp_tensor(dims, k, noise=0.01, seed=seed + i)
        out.append((X, init_factors(dims, k, seed=seed + 100 + i)))
    return out


@pytest.mark.parametrize("prec", ["fp64", "bf16"])
def test_batch_matches_single_contexts(gpu, oracle_lib, prec):
    members = _members()
    iters = 8
    with gpu.Batch(0, prec, nstreams=4) as b:
        for X, F0 in members:
            b.add(X.astype(np.float32) if prec != "fp64" else X, F0)
        errs = b.run("hals", iters)
        for i, (X, F0) in enumerate(members):
            Fb, lb = b.get_factors(i)
            with gpu.Context(0, prec) as c:
                c.set_tensor(X.astype(np.float32) if prec != "fp64" else X)
                c.set_factors(F0)
                e = c.run("hals", iters)
                Fc, lc = c.get_factors()
            assert rel(errs[i], e) < 1e-13
            assert all(rel(a, b_) < 1e-13 for a, b_ in zip(Fb, Fc))
            if prec == "fp64":
                Fo, lo, eo = oracle_lib.ntf_run(X, F0, "hals", iters)
                assert rel(errs[i], eo) < 1e-10


@pytest.mark.parametrize("prec", ["fp64", "bf16"])
def test_batch_autotune_keeps_results(gpu, prec):
    members = _members(n=5, seed=50)
    with gpu.Batch(0, prec, nstreams=4) as b:
        for X, F0 in members:
            b.add(X.astype(np.float32) if prec != "fp64" else X, F0)
        e_ref = b.run("hals", 4)
        for i, (X, F0) in enumerate(members):
            b.set_factors(i, F0)
        ms = b.autotune("hals", trials=2)
        assert ms > 0
        e_tuned = b.run("hals", 4)
    # a retuned split-K count reorders the tensor cores' FP32 sums (BF16)
    assert rel(e_tuned, e_ref) < (1e-10 if prec == "fp64" else 1e-5)


def _grouped_members():
    # uneven shapes and ranks, including a mode-0 size that is a multiple of
    # 128 (the right contraction then forms mode 0's multi-TTV itself) and a
    # rank above 32 (the 64-column instances of the grouped kernels)
    rng = np.random.default_rng(60)
    specs = [((128, 40, 30), 8), ((30, 35, 40), 40), ((64, 20, 90), 32)]
    specs += [(tuple(int(d) for d in rng.integers(20, 70, size=3)), int(rng.choice([4, 8, 16, 32])))
              for _ in range(5)]
    out = []
    for i, (dims, k) in enumerate(specs):
        X, _ = cp_tensor(dims, min(k, 8), noise=0.01, seed=70 + i)
        out.append((X.astype(np.float32), init_factors(dims, k, seed=170 + i)))
    return out


@pytest.mark.parametrize("prec,algo", [("bf16", "hals"), ("bf16", "mu"), ("bf16x2", "hals")])
def test_batch_grouped_phases_give_the_same_bits(gpu, prec, algo, monkeypatch):
    # one launch per phase for all members vs one launch per member: the same
    # kernel bodies and summation orders, so the same bits
    members = _grouped_members()
    iters = 4
    res = {}
    for grouped in ("1", "0"):
        monkeypatch.setenv("PLANC_GPU_BATCH_GROUPED", grouped)
        with gpu.Batch(0, prec, nstreams=4) as b:
            for X, F0 in members:
                b.add(X, F0)
            errs = b.run(algo, iters)
            res[grouped] = (errs, [b.get_factors(i) for i in range(len(members))])
    (e1, f1), (e0, f0) = res["1"], res["0"]
    assert np.array_equal(e1, e0)
    for (Fa, la), (Fb, lb) in zip(f1, f0):
        assert np.array_equal(la, lb)
        assert all(np.array_equal(a, b_) for a, b_ in zip(Fa, Fb))
