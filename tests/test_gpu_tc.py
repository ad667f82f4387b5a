"""GPU parity of the tensor-core (tcgen05) MTTKRP paths against the FP64
oracle, through the C ABI.

Stated error bounds (max-abs error / max-abs value of the FP64 result):
  bf16   : the tensor is rounded to BF16 (relative 2^-9 per element), factors
           and Khatri-Rao rows are split hi+lo (relative ~2^-17), FP32
           accumulation: bound 4e-3.
  bf16x2 : the tensor is split hi+lo as well: bound 2e-5.
Final relative error of a full NTF run vs the FP64 path: within 1e-4
(absolute), the north-star bar for mixed precision, for bf16x2 at every size
and for bf16 at 192^3. The bf16 error estimate carries its own noise: the
Gram-form error uses <bf16(X), model>, whose deviation from <X, model> is a
sum of numel rounding errors, about 2 * 0.0016 / sqrt(numel) relative to
||X||^2; divided by 2*err that is ~3e-4 at 64^3 with err ~ 0.01 (and ~5e-6
at 1024^3). At 64^3 the bf16 bound is therefore 1e-3."""
import numpy as np
import pytest

from helpers import cp_tensor, init_factors, rel

pytestmark = pytest.mark.gpu
BOUND = {"bf16": 4e-3, "bf16x2": 2e-5}


def _normalized(F):
    return [f / np.linalg.norm(f, axis=0) for f in F]


@pytest.mark.parametrize("prec", ["bf16", "bf16x2"])
@pytest.mark.parametrize("dims,k", [((64, 64, 64), 8), ((40, 33, 21), 32), ((13, 7, 20), 5),
                                    ((9, 8, 7, 10), 64), ((130, 3, 300), 16), ((24, 16, 16, 40), 32),
                                    # 4-way, balanced tree: split-K of the long right
                                    # contraction (128 rows, K = 4096), ragged K
                                    ((8, 16, 64, 64), 16), ((7, 9, 33, 65), 20),
                                    ((16, 12, 40, 40), 64)])
def test_tc_mttkrp_all_modes(gpu, oracle_lib, prec, dims, k):
    X, _ = cp_tensor(dims, 4, seed=21)
    F = init_factors(dims, k, seed=22)
    Fn = _normalized(F)
    with gpu.Context(0, prec) as c:
        c.set_tensor(X)
        c.set_factors(F)
        for n in range(len(dims)):
            ref = oracle_lib.mttkrp_direct(X, Fn, n)
            got = c.mttkrp(n, dimtree=True)
            assert rel(got, ref) < BOUND[prec], (n, rel(got, ref))


@pytest.mark.parametrize("prec", ["bf16", "bf16x2"])
@pytest.mark.parametrize("algo", ["hals", "mu", "anlsbpp"])
def test_tc_ntf_matches_fp64_error(gpu, prec, algo):
    dims, k, iters = (64, 64, 64), 8, 20
    X, _ = cp_tensor(dims, k, noise=0.01, seed=23)
    F0 = init_factors(dims, k, seed=24)
    with gpu.Context(0, "fp64") as c:
        c.set_tensor(X)
        c.set_factors(F0)
        e64 = c.run(algo, iters)
    with gpu.Context(0, prec) as c:
        c.set_tensor(X.astype(np.float32))
        c.set_factors(F0)
        e = c.run(algo, iters)
        assert abs(c.objective_error() - e[-1]) < 1e-4
    assert np.all(np.isfinite(e))
    tol = 1e-4 if prec == "bf16x2" else 1e-3
    assert abs(e[-1] - e64[-1]) < tol, (e[-1], e64[-1])


@pytest.mark.parametrize("algo", ["hals", "anlsbpp"])
def test_tc_bf16_error_within_1e4_at_192cube(gpu, algo):
    dims, k, iters = (192, 192, 192), 16, 12
    X, _ = cp_tensor(dims, k, noise=0.01, seed=26)
    F0 = init_factors(dims, k, seed=27)
    errs = {}
    for prec in ("fp64", "bf16"):
        with gpu.Context(0, prec) as c:
            c.set_tensor(X.astype(np.float32))
            c.set_factors(F0)
            errs[prec] = c.run(algo, iters)[-1]
    assert abs(errs["bf16"] - errs["fp64"]) < 1e-4, errs


@pytest.mark.parametrize("prec", ["bf16", "bf16x2"])
# mode 1 of the 3-way tree reads the FP32 P with k_ttv_left_f4 (two i1 per
# CTA, float4 loads) once I1 / 2 gives a CTA per SM: 8 and 16 threads a row,
# and an odd I1 whose last CTA has a single i1
@pytest.mark.parametrize("dims,k", [((64, 320, 24), 12), ((40, 297, 20), 32), ((32, 300, 16), 64)])
def test_tc_mode1_ttv_two_rows_per_cta(gpu, oracle_lib, prec, dims, k):
    X, _ = cp_tensor(dims, 4, seed=33)
    F = init_factors(dims, k, seed=34)
    Fn = _normalized(F)
    with gpu.Context(0, prec) as c:
        c.set_tensor(X)
        c.set_factors(F)
        for n in range(3):
            ref = oracle_lib.mttkrp_direct(X, Fn, n)
            got = c.mttkrp(n, dimtree=True)
            assert rel(got, ref) < BOUND[prec], (n, rel(got, ref))


def test_tc_large_split_k(gpu, oracle_lib):
    # long reduction (L = 147456 -> many split-K partials) and R = 300 with a
    # ragged last tile
    dims, k = (384, 384, 300), 32
    rng = np.random.default_rng(5)
    X = np.asfortranarray(rng.random(dims, dtype=np.float32))
    F = init_factors(dims, k, seed=25)
    Fn = _normalized(F)
    with gpu.Context(0, "bf16x2") as c:
        c.set_tensor(X)
        c.set_factors(F)
        for n in (0, 2):
            ref = oracle_lib.mttkrp_direct(X.astype(np.float64), Fn, n)
            assert rel(c.mttkrp(n), ref) < BOUND["bf16x2"]


@pytest.mark.parametrize("prec", ["bf16x2"])
def test_tc_4way_ntf_matches_fp64_error(gpu, prec):
    # the 4-way tensor-core path runs the balanced {0,1}|{2,3} tree, the FP64
    # path the reference's {0,1,2}|{3}: same iterates within the bf16x2 bound
    dims, k, iters = (24, 20, 32, 28), 6, 15
    X, _ = cp_tensor(dims, k, noise=0.01, seed=41)
    F0 = init_factors(dims, k, seed=42)
    errs = {}
    for p in ("fp64", prec):
        with gpu.Context(0, p) as c:
            c.set_tensor(X if p == "fp64" else X.astype(np.float32))
            c.set_factors(F0)
            errs[p] = c.run("hals", iters)
    assert abs(errs[prec][-1] - errs["fp64"][-1]) < 1e-4, (errs[prec][-1], errs["fp64"][-1])


@pytest.mark.parametrize("prec", ["bf16", "bf16x2"])
@pytest.mark.parametrize("dims,k", [((256, 40, 50), 16), ((512, 30, 20), 32), ((384, 17, 23), 24),
                                    ((128, 9, 31), 5)])
def test_tc_mode0_ttv_in_right_contraction(gpu, oracle_lib, prec, dims, k):
    # 3-way tensors whose mode 0 is a multiple of 128 form the mode-0
    # multi-TTV inside the right contraction's epilogue (per-CTA partials
    # reduced in order) instead of re-reading P
    X, _ = cp_tensor(dims, 4, seed=28)
    F = init_factors(dims, k, seed=29)
    Fn = _normalized(F)
    with gpu.Context(0, prec) as c:
        c.set_tensor(X)
        c.set_factors(F)
        for n in range(3):
            ref = oracle_lib.mttkrp_direct(X, Fn, n)
            assert rel(c.mttkrp(n, dimtree=True), ref) < BOUND[prec], n


def test_tc_ntf_fused_ttv_matches_fp64_error(gpu):
    dims, k, iters = (256, 64, 48), 8, 15
    X, _ = cp_tensor(dims, k, noise=0.01, seed=30)
    F0 = init_factors(dims, k, seed=31)
    errs = {}
    for p in ("fp64", "bf16x2"):
        with gpu.Context(0, p) as c:
            c.set_tensor(X if p == "fp64" else X.astype(np.float32))
            c.set_factors(F0)
            errs[p] = c.run("hals", iters)
    assert abs(errs["bf16x2"][-1] - errs["fp64"][-1]) < 1e-4


# ---- direct (non-tree) MTTKRP on the tensor cores: AUNTF's default
# dim_tree(false) path (common/tensor.hpp:246-327) and tensors of 2 or 5+ modes.
# Each mode is the left contraction of a copy of the BF16 tensor with that
# mode moved last (a permutation of the stored values).
@pytest.mark.parametrize("prec", ["bf16", "bf16x2"])
@pytest.mark.parametrize("dims,k", [((64, 64, 64), 8), ((40, 33, 21), 32), ((13, 7, 20), 5),
                                    ((9, 8, 7, 10), 64), ((128, 5, 9, 64), 16),
                                    ((5, 4, 6, 3, 4), 6), ((4, 3, 5, 2, 3, 4), 12),
                                    ((300, 70), 20), ((64, 128), 64)])
def test_tc_direct_mttkrp_all_modes(gpu, oracle_lib, prec, dims, k):
    X, _ = cp_tensor(dims, 3, seed=25)
    F = init_factors(dims, k, seed=26)
    Fn = _normalized(F)
    with gpu.Context(0, prec) as c:
        c.set_tensor(X)
        c.set_factors(F)
        for n in range(len(dims)):
            ref = oracle_lib.mttkrp_direct(X, Fn, n)
            got = c.mttkrp(n, dimtree=False)
            assert rel(got, ref) < BOUND[prec], (n, rel(got, ref))
        if len(dims) in (3, 4):  # the tree and the direct path agree as well
            for n in range(len(dims)):
                assert rel(c.mttkrp(n, dimtree=True), c.mttkrp(n, dimtree=False)) < 2 * BOUND[prec]


@pytest.mark.parametrize("prec", ["bf16", "bf16x2"])
@pytest.mark.parametrize("dims,k,algo", [((64, 64, 64), 8, "hals"), ((30, 24, 20, 16), 5, "anlsbpp"),
                                         ((12, 10, 9, 8, 7), 4, "mu")])
def test_tc_direct_ntf_matches_fp64(gpu, prec, dims, k, algo):
    # whole runs with dimtree = false (and 5 modes, where no tree exists):
    # final relative error within the mixed-precision bounds of the FP64 path
    iters = 12
    X, _ = cp_tensor(dims, k, noise=0.01, seed=27)
    F0 = init_factors(dims, k, seed=28)
    with gpu.Context(0, "fp64") as c:
        c.set_tensor(X)
        c.set_factors(F0)
        e64 = c.run(algo, iters, dimtree=False)
    with gpu.Context(0, prec) as c:
        c.set_tensor(X.astype(np.float32))
        c.set_factors(F0)
        e = c.run(algo, iters, dimtree=False)
        assert abs(c.objective_error() - e[-1]) < 1e-3
    bound = 1e-3 if prec == "bf16" else 1e-4
    assert abs(e[-1] - e64[-1]) < bound, (e[-1], e64[-1])


@pytest.mark.parametrize("prec", ["bf16", "bf16x2"])
@pytest.mark.parametrize("chunks", [1, 8, 1000])
def test_tc_left_split_length_keeps_the_bound(gpu, oracle_lib, prec, chunks, monkeypatch):
    # PLANC_GPU_LEFT_CHUNKS (the batch autotuner's split-K length of the left
    # contraction) only reorders the FP32 partial sums: every mode stays
    # within the precision's bound, for the generic (I0 % 64 != 0) and the
    # factored (I0 % 64 == 0) left contraction
    monkeypatch.setenv("PLANC_GPU_LEFT_CHUNKS", str(chunks))
    # the producer-warp form of the generic left contraction (the default for
    # I0 % 64 != 0 is the long-K kernel over a Khatri-Rao image)
    monkeypatch.setenv("PLANC_GPU_LEFT_FORM", "producers")
    for dims, k in (((40, 33, 96), 16), ((64, 20, 70), 32)):
        X, _ = cp_tensor(dims, 4, seed=31)
        F = init_factors(dims, k, seed=32)
        Fn = _normalized(F)
        with gpu.Context(0, prec) as c:
            c.set_tensor(X)
            c.set_factors(F)
            for n in range(3):
                ref = oracle_lib.mttkrp_direct(X, Fn, n)
                got = c.mttkrp(n, dimtree=True)
                assert rel(got, ref) < BOUND[prec], (dims, n, rel(got, ref))


@pytest.mark.parametrize("prec", ["bf16", "bf16x2"])
def test_tc_tile_loads_agree(gpu, prec, monkeypatch):
    # the tensor tiles of the right and factored left contractions through
    # cp.async producer warps (PLANC_GPU_TC_LOADS=cpasync) or TMA. The right
    # contraction fills the same shared-memory image and runs the same MMAs,
    # so mode 0 (formed from it alone) has the same bits; the factored left
    # contraction's cp.async instance takes one 128-row tile a CTA (TMA: two
    # when R > 128), so its split-K partials are summed in another order
    # (FP64, relative 1e-12). Shapes cover ragged rows (L = I0*I1 not a
    # multiple of 8 or of 128), ragged K (I2 < 64, I2 % 64 != 0), ranks of the
    # 16-, 32- and 64-column instances, the fused mode-0 multi-TTV
    # (I0 % 128 == 0), the factored left contraction (I0 % 64 == 0; I0 = 64 has
    # runs of one chunk, which the cp.async instance does not take) with ragged
    # j, and the direct (non-tree) MTTKRP of every mode
    cases = [((13, 7, 20), 5), ((40, 33, 21), 32), ((130, 3, 300), 16), ((256, 40, 50), 16),
             ((384, 17, 23), 24), ((9, 8, 7, 10), 64), ((64, 20, 90), 40), ((128, 12, 300), 32),
             ((64, 10, 200), 16), ((256, 6, 333), 8)]
    for dims, k in cases:
        X, _ = cp_tensor(dims, 4, seed=33)
        F = init_factors(dims, k, seed=34)
        res = {}
        for loads in ("tma", "cpasync"):
            monkeypatch.setenv("PLANC_GPU_TC_LOADS", loads)
            with gpu.Context(0, prec) as c:
                c.set_tensor(X)
                c.set_factors(F)
                ms = [c.mttkrp(n, dimtree=True) for n in range(len(dims))]
                ms += [c.mttkrp(n, dimtree=False) for n in range(len(dims))]
                e = c.run("hals", 3)
                res[loads] = (ms, e, c.get_factors()[0])
        (m1, e1, f1), (m2, e2, f2) = res["tma"], res["cpasync"]
        assert np.array_equal(m1[0], m2[0]), dims
        assert all(rel(a, b) < 1e-12 for a, b in zip(m1, m2)), (dims, [rel(a, b) for a, b in zip(m1, m2)])
        assert np.max(np.abs(np.asarray(e1) - np.asarray(e2))) < 1e-10, dims
        assert all(rel(a, b) < 1e-8 for a, b in zip(f1, f2)), dims


@pytest.mark.parametrize("prec", ["bf16", "bf16x2"])
@pytest.mark.parametrize("form", ["image", "producers"])
def test_tc_generic_left_forms_keep_the_bound(gpu, oracle_lib, prec, form, monkeypatch):
    # 3-way tensors with I0 % 64 != 0: the left contraction (mode 2 of the
    # tree, and the direct MTTKRP of modes whose view lacks the factored form)
    # against a Khatri-Rao image with the long-K kernel, or with Khatri-Rao
    # producer warps; both within the precision's bound, for one and two
    # 128-row tiles per CTA (R > 128 at rank <= 32) and rank 64
    monkeypatch.setenv("PLANC_GPU_LEFT_FORM", form)
    for dims, k in (((40, 33, 96), 16), ((37, 45, 300), 32), ((50, 21, 140), 64), ((13, 7, 20), 5)):
        X, _ = cp_tensor(dims, 4, seed=35)
        F = init_factors(dims, k, seed=36)
        Fn = _normalized(F)
        with gpu.Context(0, prec) as c:
            c.set_tensor(X)
            c.set_factors(F)
            for n in range(3):
                ref = oracle_lib.mttkrp_direct(X, Fn, n)
                for tree in (True, False):
                    got = c.mttkrp(n, dimtree=tree)
                    assert rel(got, ref) < BOUND[prec], (dims, n, tree, rel(got, ref))
            e = c.run("hals", 3)
            assert np.all(np.isfinite(e))
