"""The C++ drop-in layer on the GPU: the dense_ntf driver (Tensor(dims) data,
--init injection through AUNTF::reset, the reference's printed error lines)
and a user AUNTF subclass with a host update(), both against the oracle."""
import os
import re
import subprocess

import numpy as np
import pytest

from helpers import init_factors, rel

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "planc_b200")


def _compile(src, out):
    cmd = ["g++", "-O2", "-std=c++17", "-I" + os.path.join(ROOT, "include"),
           "-I" + os.path.join(PKG, "cpp"), src, "-L" + PKG, "-lplanc_gpu",
           "-Wl,-rpath," + PKG, "-o", out]
    subprocess.run(cmd, check=True)


def _write_init(prefix, F):
    for n, f in enumerate(F):
        np.savetxt("%s_%d.txt" % (prefix, n), f, fmt="%.17g")


def _read_factors(prefix, N):
    return [np.loadtxt("%s_%d.txt" % (prefix, n), ndmin=2) for n in range(N)]


@pytest.mark.parametrize("algo,code", [("hals", 1), ("mu", 0), ("anlsbpp", 2), ("aoadmm", 4),
                                       ("nesterov", 5)])
def test_dense_ntf_driver_matches_oracle(gpu, oracle_lib, tmp_path, algo, code):
    exe = str(tmp_path / "dense_ntf")
    _compile(os.path.join(PKG, "cpp", "ntf.cpp"), exe)
    # 8 iterations: the Nesterov acceleration runs from iteration 6 on
    dims, k, iters = (24, 20, 16), 4, 8
    F0 = init_factors(dims, k, seed=60)
    init = str(tmp_path / "init")
    _write_init(init, F0)
    out = str(tmp_path / "out")
    res = subprocess.run([exe, "-a", str(code), "-d", " ".join(map(str, dims)), "-k", str(k),
                          "-t", str(iters), "-e", "1", "--init", init, "-o", out],
                         capture_output=True, text=True, check=True)
    errs = [float(m) for m in re.findall(r"relative_error at it::\d+::([0-9.eE+-]+)", res.stdout)]
    assert len(errs) == iters
    X = oracle_lib.tensor_randu(dims, 103)  # Tensor(dims) data
    Fo, lo, eo = oracle_lib.ntf_run(X, F0, algo, iters)
    assert rel(np.array(errs), eo) < 1e-5  # printed with 6 significant digits
    Fg = _read_factors(out, 3)
    # the driver writes NCPFactors::factor(n) (I_n x k)
    assert all(rel(a, b) < 1e-10 for a, b in zip(Fg, Fo))


def test_custom_host_update_subclass(gpu, oracle_lib, tmp_path):
    exe = str(tmp_path / "custom_update")
    _compile(os.path.join(ROOT, "tests", "cpp", "custom_update.cpp"), exe)
    dims, k, iters = (18, 15, 12), 3, 4
    F0 = init_factors(dims, k, seed=61)
    init, out = str(tmp_path / "init"), str(tmp_path / "out")
    _write_init(init, F0)
    res = subprocess.run([exe] + [str(d) for d in dims] + [str(k), str(iters), init, out],
                         capture_output=True, text=True, check=True)
    X = oracle_lib.tensor_randu(dims, 103)
    Fo, lo, eo = oracle_lib.ntf_run(X, F0, "hals", iters)
    Fg = _read_factors(out, 3)
    assert all(rel(a, b) < 1e-10 for a, b in zip(Fg, Fo))
    final = float(re.search(r"final_error ([0-9.eE+-]+)", res.stdout).group(1))
    assert abs(final - eo[-1]) / eo[-1] < 1e-5


def test_dense_ntf_reads_npy(gpu, oracle_lib, tmp_path):
    # -i <file>.npy goes through NumPyArray::load (common/npyio.hpp); the shape
    # comes from the file, so -d is left out
    exe = str(tmp_path / "dense_ntf")
    _compile(os.path.join(PKG, "cpp", "ntf.cpp"), exe)
    dims, k, iters = (20, 16, 12), 4, 6
    rng = np.random.default_rng(62)
    X = np.asfortranarray(rng.random(dims))
    src = str(tmp_path / "x.npy")
    np.save(src, X)
    F0 = init_factors(dims, k, seed=63)
    init, out = str(tmp_path / "init"), str(tmp_path / "out")
    _write_init(init, F0)
    res = subprocess.run([exe, "-a", "1", "-i", src, "-k", str(k), "-t", str(iters), "-e", "1",
                          "--init", init, "-o", out], capture_output=True, text=True, check=True)
    errs = [float(m) for m in re.findall(r"relative_error at it::\d+::([0-9.eE+-]+)", res.stdout)]
    Fo, lo, eo = oracle_lib.ntf_run(X, F0, "hals", iters)
    assert rel(np.array(errs), eo) < 1e-5
    assert all(rel(a, b) < 1e-10 for a, b in zip(_read_factors(out, 3), Fo))


@pytest.mark.parametrize("algo,code", [("mu", 0), ("hals", 1), ("anlsbpp", 2)])
def test_dense_nmf_driver_matches_oracle(gpu, oracle_lib, tmp_path, algo, code):
    # the NMF classes of the C++ API (HALSNMF / MUNMF / BPPNMF) through the
    # dense_nmf driver: A from a .npy file, W and H injected, L1/L2
    # regularisation on both factors
    exe = str(tmp_path / "dense_nmf")
    _compile(os.path.join(PKG, "cpp", "nmf.cpp"), exe)
    m, n, k, iters = 48, 36, 5, 7
    rng = np.random.default_rng(64)
    A = np.asfortranarray(rng.random((m, k)) @ rng.random((k, n)) + 0.01 * rng.random((m, n)))
    src = str(tmp_path / "a.npy")
    np.save(src, A)
    W0, H0 = rng.random((m, k)), rng.random((n, k))
    init, out = str(tmp_path / "init"), str(tmp_path / "out")
    np.savetxt(init + "_W.txt", W0, fmt="%.17g")
    np.savetxt(init + "_H.txt", H0, fmt="%.17g")
    res = subprocess.run([exe, "-a", str(code), "-i", src, "-k", str(k), "-t", str(iters),
                          "--init", init, "-o", out, "-r", "0.1 0.05 0.2 0.01"],
                         capture_output=True, text=True, check=True)
    rels = [float(x) for x in re.findall(r"relative error::([0-9.eE+-]+)", res.stdout)]
    assert len(rels) == iters
    # the regularisers are FVEC (float) in the API, as in the reference
    # (common/nmf.hpp:49-50, 82, 88): the oracle gets the float values
    regf = tuple(float(np.float32(x)) for x in (0.1, 0.05, 0.2, 0.01)) + (0.0,)
    Wo, Ho, oo, ro = oracle_lib.nmf_run(A, W0, H0, algo, iters, reg=regf)
    assert rel(np.array(rels), ro) < 1e-5  # printed with 6 significant digits
    W = np.loadtxt(out + "_W", ndmin=2)
    H = np.loadtxt(out + "_H", ndmin=2)
    assert rel(W, Wo) < 1e-10 and rel(H, Ho) < 1e-10


@pytest.mark.parametrize("prec", ["bf16", "bf16x2"])
def test_dense_ntf_direct_mttkrp_mixed_precision(gpu, oracle_lib, tmp_path, prec):
    # AUNTF's default dim_tree(false) (the reference's direct MTTKRP,
    # common/tensor.hpp:246-327) on the tensor-core precisions:
    # dense_ntf --dimtree 0 --precision bf16|bf16x2 against the FP64 oracle
    exe = str(tmp_path / "dense_ntf")
    _compile(os.path.join(PKG, "cpp", "ntf.cpp"), exe)
    dims, k, iters = (48, 40, 36), 4, 8
    F0 = init_factors(dims, k, seed=65)
    init, out = str(tmp_path / "init"), str(tmp_path / "out")
    _write_init(init, F0)
    res = subprocess.run([exe, "-a", "1", "-d", " ".join(map(str, dims)), "-k", str(k), "-t",
                          str(iters), "-e", "1", "--dimtree", "0", "--precision", prec, "--init",
                          init, "-o", out], capture_output=True, text=True, check=True)
    errs = [float(m) for m in re.findall(r"relative_error at it::\d+::([0-9.eE+-]+)", res.stdout)]
    assert len(errs) == iters
    X = oracle_lib.tensor_randu(dims, 103)
    Fo, lo, eo = oracle_lib.ntf_run(X, F0, "hals", iters, dimtree=False)
    # the tensor is uniform noise (error ~0.5): BF16 rounding moves the
    # reported error by ~1e-4
    assert abs(errs[-1] - eo[-1]) < (1e-3 if prec == "bf16" else 1e-5)
