"""Tensor IO of the C++ API, on the CPU: NumPyArray::load (the .npy reader of
common/npyio.hpp) and Tensor::read / Tensor::write (raw FP64 with a .info
sidecar, common/tensor.hpp:430-503), checked against numpy."""
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def exe(tmp_path_factory):
    out = str(tmp_path_factory.mktemp("io") / "tensor_io")
    subprocess.run(["g++", "-O2", "-std=c++17", "-I" + os.path.join(ROOT, "planc_b200", "cpp"),
                    os.path.join(ROOT, "tests", "cpp", "tensor_io.cpp"), "-o", out], check=True)
    return out


def _run(exe, how, src, dst):
    res = subprocess.run([exe, how, src, dst], capture_output=True, text=True, check=True)
    f = res.stdout.split()
    n = int(f[0])
    return [int(x) for x in f[1:1 + n]], int(f[1 + n]), [float(x) for x in f[2 + n:]], res.stderr


def _read_bin(path):
    info = open(path[:path.rfind(".")] + ".info").read().split()
    dims = [int(x) for x in info[1:1 + int(info[0])]]
    return np.fromfile(path, dtype=np.float64).reshape(dims, order="F")


@pytest.mark.parametrize("dtype,dims,version", [(np.float64, (7, 5, 3), (1, 0)),
                                                (np.float32, (4, 3, 5, 2), (1, 0)),
                                                (np.float64, (6, 4, 3), (2, 0)),
                                                (np.float64, (9,), (1, 0))])
def test_npy_fortran_order(exe, tmp_path, dtype, dims, version):
    rng = np.random.default_rng(3)
    X = np.asfortranarray(rng.random(dims).astype(dtype))
    src = str(tmp_path / "x.npy")
    with open(src, "wb") as f:
        np.lib.format.write_array(f, X, version=version)
    out = str(tmp_path / "x.bin")
    d, n, (s, first, last), _ = _run(exe, "npy", src, out)
    assert tuple(d) == dims and n == X.size
    ref = X.astype(np.float64)
    assert first == ref.ravel(order="F")[0] and last == ref.ravel(order="F")[-1]
    assert abs(s - ref.sum()) < 1e-12 * abs(ref.sum())
    # Tensor::write of what was read: the .info sidecar and the raw FP64 data
    assert np.array_equal(_read_bin(out), ref)


def test_npy_c_order_is_read_as_stored(exe, tmp_path):
    # the reference reads the stored words as mode-0-fastest data whatever the
    # header's fortran_order says; the reader does the same and warns
    X = np.arange(24, dtype=np.float64).reshape(2, 3, 4)  # C order
    src = str(tmp_path / "c.npy")
    np.save(src, X)
    d, n, (s, first, last), err = _run(exe, "npy", src, str(tmp_path / "c.bin"))
    assert d == [2, 3, 4] and first == 0.0 and last == 23.0
    assert "C order" in err
    got = _read_bin(str(tmp_path / "c.bin"))
    assert np.array_equal(got.ravel(order="F"), X.ravel(order="C"))


def test_bin_info_roundtrip(exe, tmp_path):
    rng = np.random.default_rng(4)
    X = np.asfortranarray(rng.random((5, 6, 7)))
    src = str(tmp_path / "t.bin")
    X.ravel(order="F").tofile(src)
    with open(str(tmp_path / "t.info"), "w") as f:
        f.write("3\n5\n6\n7\n\n")
    out = str(tmp_path / "u.bin")
    d, n, (s, first, last), _ = _run(exe, "bin", src, out)
    assert d == [5, 6, 7] and n == X.size
    assert np.array_equal(_read_bin(out), X)
