"""Build recipe of the native library: nvcc for sm_100a, in-tree output.

    python -m planc_b200.build          # builds planc_b200/libplanc_gpu.so
                                        # and the dense_ntf driver (g++)
"""
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
SRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libplanc_gpu.so")
DRIVER = os.path.join(HERE, "dense_ntf")
DRIVERS = {"dense_ntf": "ntf.cpp", "dense_nmf": "nmf.cpp"}

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-lineinfo", "-O3", "-std=c++17",
    "-Xcompiler", "-fPIC", "-shared",
    "--expt-relaxed-constexpr",
    "-Xptxas", "-v",
]


def nvcc():
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if c and os.path.exists(c):
            return c
    raise RuntimeError("nvcc not found")


def sources():
    return [os.path.join(SRC, f) for f in sorted(os.listdir(SRC)) if f.endswith((".cu", ".cuh"))] + [
        os.path.join(ROOT, "include", "planc_gpu.h")]


def needs_build():
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    return any(os.path.getmtime(s) > t for s in sources())


def build(force=False, verbose=False):
    if not force and not needs_build():
        build_driver()
        return LIB
    cmd = [nvcc()] + NVCC_FLAGS + ["-o", LIB + ".tmp", os.path.join(SRC, "planc_gpu.cu"), "-lcuda"]
    cmd[cmd.index("-lcuda"):] = ["-L/usr/local/cuda/lib64/stubs", "-lcuda"]
    res = subprocess.run(cmd, capture_output=True, text=True)
    log = os.path.join(HERE, "build.log")
    with open(log, "w") as f:
        f.write(" ".join(cmd) + "\n" + res.stdout + res.stderr)
    if res.returncode != 0:
        sys.stderr.write(res.stdout + res.stderr)
        raise RuntimeError("nvcc failed (see %s)" % log)
    if verbose:
        sys.stderr.write(res.stderr)
    os.replace(LIB + ".tmp", LIB)
    build_driver()
    return LIB


def driver_sources():
    cpp = os.path.join(HERE, "cpp")
    return [os.path.join(cpp, f) for f in DRIVERS.values()] + [
        os.path.join(cpp, "planc", f) for f in sorted(os.listdir(os.path.join(cpp, "planc")))]


def build_driver(force=False):
    """The dense_ntf and dense_nmf command-line drivers over the C++ API,
    linked to the library."""
    for exe, src in DRIVERS.items():
        out = os.path.join(HERE, exe)
        if (not force and os.path.exists(out) and
                all(os.path.getmtime(s) <= os.path.getmtime(out) for s in driver_sources() + [LIB])):
            continue
        cmd = ["g++", "-O2", "-std=c++17", "-I" + os.path.join(ROOT, "include"),
               "-I" + os.path.join(HERE, "cpp"), os.path.join(HERE, "cpp", src),
               "-L" + HERE, "-lplanc_gpu", "-Wl,-rpath,$ORIGIN", "-o", out]
        subprocess.run(cmd, check=True)
    return DRIVER


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
    print(LIB)
