"""CPU checks of the C ABI boundary: the library loads and exports exactly the
entry points include/planc_gpu.h declares (no compute calls)."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for hdr in os.listdir(os.path.join(ROOT, "include")):
        if hdr.endswith(".h"):
            txt = open(os.path.join(ROOT, "include", hdr)).read()
            txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
            names |= set(re.findall(r"\b(planc_gpu_\w+)\s*\(", txt))
    return names


def test_header_declares_entry_points():
    names = declared_symbols()
    assert "planc_gpu_run" in names and "planc_gpu_set_tensor" in names
    assert len(names) >= 15


def test_library_exports_every_declared_symbol(gpu):
    lib = ctypes.CDLL(gpu.LIB_PATH)
    missing = [n for n in sorted(declared_symbols()) if not hasattr(lib, n)]
    assert not missing, missing
    assert set(gpu.EXPORTS) <= declared_symbols()


def test_abi_version(gpu):
    assert gpu.load().planc_gpu_abi_version() == 1


def test_null_arguments_rejected_without_device(gpu):
    L = gpu.load()
    # argument validation happens before any device work
    assert L.planc_gpu_create(None, 0, 0, None) == -1
    assert L.planc_gpu_destroy(None) == 0
    assert L.planc_gpu_set_tensor(None, None, 0, None, 3, 0) == -1
    assert L.planc_gpu_run(None, 1, 1, 1, 0, None) == -1


@pytest.mark.skipif(__import__("torch").cuda.is_available(), reason="has a GPU")
def test_create_without_gpu_fails_cleanly(gpu):
    with pytest.raises(gpu.PlancGpuError):
        gpu.Context(0, "fp64")
