"""The C-ABI library loads on a CPU-only machine and exports every entry
point include/rome_gpu.h declares (no compute call is made)."""
import ctypes
import os
import re

from rome_b200 import abi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    src = open(os.path.join(ROOT, "include", "rome_gpu.h")).read()
    return sorted(set(re.findall(r"\b(rome_gpu_[a-z0-9_]+)\s*\(", src)))


def test_header_and_binding_agree():
    assert declared_symbols() == sorted(abi.EXPORTED_SYMBOLS)


def test_library_exports_every_declared_symbol():
    lib = abi.load_library()
    for name in declared_symbols():
        assert hasattr(lib, name), name
        assert ctypes.cast(getattr(lib, name), ctypes.c_void_p).value


def test_abi_version_callable_without_gpu():
    lib = abi.load_library()
    lib.rome_gpu_abi_version.restype = ctypes.c_int
    assert lib.rome_gpu_abi_version() == abi.ABI_VERSION == 4


def test_create_fails_cleanly_without_device():
    """On a machine without a usable sm_100 device, create returns an error code."""
    import torch
    if torch.cuda.is_available():
        return
    lib = abi.load_library()
    h = ctypes.c_void_p()
    rc = lib.rome_gpu_create(0, None, ctypes.byref(h))
    assert rc != abi.ROME_OK and not h.value
