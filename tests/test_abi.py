"""The C-ABI library builds, loads without a GPU and exports every entry
point that include/sardine_b200.h declares."""
import ctypes
import os
import re

from sardine_b200 import _lib, build

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    hdr = open(os.path.join(ROOT, "include", "sardine_b200.h")).read()
    return sorted(set(re.findall(r"\b(sd_[a-z0-9_]+)\s*\(", hdr)))


def test_library_loads_and_exports_all_declared_symbols():
    path = build.build()
    lib = ctypes.CDLL(path)
    missing = [s for s in declared_symbols() if not hasattr(lib, s)]
    assert not missing, f"missing exports: {missing}"
    assert lib.sd_abi_version() == 1


def test_python_binding_covers_header():
    assert set(declared_symbols()) <= set(_lib.exported_symbols())


def test_ctx_create_without_gpu_fails_cleanly():
    import torch
    if torch.cuda.is_available():
        return
    h = ctypes.c_void_p()
    rc = _lib.lib().sd_ctx_create(0, ctypes.byref(h))
    assert rc != 0 and not h.value
