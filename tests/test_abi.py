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


def test_stage_timing_lines_in_the_reference_format():
    """With SARDINE_B200_TIMING=1 every entry point reports its stage on
    stderr as the reference's report_timing does ("[timing] <stage> = <s> s",
    run.rs:54-60), also when it returns an error status; each call is an
    NVTX range under the same name.  A null context needs no GPU."""
    import subprocess
    import sys
    code = ("import ctypes; from sardine_b200 import _lib; L = _lib.lib(); "
            "rc = L.sd_speckle(None, None, 0, 0, 0, 0, 3, ctypes.c_float(1.0), ctypes.c_float(0.0), None); "
            "rc2 = L.sd_to_db(None, None, 0, ctypes.c_float(0.0), None, None); print(rc, rc2)")
    env = dict(os.environ, SARDINE_B200_TIMING="1")
    out = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True, timeout=120)
    assert out.returncode == 0, out.stderr
    assert re.search(r"^\[timing\] speckle = \d+\.\d{3} s$", out.stderr, re.M), out.stderr
    assert re.search(r"^\[timing\] db_conversion = \d+\.\d{3} s$", out.stderr, re.M), out.stderr
    env.pop("SARDINE_B200_TIMING")
    out = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True, timeout=120)
    assert "[timing]" not in out.stderr
