"""Loader for libsardine_b200.so (the CUDA implementation behind the C ABI).

There is no CPU fallback: if the shared library is missing or no CUDA device
is present, calls raise.
"""
from __future__ import annotations

import ctypes as C
import os
import threading

from . import _abi

_HERE = os.path.dirname(os.path.abspath(__file__))
# SARDINE_B200_LIB selects another build of the same library (a variant
# compiled with different switches); the default is the in-tree build
LIB_PATH = os.environ.get("SARDINE_B200_LIB", os.path.join(_HERE, "libsardine_b200.so"))
_lib = None
_lock = threading.Lock()

P = C.c_void_p
_SIGS = {
    "sd_abi_version": (C.c_int, []),
    "sd_ctx_create": (C.c_int, [C.c_int, C.POINTER(C.c_void_p)]),
    "sd_ctx_destroy": (None, [P]),
    "sd_last_error": (C.c_char_p, [P]),
    "sd_kernel_launches": (C.c_uint64, [P]),
    "sd_ctx_stream": (P, [P]),
    "sd_ctx_set_timing": (C.c_int, [P, C.c_int]),
    "sd_ctx_kernel_times": (C.c_int, [P, P, C.c_uint64, P, P, C.c_uint64, P]),
    "sd_speckle": (C.c_int, [P, P, C.c_uint64, C.c_uint64, C.c_uint64, C.c_int32, C.c_uint64,
                             C.c_float, C.c_float, P]),
    "sd_compute_overlap_lines": (C.c_int, [P, P, P, C.c_double, C.c_uint64, P]),
    "sd_deburst_plan": (C.c_int, [P, P, P, C.c_uint64, C.c_uint64, P, P, P]),
    "sd_deburst_subswath": (C.c_int, [P, P, C.c_uint64, C.c_uint64, P, P, C.c_uint64, P]),
    "sd_apply_calibration": (C.c_int, [P, P, C.c_uint64, C.c_uint64, C.c_uint64, P, C.c_uint64, P,
                                       C.c_uint64, P, C.c_uint64, P, P, P, P]),
    "sd_apply_calibration_noalloc": (C.c_int, [P, P, C.c_uint64, C.c_uint64, C.c_uint64, P,
                                               C.c_uint64, P, C.c_uint64, P, C.c_uint64, P, P,
                                               P, P, P, C.c_uint64]),
    "sd_merge_subswaths": (C.c_int, [P, C.c_int32, P, P, P, P, P, P, P, P, P, P, P, P]),
    "sd_calibrate_deburst_merge": (C.c_int, [P, C.c_int32, P, P, P, P]),
    "sd_tc_output_grid": (C.c_int, [P, P, P, P]),
    "sd_terrain_correction": (C.c_int, [P, P, P, P, P, P, C.c_uint64, P, P, P, P, P]),
    "sd_terrain_correction_with_times": (C.c_int, [P, P, P, P, P, P, C.c_uint64, P, P, P, P, P, P]),
    "sd_terrain_correction_rows": (C.c_int, [P, P, P, P, P, P, C.c_uint64, P, C.c_uint64, C.c_uint64,
                                             P, P, P, P, P]),
    "sd_scene_create": (C.c_int, [P, P, P, P, P, P, C.c_uint64, P]),
    "sd_scene_device_bytes": (C.c_uint64, [P]),
    "sd_scene_destroy": (None, [P]),
    "sd_tc_tiles_launch": (C.c_int, [P, P, C.c_uint64]),
    "sd_tc_tiles_copy_out": (C.c_int, [P, P, P, C.c_uint64]),
    "sd_tc_tiles_poll": (C.c_int, [P]),
    "sd_tc_tiles_finish": (C.c_int, [P, P, C.c_uint64]),
    "sd_tc_tiles": (C.c_int, [P, P, C.c_uint64, P]),
    "sd_ctx_set_graphs": (C.c_int, [P, C.c_int]),
    "sd_ctx_reserve": (C.c_int, [P, C.c_uint64]),
    "sd_ctx_set_tile_shape": (C.c_int, [P, C.c_int32, C.c_int32, C.c_int32]),
    "sd_orbit_states": (C.c_int, [P, P, C.c_uint64, P, C.c_uint64, P]),
    "sd_to_db": (C.c_int, [P, P, C.c_uint64, C.c_float, P, P]),
    "sd_ctx_set_db_output": (C.c_int, [P, C.c_int32, C.c_float]),
    "sd_ctx_db_result": (C.c_int, [P, P, P]),
    "sd_debug_bounds": (C.c_int, [P, P]),
    "sd_slc_open": (C.c_int, [P, C.c_char_p, P]),
    "sd_slc_dims": (C.c_int, [P, P, P, P]),
    "sd_slc_close": (None, [P]),
    "sd_multilook": (C.c_int, [P, P, P, C.c_uint64, C.c_uint64, C.c_uint32, C.c_uint32, P, P]),
    "sd_to_ground_range": (C.c_int, [P, P, C.c_uint64, C.c_uint64, C.c_double, C.c_double, C.c_double, P,
                                     C.c_int32, C.c_double, C.c_double, P, P]),
    "sd_slc_read_burst_raw": (C.c_int, [P, P, C.c_uint64, C.c_uint64, P]),
    "sd_coreg_offsets": (C.c_int, [P, P, C.c_uint64, C.c_int64, C.c_uint64, C.c_uint64, C.c_uint64, C.c_double,
                                   C.c_double, C.c_double, P, C.c_uint64, C.c_int64, C.c_double, C.c_double,
                                   C.c_double, C.c_uint64, P]),
    "sd_resample_secondary": (C.c_int, [P, P, C.c_uint64, C.c_uint64, C.c_uint64, C.c_uint64, P, P, P]),
    "sd_form_interferogram": (C.c_int, [P, P, P, C.c_uint64, C.c_uint64, C.c_uint64, C.c_double, C.c_double,
                                        C.c_double, P, C.c_uint64, C.c_int64, P, C.c_uint64, C.c_double,
                                        C.c_uint32, C.c_uint32, P, P]),
    "sd_deramp_subswath": (C.c_int, [P, P, C.c_uint64, C.c_uint64, C.c_uint64, C.c_double, C.c_double,
                                     C.c_double, P, C.c_uint64, C.c_int64, C.c_int32, P]),
    "sd_downsample_2x": (C.c_int, [P, P, C.c_uint64, C.c_uint64, P]),
    "sd_write_cog": (C.c_int, [P, C.c_char_p, P, C.c_uint64, C.c_uint64, P, C.c_int32, C.c_int32, C.c_uint32]),
    "sd_measure_fp64_peak": (C.c_int, [P, C.c_int32, P]),
    "sd_cr_sincos": (C.c_int, [P, P, C.c_uint64, P, P]),
    "sd_measure_fp32_peak": (C.c_int, [P, C.c_int32, P]),
}


def lib():
    """Load (and declare) the library; raises if it has not been built."""
    global _lib
    with _lock:
        if _lib is None:
            if not os.path.exists(LIB_PATH):
                raise RuntimeError(
                    f"{LIB_PATH} is missing: build it with `python -m sardine_b200.build` "
                    "(there is no CPU fallback)")
            L = C.CDLL(LIB_PATH)
            for name, (res, args) in _SIGS.items():
                fn = getattr(L, name)
                fn.restype = res
                fn.argtypes = args
            if L.sd_abi_version() != 1:
                raise RuntimeError("libsardine_b200.so ABI version mismatch")
            _lib = L
    return _lib


def exported_symbols():
    return list(_SIGS)


class Context:
    """One CUDA stream + scratch pool (sd_ctx).  Not thread-safe."""

    def __init__(self, device: int = 0):
        h = C.c_void_p()
        rc = lib().sd_ctx_create(device, C.byref(h))
        if rc != 0:
            raise RuntimeError(f"sd_ctx_create(device={device}) failed with status {rc} "
                               "(no usable CUDA device?)")
        self.handle = h
        self.device = device

    def close(self):
        if self.handle:
            lib().sd_ctx_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def launches(self) -> int:
        return int(lib().sd_kernel_launches(self.handle))

    @property
    def stream_ptr(self) -> int:
        return int(lib().sd_ctx_stream(self.handle) or 0)

    def set_timing(self, on: bool) -> None:
        """Bracket every kernel launch with CUDA events on the context's stream."""
        lib().sd_ctx_set_timing(self.handle, int(on))

    def kernel_times(self) -> dict:
        """{kernel name: (total ms, launches)} accumulated since set_timing(True)."""
        n = C.c_uint64()
        lib().sd_ctx_kernel_times(self.handle, None, 0, None, None, 0, C.byref(n))
        m = int(n.value)
        if m == 0:
            return {}
        names = C.create_string_buffer(64 * m + 64)
        ms = (C.c_double * m)()
        cnt = (C.c_uint64 * m)()
        lib().sd_ctx_kernel_times(self.handle, names, len(names), ms, cnt, m, C.byref(n))
        keys = names.value.decode().split("\n")[:m]
        return {k: (ms[i], int(cnt[i])) for i, k in enumerate(keys)}

    def last_error(self) -> str:
        s = lib().sd_last_error(self.handle)
        return s.decode("utf-8", "replace") if s else ""


_default = {}


def default_context(device: int = 0) -> Context:
    ctx = _default.get(device)
    if ctx is None:
        ctx = Context(device)
        _default[device] = ctx
    return ctx
