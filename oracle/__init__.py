"""ctypes binding of the CPU oracle (oracle/sardine_oracle.cpp).

TEST INFRASTRUCTURE ONLY: imported by tests/, by __graft_entry__.smoke() to
check its results, and by bench.py for the CPU-baseline leg.  The product package
never imports this module.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from typing import Sequence

import numpy as np

from sardine_b200 import _abi
from sardine_b200 import types as T

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "libsardine_oracle.so")
_lib = None


def build() -> str:
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        _lib = C.CDLL(_LIB_PATH)
        _declare(_lib)
    return _lib


def _declare(L):
    P = C.c_void_p
    d, f, i32, i64, u64 = C.c_double, C.c_float, C.c_int32, C.c_int64, C.c_uint64
    sig = {
        "orc_set_threads": (None, [C.c_int]),
        "orc_set_libm": (None, [C.c_int]),
        "orc_get_libm": (C.c_int, []),
        "orc_cr_sincos": (None, [P, C.c_uint64, P, P]),
        "orc_get_threads": (C.c_int, []),
        "orc_interpolate_orbit_and_accel": (C.c_int, [P, u64, i64, P, P, P]),
        "orc_solve_zero_doppler": (C.c_int, [P, P, u64, i64, u64, d, P, P, P]),
        "orc_geodetic_to_ecef": (None, [d, d, d, P]),
        "orc_utm_lonlat_to_xy": (None, [C.c_int, C.c_int, d, d, P, P]),
        "orc_utm_xy_to_lonlat": (None, [C.c_int, C.c_int, d, d, P, P]),
        "orc_project_row": (None, [C.c_int, C.c_int, d, d, d, u64, u64, P, P]),
        "orc_bilinear_sample": (f, [P, u64, u64, d, d]),
        "orc_bicubic_sample": (f, [P, u64, u64, d, d]),
        "orc_lanczos_sample": (f, [P, u64, u64, d, d]),
        "orc_keys_weight": (d, [d]),
        "orc_lanczos_weight": (d, [d]),
        "orc_flat_cell_area": (d, [d, d, d]),
        "orc_terrain_geometry": (C.c_int, [d, d, d, d, d, d, P, P, d, d, P, P]),
        "orc_geoid_undulation": (d, [P, d, d]),
        "orc_dem_elevation": (C.c_int, [P, d, d, P]),
        "orc_guess_azimuth_time": (i64, [P, u64, d]),
        "orc_tc_output_grid": (C.c_int, [P, P, P]),
        "orc_terrain_correction": (C.c_int, [P, P, P, P, P, u64, P, u64, u64, P, P, P, P, P, P]),
        "orc_terrain_correction_grid": (C.c_int, [P, P, P, P, P, u64, P, C.c_double, C.c_double, u64,
                                                  u64, P, P, P, P, P]),
        "orc_compute_overlap_lines": (C.c_int, [P, P, d, u64, P]),
        "orc_deburst_plan": (C.c_int, [P, P, u64, u64, P, P, P, P, P]),
        "orc_deburst_subswath": (C.c_int, [P, u64, u64, P, P, u64, P]),
        "orc_apply_calibration": (C.c_int, [P, u64, u64, u64, P, u64, P, u64, P, u64, P, P, P, P]),
        "orc_merge_plan": (C.c_int, [i32, P, P, P, P, P, P]),
        "orc_merge_subswaths": (C.c_int, [i32, P, P, P, P, P, P, P, P, P, P, P, P]),
        "orc_speckle": (C.c_int, [P, u64, u64, u64, C.c_int, u64, f, f, P]),
        "orc_to_db_inplace": (C.c_int, [P, u64, f, P, P]),
        "orc_db_stats": (None, [P, u64, P]),
        "orc_downsample_2x": (None, [P, u64, u64, P]),
        "orc_write_cog": (C.c_int, [C.c_char_p, P, u64, u64, P, C.c_int, C.c_int, C.c_uint32]),
        "orc_slc_read": (C.c_int, [C.c_char_p, u64, u64, P, P, P]),
        "orc_multilook": (C.c_int, [P, P, u64, u64, C.c_uint32, C.c_uint32, P, P]),
        "orc_to_ground_range": (C.c_int, [P, u64, u64, d, d, d, P, C.c_int32, d, d, P, P]),
        "orc_deramp": (C.c_int, [P, u64, u64, u64, d, d, d, P, u64, i64, P, P]),
        "orc_fit_poly6": (C.c_int, [P, u64, C.c_int, P, P]),
        "orc_coreg_offsets": (C.c_int, [P, u64, i64, u64, u64, u64, d, d, d, P, u64, i64, d, d, d, u64, P, P, P, P]),
        "orc_resample_secondary": (C.c_int, [P, u64, u64, u64, u64, P, P, P]),
        "orc_ecef_from_slant_range_doppler": (C.c_int, [P, P, d, u64, d, P]),
        "orc_form_interferogram": (C.c_int, [P, P, u64, u64, u64, d, d, d, P, u64, i64, P, u64, d, u64, u64, P,
                                             P]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args


class OracleError(RuntimeError):
    def __init__(self, code: int, what: str):
        super().__init__(f"{what}: status {code}")
        self.code = code


def _check(code: int, what: str):
    if code != 0:
        raise OracleError(code, what)


def _a(x):
    return C.cast(x, C.c_void_p) if x is not None else None


def set_threads(n: int) -> None:
    lib().orc_set_threads(n)


class libm:
    """Context manager selecting the oracle's libm for the sines and cosines
    of geodetic_to_ecef and the forward UTM projection: "glibc" (the platform
    libm, as the reference calls it; the default) or "cr" (correctly rounded
    sin/cos: the reference on a platform whose libm rounds correctly)."""

    def __init__(self, kind: str):
        if kind not in ("glibc", "cr"):
            raise ValueError(kind)
        self.kind = kind

    def __enter__(self):
        self.prev = lib().orc_get_libm()
        lib().orc_set_libm(1 if self.kind == "cr" else 0)
        return self

    def __exit__(self, *exc):
        lib().orc_set_libm(self.prev)
        return False


def cr_sincos(x):
    """Correctly rounded sin and cos of a float64 array."""
    x = np.ascontiguousarray(x, dtype=np.float64)
    s = np.empty_like(x)
    c = np.empty_like(x)
    lib().orc_cr_sincos(x.ctypes.data, x.size, s.ctypes.data, c.ctypes.data)
    return s, c


def threads() -> int:
    return lib().orc_get_threads()


# ── geometry primitives ────────────────────────────────────────────────────
def interpolate_orbit_and_accel(orbit: T.OrbitData, t_us: int):
    svs = orbit.to_c()
    p, v, a = (C.c_double * 3)(), (C.c_double * 3)(), (C.c_double * 3)()
    rc = lib().orc_interpolate_orbit_and_accel(svs, len(orbit.times_us), int(t_us), p, v, a)
    return rc, np.array(p[:]), np.array(v[:]), np.array(a[:])


def solve_zero_doppler(target, orbit: T.OrbitData, guess_us: int, max_iter=10, tol=1e-6):
    tg = (C.c_double * 3)(*[float(x) for x in target])
    svs = orbit.to_c()
    t, it, res = C.c_int64(), C.c_int32(), C.c_double()
    st = lib().orc_solve_zero_doppler(tg, svs, len(orbit.times_us), int(guess_us), max_iter, tol,
                                      C.byref(t), C.byref(it), C.byref(res))
    return st, t.value, it.value, res.value


def geodetic_to_ecef(lat, lon, h):
    o = (C.c_double * 3)()
    lib().orc_geodetic_to_ecef(lat, lon, h, o)
    return np.array(o[:])


def utm_lonlat_to_xy(zone, south, lon, lat):
    x, y = C.c_double(), C.c_double()
    lib().orc_utm_lonlat_to_xy(zone, int(south), lon, lat, C.byref(x), C.byref(y))
    return x.value, y.value


def utm_xy_to_lonlat(zone, south, x, y):
    lo, la = C.c_double(), C.c_double()
    lib().orc_utm_xy_to_lonlat(zone, int(south), x, y, C.byref(lo), C.byref(la))
    return lo.value, la.value


def project_row(zone, south, y, x_start, x_step, n_cols, n_anchors):
    lon = np.zeros(n_cols)
    lat = np.zeros(n_cols)
    lib().orc_project_row(zone, int(south), y, x_start, x_step, n_cols, n_anchors,
                          lon.ctypes.data, lat.ctypes.data)
    return lon, lat


def sample(kind: int, data: np.ndarray, line: float, samp: float) -> float:
    data = np.ascontiguousarray(data, dtype=np.float32)
    fn = {_abi.RESAMPLE_BILINEAR: lib().orc_bilinear_sample,
          _abi.RESAMPLE_BICUBIC: lib().orc_bicubic_sample,
          _abi.RESAMPLE_LANCZOS3: lib().orc_lanczos_sample}[kind]
    return fn(data.ctypes.data, data.shape[0], data.shape[1], line, samp)


def keys_weight(t):
    return lib().orc_keys_weight(t)


def lanczos_weight(x):
    return lib().orc_lanczos_weight(x)


def flat_cell_area(lat, lon, sp):
    return lib().orc_flat_cell_area(lat, lon, sp)


GEOM_VALID, GEOM_FORESHORTENING, GEOM_LAYOVER, GEOM_SHADOW = 0, 1, 2, 3


def terrain_geometry(lat, lon, he, hw, hn, hs, sat, target, sp, flat_area=None):
    if flat_area is None:
        flat_area = flat_cell_area(lat, lon, sp)
    s = (C.c_double * 3)(*sat)
    t = (C.c_double * 3)(*target)
    w, cl = C.c_double(float("nan")), C.c_double(float("nan"))
    g = lib().orc_terrain_geometry(lat, lon, he, hw, hn, hs, s, t, sp, flat_area, C.byref(w),
                                   C.byref(cl))
    return g, w.value, cl.value


def geoid_undulation(model: T.GeoidModel, lat, lon):
    keep = T._Keep()
    g = model.to_c(keep)
    return lib().orc_geoid_undulation(C.byref(g), lat, lon)


def dem_elevation(dem: T.DemGrid, lat, lon):
    d = dem.to_c()
    h = C.c_float()
    rc = lib().orc_dem_elevation(C.byref(d), lat, lon, C.byref(h))
    return rc, h.value


def guess_azimuth_time(points: Sequence[T.GeolocationGridPoint], lat):
    g = T.grid_to_c(points)
    return lib().orc_guess_azimuth_time(g, len(points), lat)


# ── hot-path functions ─────────────────────────────────────────────────────
def tc_output_grid(scene: T.SceneMetadata, config: T.TerrainCorrectionConfig, anchors=256):
    keep = T._Keep()
    sc = scene_to_c = T.scene_to_c(scene, keep)
    cfg = config.to_c(anchors)
    info = _abi.GeocodedInfo()
    rc = lib().orc_tc_output_grid(C.byref(sc), C.byref(cfg), C.byref(info))
    return rc, info


def terrain_correction(merged: T.MergedSigma0, scene: T.SceneMetadata, dem: T.DemGrid, grids,
                       config: T.TerrainCorrectionConfig, anchors: int = 256, row_begin: int = 0,
                       row_end: int = 0, return_times: bool = False):
    """terrain_correction (terrain_correction.rs:1245-1836) on rows
    [row_begin, row_end) (row_end 0 = all)."""
    keep = T._Keep()
    img = merged.to_c()
    sc = T.scene_to_c(scene, keep)
    d = dem.to_c()
    geo = config.geoid.to_c(keep)
    pts = T.pick_lut_grid(grids)
    g = T.grid_to_c(pts)
    cfg = config.to_c(anchors)
    info = _abi.GeocodedInfo()
    rc = lib().orc_tc_output_grid(C.byref(sc), C.byref(cfg), C.byref(info))
    if rc != 0 and len(pts) > 0 and scene.sub_swaths:
        raise OracleError(rc, "tc_output_grid")
    rows, cols = int(info.rows), int(info.cols)
    rb = row_begin
    re_ = row_end if row_end else rows
    nr = max(0, re_ - rb)
    data = np.empty((nr, cols), np.float32)
    cos = np.empty((nr, cols), np.float32) if config.compute_lia else None
    mask = np.empty((nr, cols), np.uint8) if config.compute_lia else None
    t_us = np.empty((nr, cols), np.int64) if return_times else None
    iters = np.empty((nr, cols), np.uint8) if return_times else None
    rc = lib().orc_terrain_correction(
        C.byref(img), C.byref(sc), C.byref(d), C.byref(geo), g, len(pts), C.byref(cfg), rb, re_,
        data.ctypes.data, cos.ctypes.data if cos is not None else None,
        mask.ctypes.data if mask is not None else None,
        t_us.ctypes.data if t_us is not None else None,
        iters.ctypes.data if iters is not None else None, C.byref(info))
    _check(rc, "terrain_correction")
    out = T.GeocodedImage.from_info(info, config.crs, data, cos, mask)
    if return_times:
        return out, t_us, iters
    return out


def terrain_correction_grid(merged: T.MergedSigma0, scene: T.SceneMetadata, dem: T.DemGrid, grids,
                            config: T.TerrainCorrectionConfig, origin_x: float, origin_y: float,
                            rows: int, cols: int, anchors: int = 256, return_times: bool = False):
    """terrain_correction onto an explicit output grid: west edge origin_x,
    north edge origin_y (config CRS units), rows x cols at the config spacing."""
    keep = T._Keep()
    img = merged.to_c()
    sc = T.scene_to_c(scene, keep)
    d = dem.to_c()
    geo = config.geoid.to_c(keep)
    pts = T.pick_lut_grid(grids)
    g = T.grid_to_c(pts)
    cfg = config.to_c(anchors)
    info = _abi.GeocodedInfo()
    data = np.empty((rows, cols), np.float32)
    cos = np.empty((rows, cols), np.float32) if config.compute_lia else None
    mask = np.empty((rows, cols), np.uint8) if config.compute_lia else None
    t_us = np.empty((rows, cols), np.int64) if return_times else None
    rc = lib().orc_terrain_correction_grid(
        C.byref(img), C.byref(sc), C.byref(d), C.byref(geo), g, len(pts), C.byref(cfg),
        float(origin_x), float(origin_y), rows, cols, data.ctypes.data,
        cos.ctypes.data if cos is not None else None, mask.ctypes.data if mask is not None else None,
        t_us.ctypes.data if t_us is not None else None, C.byref(info))
    _check(rc, "terrain_correction_grid")
    out = T.GeocodedImage.from_info(info, config.crs, data, cos, mask)
    if return_times:
        return out, t_us
    return out


def compute_overlap_lines(bk: T.BurstEntry, bk1: T.BurstEntry, ati: float, lps: int):
    a, b = bk.to_c(), bk1.to_c()
    ov = C.c_int64()
    rc = lib().orc_compute_overlap_lines(C.byref(a), C.byref(b), ati, lps, C.byref(ov))
    return rc, ov.value


def deburst_subswath(slc_iq: np.ndarray, sw: T.SubSwathMetadata, bursts) -> T.DeburstArray:
    slc_iq = np.ascontiguousarray(slc_iq, dtype=np.int16)
    h, w = slc_iq.shape[0], slc_iq.shape[1]
    swc = sw.to_c()
    bc = T.bursts_to_c(bursts)
    lines, samples, off = C.c_uint64(), C.c_uint64(), C.c_uint64()
    rc = lib().orc_deburst_plan(C.byref(swc), bc, len(bursts), h, C.byref(lines), C.byref(samples),
                                C.byref(off), None, None)
    _check(rc, "deburst_plan")
    out = np.empty((lines.value, samples.value, 2), np.int16)
    rc = lib().orc_deburst_subswath(slc_iq.ctypes.data, w, h, C.byref(swc), bc, len(bursts),
                                    out.ctypes.data)
    _check(rc, "deburst_subswath")
    return T.DeburstArray(out, lines.value, samples.value, off.value)


def apply_calibration(deb: T.DeburstArray, cal: T.SwathCalibration, noise: T.SwathNoise,
                      tiff_line_origin: int) -> T.Sigma0Array:
    keep = T._Keep()
    cv = T.lut_vectors_to_c(cal.vectors, keep, "sigma_nought")
    nv = T.lut_vectors_to_c(noise.range_vectors, keep, "noise_range_lut")
    na = T.noise_azimuth_to_c(noise, keep)
    iq = np.ascontiguousarray(deb.data, dtype=np.int16)
    out = np.empty((deb.lines, deb.samples), np.float32)
    nesz = np.empty((deb.lines, deb.samples), np.float32)
    cg, ng = C.c_uint32(), C.c_uint32()
    rc = lib().orc_apply_calibration(iq.ctypes.data, deb.lines, deb.samples,
                                     deb.valid_sample_offset, cv, len(cal.vectors), nv,
                                     len(noise.range_vectors), C.byref(na), tiff_line_origin,
                                     out.ctypes.data, nesz.ctypes.data, C.byref(cg), C.byref(ng))
    _check(rc, "apply_calibration")
    return T.Sigma0Array(out, deb.lines, deb.samples, deb.valid_sample_offset, cg.value, ng.value,
                         nesz)


def merge_subswaths(inputs: Sequence[T.SwathInput]) -> T.MergedSigma0:
    n = len(inputs)
    arrs = [(np.ascontiguousarray(i.sigma0.data, np.float32),
             np.ascontiguousarray(i.sigma0.nesz, np.float32)) for i in inputs]
    sig = (C.c_void_p * max(1, n))(*[a[0].ctypes.data for a in arrs])
    nes = (C.c_void_p * max(1, n))(*[a[1].ctypes.data for a in arrs])
    u64 = lambda vals: (C.c_uint64 * max(1, n))(*vals)
    lines = u64([i.sigma0.lines for i in inputs])
    samples = u64([i.sigma0.samples for i in inputs])
    voff = u64([i.sigma0.valid_sample_offset for i in inputs])
    cg = (C.c_uint32 * max(1, n))(*[i.sigma0.cal_lut_extrapolation_gap_px for i in inputs])
    ng = (C.c_uint32 * max(1, n))(*[i.sigma0.noise_lut_extrapolation_gap_px for i in inputs])
    sw = (_abi.SubSwath * max(1, n))(*[i.swath.to_c() for i in inputs])
    az = (C.c_int64 * max(1, n))(*[int(i.azimuth_start_time_us) for i in inputs])
    info = _abi.MergedInfo()
    rc = lib().orc_merge_subswaths(n, sig, nes, lines, samples, voff, cg, ng, sw, az, None, None,
                                   C.byref(info))
    _check(rc, "merge_subswaths")
    out = np.empty((info.lines, info.samples), np.float32)
    onz = np.empty((info.lines, info.samples), np.float32)
    rc = lib().orc_merge_subswaths(n, sig, nes, lines, samples, voff, cg, ng, sw, az,
                                   out.ctypes.data, onz.ctypes.data, C.byref(info))
    _check(rc, "merge_subswaths")
    return T.MergedSigma0(out, int(info.lines), int(info.samples), info.near_slant_range_time_s,
                          info.range_pixel_spacing_s, info.range_pixel_spacing_m,
                          info.cal_lut_extrapolation_gap_px, info.noise_lut_extrapolation_gap_px,
                          onz, info.azimuth_start_time_us), info


def apply_speckle_filter(data: np.ndarray, cols: int, rows: int, flt: T.SpeckleFilter):
    data = np.ascontiguousarray(data, dtype=np.float32).reshape(-1)
    out = np.empty_like(data)
    rc = lib().orc_speckle(data.ctypes.data, data.size, cols, rows, flt.kind, flt.window, flt.enl,
                           flt.damping, out.ctypes.data)
    _check(rc, "apply_speckle_filter")
    return out


# ── output path (oracle/export_oracle.cpp) ───────────────────────────────────
def to_db_inplace(data: np.ndarray, noise_floor_linear: float):
    """to_db_inplace (export.rs:59-99) on a contiguous float32 array:
    returns (converted, noise_masked); raises for a negative floor."""
    assert data.dtype == np.float32 and data.flags.c_contiguous
    cv, nm = C.c_uint64(), C.c_uint64()
    rc = lib().orc_to_db_inplace(data.ctypes.data, data.size, float(noise_floor_linear), C.byref(cv),
                                 C.byref(nm))
    _check(rc, "to_db_inplace")
    return int(cv.value), int(nm.value)


def db_stats(data: np.ndarray):
    """compute_db_stats (run.rs:63-97): (min, max, mean, median)."""
    data = np.ascontiguousarray(data, dtype=np.float32).reshape(-1)
    out = (C.c_float * 4)()
    lib().orc_db_stats(data.ctypes.data, data.size, out)
    return tuple(float(x) for x in out)


def downsample_2x(src: np.ndarray, cols: int, rows: int) -> np.ndarray:
    """downsample_2x (export.rs:362-392)."""
    src = np.ascontiguousarray(src, dtype=np.float32).reshape(-1)
    out = np.empty(((rows + 1) // 2, (cols + 1) // 2), np.float32)
    lib().orc_downsample_2x(src.ctypes.data, cols, rows, out.ctypes.data)
    return out


def write_cog(path: str, data: np.ndarray, cols: int, rows: int, geotransform, crs: T.OutputCrs,
              tile_size: int = 512) -> int:
    """write_cog_with_crs (export.rs:329-760); returns the status code."""
    data = np.ascontiguousarray(data, dtype=np.float32).reshape(-1)
    gt = (C.c_double * 6)(*[float(x) for x in geotransform])
    return int(lib().orc_write_cog(os.fsencode(path), data.ctypes.data, cols, rows, gt, int(crs.kind),
                                   int(crs.zone), int(tile_size)))


def slc_read(path: str, first_line: int = 0, line_count: int = 0, read: bool = True):
    """SlcReader::open + read_burst_raw (slc_reader.rs:268-583): returns
    (status, width, height, rows as int16 [line_count, width, 2] or None)."""
    w, h = C.c_uint32(), C.c_uint32()
    rc = lib().orc_slc_read(os.fsencode(path), 0, 0, None, C.byref(w), C.byref(h))
    if rc != 0 or not read:
        return rc, int(w.value), int(h.value), None
    out = np.empty((line_count, w.value, 2), np.int16)
    rc = lib().orc_slc_read(os.fsencode(path), first_line, line_count, out.ctypes.data, None, None)
    return rc, int(w.value), int(h.value), (out if rc == 0 else None)


def multilook(data: np.ndarray, nesz: np.ndarray, lines: int, samples: int, range_looks: int, azimuth_looks: int):
    """The boxcar of apply_multilook (scene_prep.rs:1060-1160): (status, data, nesz)."""
    d = np.ascontiguousarray(data, dtype=np.float32).reshape(-1)
    n = np.ascontiguousarray(nesz, dtype=np.float32).reshape(-1)
    ol, os_ = (lines // azimuth_looks if azimuth_looks else 0), (samples // range_looks if range_looks else 0)
    od = np.empty((max(ol, 1), max(os_, 1)), np.float32)
    on = np.empty_like(od)
    rc = lib().orc_multilook(d.ctypes.data, n.ctypes.data, lines, samples, range_looks, azimuth_looks,
                             od.ctypes.data, on.ctypes.data)
    return rc, (od if rc == 0 else None), (on if rc == 0 else None)


def to_ground_range(merged: T.MergedSigma0, grids, target_spacing_m: float, azimuth_pixel_spacing_m: float):
    """to_ground_range (ground_range.rs:303-427): (status, GroundRangeImage or None)."""
    from sardine_b200 import _grd_grids
    d = np.ascontiguousarray(merged.data, dtype=np.float32).reshape(-1)
    arr, keep = _grd_grids(grids)
    info = _abi.GrdInfo()
    args = (merged.lines, merged.samples, float(merged.near_slant_range_time_s), float(merged.range_pixel_spacing_s),
            float(merged.range_pixel_spacing_m), arr, len(grids), float(target_spacing_m),
            float(azimuth_pixel_spacing_m))
    rc = lib().orc_to_ground_range(d.ctypes.data, *args, None, C.byref(info))
    if rc != 0:
        return rc, None
    out = np.empty((int(info.lines), int(info.samples)), np.float32)
    rc = lib().orc_to_ground_range(d.ctypes.data, *args, out.ctypes.data if out.size else None, C.byref(info))
    return rc, T.GroundRangeImage(out, int(info.lines), int(info.samples), info.range_pixel_spacing_m,
                                  info.azimuth_pixel_spacing_m, int(info.range_looks), int(info.azimuth_looks))


def deramp_subswath(deburst: T.DeburstArray, swath: T.SubSwathMetadata, burst_start_us: int):
    """deramp_subswath (insar/deramp.rs:114-210): (status, Deramped or None);
    for AzimuthTimeBeforeDcEstimates the status comes with the failing line's
    relative time in Deramped.data."""
    from sardine_b200 import _dc_to_c
    est = list(swath.dc_estimates or [])
    iq = np.ascontiguousarray(deburst.data, dtype=np.int16).reshape(-1)
    lines, samples = int(deburst.lines), int(deburst.samples)
    out = np.empty((lines, samples, 2), np.float32)
    bad = C.c_double(0.0)
    rc = lib().orc_deramp(iq.ctypes.data, lines, samples, int(deburst.valid_sample_offset),
                          float(swath.slant_range_time_s), float(swath.range_pixel_spacing_m),
                          float(swath.azimuth_time_interval_s), _dc_to_c(est), len(est), int(burst_start_us),
                          out.ctypes.data, C.byref(bad))
    if rc != 0:
        return rc, (bad.value if rc == _abi.SD_ERR_INSAR_AZIMUTH_TIME_BEFORE_DC else None)
    return rc, T.Deramped(out, lines, samples, int(deburst.valid_sample_offset))


def resample_secondary(ref_lines: int, ref_samples: int, poly: T.CoregPoly, secondary: T.Deramped):
    """resample_secondary (insar/coreg.rs:230-264): Deramped."""
    sec = np.ascontiguousarray(secondary.data, dtype=np.float32).reshape(-1)
    out = np.empty((int(ref_lines), int(ref_samples), 2), np.float32)
    az = (C.c_double * 6)(*[float(v) for v in poly.az])
    rg = (C.c_double * 6)(*[float(v) for v in poly.rg])
    _check(lib().orc_resample_secondary(sec.ctypes.data, int(secondary.lines), int(secondary.samples),
                                        int(ref_lines), int(ref_samples), az, rg, out.ctypes.data),
           "resample_secondary")
    return T.Deramped(out, int(ref_lines), int(ref_samples), int(secondary.valid_sample_offset))


def ecef_from_slant_range_doppler(sat_pos, sat_vel, range_m: float, max_iter: int, tol_m: float):
    """ecef_from_slant_range_doppler (insar/coreg.rs:280-362): the point, or None."""
    out = (C.c_double * 3)()
    rc = lib().orc_ecef_from_slant_range_doppler((C.c_double * 3)(*sat_pos), (C.c_double * 3)(*sat_vel),
                                                 float(range_m), int(max_iter), float(tol_m), out)
    return None if rc else (out[0], out[1], out[2])


def form_interferogram(coreg: T.Coregistered, ref_swath: T.SubSwathMetadata, ref_orbit: T.OrbitData,
                       ref_first_us: int, sec_orbit: T.OrbitData, wavelength_m: float,
                       cfg: T.InterferogramConfig = None):
    """form_interferogram (insar/interferogram.rs:165-398): (status, Interferogram or None)."""
    cfg = cfg or T.InterferogramConfig()
    r, s_ = coreg.ref_data, coreg.secondary_resampled
    ref = np.ascontiguousarray(r.data, dtype=np.float32).reshape(-1)
    sec = np.ascontiguousarray(s_.data, dtype=np.float32).reshape(-1)
    lines, samples = int(r.lines), int(r.samples)
    coh = np.empty((lines, samples), np.float32)
    ph = np.empty((lines, samples), np.float32) if cfg.compute_phase else None
    rc = lib().orc_form_interferogram(ref.ctypes.data, sec.ctypes.data, lines, samples, int(r.valid_sample_offset),
                                      float(ref_swath.slant_range_time_s), float(ref_swath.range_pixel_spacing_m),
                                      float(ref_swath.azimuth_time_interval_s), ref_orbit.to_c(),
                                      len(ref_orbit.times_us), int(ref_first_us), sec_orbit.to_c(),
                                      len(sec_orbit.times_us), float(wavelength_m), int(cfg.az_looks),
                                      int(cfg.rg_looks), coh.ctypes.data, None if ph is None else ph.ctypes.data)
    if rc:
        return rc, None
    return rc, T.Interferogram(coh, ph, lines, samples, int(cfg.az_looks), int(cfg.rg_looks))


def fit_poly6(pts, which: int):
    """fit_poly6 (insar/coreg.rs:478-517) of column `which` (2: dl, 3: dc) of
    (l, c, dl, dc) points: (status, coefficients, residual rms)."""
    a = np.ascontiguousarray(pts, dtype=np.float64).reshape(-1)
    coef, rms = (C.c_double * 6)(), C.c_double()
    rc = lib().orc_fit_poly6(a.ctypes.data, a.size // 4, which, coef, C.byref(rms))
    return rc, list(coef), rms.value


def compute_coreg_offsets(ref_swath, ref_orbit, ref_first_us, ref_deburst, sec_swath, sec_orbit, sec_first_us):
    """compute_coreg_offsets (insar/coreg.rs:128-223): (status, CoregResult or None)."""
    rc, res, _ = _coreg_offsets(ref_swath, ref_orbit, ref_first_us, ref_deburst, sec_swath, sec_orbit, sec_first_us)
    return rc, res


def coreg_n_valid(ref_swath, ref_orbit, ref_first_us, ref_deburst, sec_swath, sec_orbit, sec_first_us):
    """(status, number of converged grid points), the count also on the
    grid-too-small error, which carries it (coreg.rs:207-208)."""
    rc, _, nv = _coreg_offsets(ref_swath, ref_orbit, ref_first_us, ref_deburst, sec_swath, sec_orbit, sec_first_us)
    return rc, nv


def _coreg_offsets(ref_swath, ref_orbit, ref_first_us, ref_deburst, sec_swath, sec_orbit, sec_first_us):
    az, rg, rms, nv = (C.c_double * 6)(), (C.c_double * 6)(), C.c_double(), C.c_uint64()
    rc = lib().orc_coreg_offsets(ref_orbit.to_c(), len(ref_orbit.times_us), int(ref_first_us), int(ref_deburst.lines),
                                 int(ref_deburst.samples), int(ref_deburst.valid_sample_offset),
                                 float(ref_swath.azimuth_time_interval_s), float(ref_swath.slant_range_time_s),
                                 float(ref_swath.range_pixel_spacing_m), sec_orbit.to_c(), len(sec_orbit.times_us),
                                 int(sec_first_us), float(sec_swath.azimuth_time_interval_s),
                                 float(sec_swath.slant_range_time_s), float(sec_swath.range_pixel_spacing_m),
                                 int(sec_swath.first_sample), az, rg, C.byref(rms), C.byref(nv))
    if rc:
        return rc, None, int(nv.value)
    return rc, T.CoregResult(T.CoregPoly(list(az), list(rg)), rms.value, int(nv.value)), int(nv.value)
