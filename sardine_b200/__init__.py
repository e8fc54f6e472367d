"""sardine_b200 — B200 (sm_100a) implementation of SARdine's hot path.

The functions here mirror the reference's Rust API for the path (same names,
argument meaning and error variants) and call the CUDA library through its
C ABI (include/sardine_b200.h):

==============================  ============================================
reference                       here
==============================  ============================================
terrain_correction              terrain_correction(merged, scene, dem, grids, config)
apply_calibration               apply_calibration(deburst, cal, noise, tiff_line_origin)
deburst_subswath                deburst_subswath(slc_iq, sw, bursts)
compute_overlap_lines           compute_overlap_lines(burst_k, burst_k1, ati_s, lines_per_burst)
merge_subswaths                 merge_subswaths(inputs)
prepare_merged_scene (core)     calibrate_deburst_merge(swaths)
apply_speckle_filter            apply_speckle_filter(data, cols, rows, filter)
SpeckleKernel                   SpeckleKernel / GpuSpeckleKernel
==============================  ============================================

Arrays may be numpy (host) or torch CUDA tensors (device resident); results
come back in the same kind of container as the main input.
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Any, List, Optional, Sequence

import numpy as np

from . import _abi
from . import types as T
from ._lib import Context, default_context, lib
from .types import (BoundingBox, BurstEntry, CalibrationVector, CoregPoly, CoregResult, Coregistered, DcEstimate, DeburstArray, Deramped, DemGrid,
                    GeocodedImage, GroundRangeImage, Interferogram, InterferogramConfig, GeoidModel, GeolocationGridPoint, MergedSigma0, NoiseAzimuthVector,
                    NoiseRangeVector, OrbitData, OutputCrs, Precision, ResamplingKernel, SceneMetadata,
                    Sigma0Array, SpeckleFilter, SubSwathMetadata, SwathCalibration, SwathInput,
                    SwathNoise, TerrainCorrectionConfig)

__all__ = [
    "terrain_correction", "apply_calibration", "deburst_subswath", "compute_overlap_lines",
    "merge_subswaths", "calibrate_deburst_merge", "apply_speckle_filter", "SpeckleKernel",
    "GpuSpeckleKernel", "SardineError", "TerrainCorrectionError", "SpeckleError",
    "CalibrationError", "DeburstError", "MergeError", "Context", "default_context",
    "tc_output_grid", "to_db_inplace", "write_cog_with_crs", "downsample_2x", "ExportError",
    "SlcReader", "SlcReadError", "apply_multilook", "to_ground_range", "GroundRangeError",
    "deramp_subswath", "InsarError", "resample_secondary", "form_interferogram",
    "compute_coreg_offsets",
] + [n for n in dir(T) if n[:1].isupper() and getattr(getattr(T, n), "__module__", "") == T.__name__]


# ── errors (one class per reference error enum; .kind = variant name) ──────
class SardineError(RuntimeError):
    def __init__(self, code: int, kind: str, message: str):
        super().__init__(f"{kind}: {message}" if message else kind)
        self.code = code
        self.kind = kind


class TerrainCorrectionError(SardineError):
    """terrain_correction.rs:45-67"""


class SpeckleError(SardineError):
    """speckle.rs:96-108"""


class CalibrationError(SardineError):
    """apply_calibration.rs:64-84"""


class DeburstError(SardineError):
    """deburst.rs:56-121"""


class MergeError(SardineError):
    """merge_subswaths.rs:62-81"""


class ExportError(SardineError):
    """export.rs:25-40"""


class SlcReadError(SardineError):
    """slc_reader.rs:66-98"""


class InsarError(SardineError):
    """insar/error.rs:7-80"""


class GroundRangeError(SardineError):
    """ground_range.rs:42-57"""


_KINDS = {
    _abi.SD_ERR_TC_ORBIT: (TerrainCorrectionError, "Orbit"),
    _abi.SD_ERR_TC_DEM: (TerrainCorrectionError, "Dem"),
    _abi.SD_ERR_TC_NO_GRID_POINTS: (TerrainCorrectionError, "NoGridPoints"),
    _abi.SD_ERR_TC_NO_SUBSWATHS: (TerrainCorrectionError, "NoSubSwaths"),
    _abi.SD_ERR_TC_CONFIG: (TerrainCorrectionError, "Config"),
    _abi.SD_ERR_TC_PROJECTION: (TerrainCorrectionError, "Projection"),
    _abi.SD_ERR_SPECKLE_DIMENSION_MISMATCH: (SpeckleError, "DimensionMismatch"),
    _abi.SD_ERR_SPECKLE_BAD_WINDOW: (SpeckleError, "BadWindow"),
    _abi.SD_ERR_SPECKLE_BAD_ENL: (SpeckleError, "BadEnl"),
    _abi.SD_ERR_SPECKLE_BAD_DAMPING: (SpeckleError, "BadDamping"),
    _abi.SD_ERR_CAL_NO_CALIBRATION_VECTORS: (CalibrationError, "NoCalibrationVectors"),
    _abi.SD_ERR_CAL_NO_NOISE_RANGE_VECTORS: (CalibrationError, "NoNoiseRangeVectors"),
    _abi.SD_ERR_CAL_LUT_RANGE_INSUFFICIENT: (CalibrationError, "LutRangeInsufficient"),
    _abi.SD_ERR_DEBURST_NO_BURSTS: (DeburstError, "NoBursts"),
    _abi.SD_ERR_DEBURST_BURST_COUNT_MISMATCH: (DeburstError, "BurstCountMismatch"),
    _abi.SD_ERR_DEBURST_TIFF_TOO_SMALL: (DeburstError, "TiffTooSmall"),
    _abi.SD_ERR_DEBURST_EMPTY_VALID_WINDOW: (DeburstError, "EmptyValidWindow"),
    _abi.SD_ERR_DEBURST_INVALID_OVERLAP: (DeburstError, "InvalidOverlap"),
    _abi.SD_ERR_DEBURST_IMPLAUSIBLE_OVERLAP: (DeburstError, "ImplausibleOverlap"),
    _abi.SD_ERR_MERGE_EMPTY_INPUTS: (MergeError, "EmptyInputs"),
    _abi.SD_ERR_MERGE_INCONSISTENT_PIXEL_SPACING: (MergeError, "InconsistentPixelSpacing"),
    _abi.SD_ERR_MERGE_EMPTY_SWATH: (MergeError, "EmptySwath"),
    _abi.SD_ERR_EXPORT_IO: (ExportError, "Io"),
    _abi.SD_ERR_EXPORT_INVALID_NOISE_FLOOR: (ExportError, "InvalidNoiseFloor"),
    _abi.SD_ERR_EXPORT_INVALID_GEOTRANSFORM: (ExportError, "InvalidGeotransform"),
    _abi.SD_ERR_EXPORT_INVALID_TILE_SIZE: (ExportError, "InvalidTileSize"),
    _abi.SD_ERR_SLC_IO: (SlcReadError, "Io"),
    _abi.SD_ERR_SLC_NOT_TIFF: (SlcReadError, "NotTiff"),
    _abi.SD_ERR_SLC_BIGTIFF: (SlcReadError, "BigTiff"),
    _abi.SD_ERR_SLC_MISSING_TAG: (SlcReadError, "MissingTag"),
    _abi.SD_ERR_SLC_UNSUPPORTED_FORMAT: (SlcReadError, "UnsupportedFormat"),
    _abi.SD_ERR_SLC_NON_CONTIGUOUS_STRIPS: (SlcReadError, "NonContiguousStrips"),
    _abi.SD_ERR_SLC_LINE_OUT_OF_BOUNDS: (SlcReadError, "LineOutOfBounds"),
    _abi.SD_ERR_GRD_NO_GRID_POINTS: (GroundRangeError, "NoGridPoints"),
    _abi.SD_ERR_GRD_EMPTY_IMAGE: (GroundRangeError, "EmptyImage"),
    _abi.SD_ERR_GRD_INVALID_SPACING: (GroundRangeError, "InvalidSpacing"),
    _abi.SD_ERR_GRD_INVALID_AZIMUTH_SPACING: (GroundRangeError, "InvalidAzimuthSpacing"),
    _abi.SD_ERR_GRD_INTERPOLATION_FAILED: (GroundRangeError, "InterpolationFailed"),
    _abi.SD_ERR_INSAR_NO_DC_ESTIMATES: (InsarError, "NoDcEstimates"),
    _abi.SD_ERR_INSAR_AZIMUTH_TIME_BEFORE_DC: (InsarError, "AzimuthTimeBeforeDcEstimates"),
    _abi.SD_ERR_INSAR_INVALID_WINDOW_SIZE: (InsarError, "InvalidWindowSize"),
    _abi.SD_ERR_INSAR_ORBIT: (InsarError, "Orbit"),
    _abi.SD_ERR_INSAR_COREG_GRID_TOO_SMALL: (InsarError, "CoregGridTooSmall"),
}


def _check(ctx: Context, rc: int, default_cls=SardineError):
    if rc == 0:
        return
    cls, kind = _KINDS.get(rc, (default_cls, {
        _abi.SD_ERR_INVALID_ARGUMENT: "InvalidArgument", _abi.SD_ERR_CUDA: "Cuda",
        _abi.SD_ERR_OUT_OF_MEMORY: "OutOfMemory", _abi.SD_ERR_INTERNAL: "Internal",
        _abi.SD_ERR_TIMEOUT: "Timeout", _abi.SD_ERR_BUSY: "Busy"}.get(rc, f"Status{rc}")))
    raise cls(rc, kind, ctx.last_error())


# ── containers ─────────────────────────────────────────────────────────────
def _is_torch_cuda(a) -> bool:
    return hasattr(a, "is_cuda") and bool(a.is_cuda)


def _empty_like_kind(ref, shape, dtype: str):
    if _is_torch_cuda(ref):
        import torch
        tdt = {"f4": torch.float32, "u1": torch.uint8, "i2": torch.int16, "i8": torch.int64}[dtype]
        return torch.empty(shape, dtype=tdt, device=ref.device)
    return np.empty(shape, dtype={"f4": np.float32, "u1": np.uint8, "i2": np.int16, "i8": np.int64}[dtype])


def _prep(a, dtype):
    """numpy arrays are made contiguous with the right dtype; torch tensors must already be."""
    if a is None:
        return None
    if isinstance(a, np.ndarray):
        return np.ascontiguousarray(a, dtype=dtype)
    return a.contiguous()


def _ctx(ctx: Optional[Context]) -> Context:
    return ctx if ctx is not None else default_context(int(os.environ.get("SARDINE_B200_DEVICE", "0")))


def _anchors_from_env() -> int:
    """SARDINE_TC_PROJECTOR_ANCHORS (terrain_correction.rs:1328-1351)."""
    s = os.environ.get("SARDINE_TC_PROJECTOR_ANCHORS")
    if s is None:
        return 256
    try:
        v = int(s)
        if v < 0:
            raise ValueError
    except ValueError:
        raise TerrainCorrectionError(_abi.SD_ERR_TC_CONFIG, "Config",
                                     f"SARDINE_TC_PROJECTOR_ANCHORS={s!r} is not a non-negative integer")
    return v


# ── terrain correction ─────────────────────────────────────────────────────
def tc_output_grid(scene: SceneMetadata, config: TerrainCorrectionConfig,
                   ctx: Optional[Context] = None) -> _abi.GeocodedInfo:
    ctx = _ctx(ctx)
    keep = T._Keep()
    sc = T.scene_to_c(scene, keep)
    cfg = config.to_c(256)
    info = _abi.GeocodedInfo()
    _check(ctx, lib().sd_tc_output_grid(ctx.handle, C.byref(sc), C.byref(cfg), C.byref(info)),
           TerrainCorrectionError)
    return info


def terrain_correction(merged: MergedSigma0, scene: SceneMetadata, dem: DemGrid, grids,
                       config: TerrainCorrectionConfig, ctx: Optional[Context] = None,
                       out=None, return_times: bool = False, row_range=None) -> GeocodedImage:
    """terrain_correction (terrain_correction.rs:1245-1836) on the GPU.

    `grids` is a sequence of (sub-swath id, geolocation points); the LUT uses
    IW2's points, else the first sub-swath's.  `out` may supply preallocated
    (data, cos_lia, mask) buffers of the output-grid shape.  With
    `return_times`, the result also carries the converged zero-Doppler time of
    every pixel (`azimuth_time_us`, int64 microseconds, INT64_MIN where none).
    `row_range=(r0, r1)` geocodes only those output rows (a row band: equal to
    the same rows of the whole grid; how one scene shards over GPUs)."""
    ctx = _ctx(ctx)
    keep = T._Keep()
    merged_data = _prep(merged.data, np.float32)
    nesz = _prep(merged.nesz, np.float32) if merged.nesz is not None else None
    img = _abi.RadarImage(T.ptr(merged_data), T.ptr(nesz), merged.lines, merged.samples,
                          int(merged.azimuth_start_time_us), merged.near_slant_range_time_s,
                          merged.range_pixel_spacing_m)
    sc = T.scene_to_c(scene, keep)
    dem_data = _prep(dem.data, np.float32)
    d = _abi.Dem(dem.kind, dem.utm_zone, int(dem.utm_south), 0, T.ptr(dem_data),
                 dem_data.shape[1], dem_data.shape[0], dem.origin_y, dem.origin_x, dem.pixel_size)
    geo = config.geoid.to_c(keep)
    pts = T.pick_lut_grid(grids)
    g = T.grid_to_c(pts)
    anchors = _anchors_from_env()
    cfg = config.to_c(anchors)
    info = _abi.GeocodedInfo()
    if len(pts) > 0 and config.pixel_spacing_deg > 0 and scene.sub_swaths:
        _check(ctx, lib().sd_tc_output_grid(ctx.handle, C.byref(sc), C.byref(cfg), C.byref(info)),
               TerrainCorrectionError)
    rows, cols = int(info.rows), int(info.cols)
    if row_range is not None:
        r0, r1 = int(row_range[0]), int(row_range[1] or rows)
        rows = max(0, min(r1, rows) - r0)
    if out is not None:
        data, cos, mask = out
    else:
        data = _empty_like_kind(merged_data, (rows, cols), "f4")
        cos = _empty_like_kind(merged_data, (rows, cols), "f4") if config.compute_lia else None
        mask = _empty_like_kind(merged_data, (rows, cols), "u1") if config.compute_lia else None
    times = _empty_like_kind(merged_data, (rows, cols), "i8") if return_times else None
    if row_range is not None:
        rc = lib().sd_terrain_correction_rows(ctx.handle, C.byref(img), C.byref(sc), C.byref(d), C.byref(geo),
                                              g, len(pts), C.byref(cfg), r0, r1, T.ptr(data), T.ptr(cos),
                                              T.ptr(mask), T.ptr(times), C.byref(info))
    elif return_times:
        rc = lib().sd_terrain_correction_with_times(
            ctx.handle, C.byref(img), C.byref(sc), C.byref(d), C.byref(geo), g, len(pts), C.byref(cfg),
            T.ptr(data), T.ptr(cos), T.ptr(mask), T.ptr(times), C.byref(info))
    else:
        rc = lib().sd_terrain_correction(ctx.handle, C.byref(img), C.byref(sc), C.byref(d), C.byref(geo),
                                         g, len(pts), C.byref(cfg), T.ptr(data), T.ptr(cos), T.ptr(mask),
                                         C.byref(info))
    _check(ctx, rc, TerrainCorrectionError)
    res = GeocodedImage.from_info(info, config.crs, data, cos, mask)
    res.azimuth_time_us = times
    return res


# ── deburst / calibration / merge ──────────────────────────────────────────
def compute_overlap_lines(burst_k: BurstEntry, burst_k1: BurstEntry, ati_s: float,
                          lines_per_burst: int, ctx: Optional[Context] = None) -> int:
    """compute_overlap_lines (deburst.rs:172-210)."""
    ctx = _ctx(ctx)
    a, b = burst_k.to_c(), burst_k1.to_c()
    ov = C.c_uint64()
    _check(ctx, lib().sd_compute_overlap_lines(ctx.handle, C.byref(a), C.byref(b), ati_s,
                                               lines_per_burst, C.byref(ov)), DeburstError)
    return int(ov.value)


def deburst_subswath(slc_iq, sw: SubSwathMetadata, bursts: Sequence[BurstEntry],
                     ctx: Optional[Context] = None) -> DeburstArray:
    """deburst_subswath (deburst.rs:230-344).  `slc_iq` is the measurement
    raster (tiff_height, tiff_width, 2) int16 — what BurstReader reads."""
    ctx = _ctx(ctx)
    slc_iq = _prep(slc_iq, np.int16)
    h, w = int(slc_iq.shape[0]), int(slc_iq.shape[1])
    swc = sw.to_c()
    bc = T.bursts_to_c(bursts)
    lines, samples, off = C.c_uint64(), C.c_uint64(), C.c_uint64()
    _check(ctx, lib().sd_deburst_plan(ctx.handle, C.byref(swc), bc, len(bursts), h, C.byref(lines),
                                      C.byref(samples), C.byref(off)), DeburstError)
    out = _empty_like_kind(slc_iq, (lines.value, samples.value, 2), "i2")
    _check(ctx, lib().sd_deburst_subswath(ctx.handle, T.ptr(slc_iq), w, h, C.byref(swc), bc,
                                          len(bursts), T.ptr(out)), DeburstError)
    return DeburstArray(out, int(lines.value), int(samples.value), int(off.value))


def apply_calibration(deburst: DeburstArray, cal: SwathCalibration, noise: SwathNoise,
                      tiff_line_origin: int, ctx: Optional[Context] = None, out=None) -> Sigma0Array:
    """apply_calibration (apply_calibration.rs:374-572).  `out` may supply
    preallocated (sigma0, nesz) buffers of shape (lines, samples)."""
    ctx = _ctx(ctx)
    keep = T._Keep()
    cv = T.lut_vectors_to_c(cal.vectors, keep, "sigma_nought")
    nv = T.lut_vectors_to_c(noise.range_vectors, keep, "noise_range_lut")
    na = T.noise_azimuth_to_c(noise, keep)
    iq = _prep(deburst.data, np.int16)
    if out is not None:
        out, nesz = out
    else:
        out = _empty_like_kind(iq, (deburst.lines, deburst.samples), "f4")
        nesz = _empty_like_kind(iq, (deburst.lines, deburst.samples), "f4")
    cg, ng = C.c_uint32(), C.c_uint32()
    rc = lib().sd_apply_calibration(ctx.handle, T.ptr(iq), deburst.lines, deburst.samples,
                                    deburst.valid_sample_offset, cv, len(cal.vectors), nv,
                                    len(noise.range_vectors), C.byref(na), tiff_line_origin,
                                    T.ptr(out), T.ptr(nesz), C.byref(cg), C.byref(ng))
    _check(ctx, rc, CalibrationError)
    return Sigma0Array(out, deburst.lines, deburst.samples, deburst.valid_sample_offset,
                       int(cg.value), int(ng.value), nesz)


def merge_subswaths(inputs: Sequence[SwathInput], ctx: Optional[Context] = None) -> MergedSigma0:
    """merge_subswaths (merge_subswaths.rs:207-450); inputs in IW1 < IW2 < IW3 order."""
    ctx = _ctx(ctx)
    n = len(inputs)
    m = max(1, n)
    arrs = [(_prep(i.sigma0.data, np.float32), _prep(i.sigma0.nesz, np.float32)) for i in inputs]
    sig = (C.c_void_p * m)(*[T.ptr(a[0]) for a in arrs])
    nes = (C.c_void_p * m)(*[T.ptr(a[1]) for a in arrs])
    u64 = lambda vals: (C.c_uint64 * m)(*vals)
    lines = u64([i.sigma0.lines for i in inputs])
    samples = u64([i.sigma0.samples for i in inputs])
    voff = u64([i.sigma0.valid_sample_offset for i in inputs])
    cg = (C.c_uint32 * m)(*[i.sigma0.cal_lut_extrapolation_gap_px for i in inputs])
    ng = (C.c_uint32 * m)(*[i.sigma0.noise_lut_extrapolation_gap_px for i in inputs])
    sw = (_abi.SubSwath * m)(*[i.swath.to_c() for i in inputs])
    az = (C.c_int64 * m)(*[int(i.azimuth_start_time_us) for i in inputs])
    info = _abi.MergedInfo()
    _check(ctx, lib().sd_merge_subswaths(ctx.handle, n, sig, nes, lines, samples, voff, cg, ng, sw,
                                         az, None, None, C.byref(info)), MergeError)
    ref = arrs[0][0]
    out = _empty_like_kind(ref, (info.lines, info.samples), "f4")
    onz = _empty_like_kind(ref, (info.lines, info.samples), "f4")
    _check(ctx, lib().sd_merge_subswaths(ctx.handle, n, sig, nes, lines, samples, voff, cg, ng, sw,
                                         az, T.ptr(out), T.ptr(onz), C.byref(info)), MergeError)
    return _merged_from_info(info, out, onz)


def _merged_from_info(info: _abi.MergedInfo, out, onz) -> MergedSigma0:
    return MergedSigma0(out, int(info.lines), int(info.samples), info.near_slant_range_time_s,
                        info.range_pixel_spacing_s, info.range_pixel_spacing_m,
                        int(info.cal_lut_extrapolation_gap_px),
                        int(info.noise_lut_extrapolation_gap_px), onz,
                        int(info.azimuth_start_time_us))


def swath_inputs_to_c(swaths, keep: T._Keep):
    """ctypes array of sd_swath_input for calibrate_deburst_merge."""
    arr = (_abi.SwathInput * max(1, len(swaths)))()
    for k, s in enumerate(swaths):
        slc = keep.add(_prep(s.slc, np.int16))
        bc = keep.add(T.bursts_to_c(s.bursts))
        cv = keep.add(T.lut_vectors_to_c(s.cal.vectors, keep, "sigma_nought"))
        nv = keep.add(T.lut_vectors_to_c(s.noise.range_vectors, keep, "noise_range_lut"))
        na = T.noise_azimuth_to_c(s.noise, keep)
        arr[k].slc_iq = T.ptr(slc)
        arr[k].tiff_width = int(slc.shape[1])
        arr[k].tiff_height = int(slc.shape[0])
        arr[k].sw = s.sw.to_c()
        arr[k].bursts = C.addressof(bc)
        arr[k].n_bursts = len(s.bursts)
        arr[k].cal = C.addressof(cv)
        arr[k].n_cal = len(s.cal.vectors)
        arr[k].noise_range = C.addressof(nv)
        arr[k].n_noise_range = len(s.noise.range_vectors)
        arr[k].noise_azimuth = na
    return arr


def calibrate_deburst_merge(swaths, ctx: Optional[Context] = None, out=None) -> MergedSigma0:
    """The per-IW deburst -> apply_calibration(tiff_line_origin =
    bursts[0].first_line) -> merge_subswaths chain of prepare_merged_scene
    (scene_prep.rs:598-699), fused into one pass per swath on the GPU.
    `swaths`: objects with .slc (raster), .sw, .bursts, .cal, .noise."""
    ctx = _ctx(ctx)
    keep = T._Keep()
    arr = swath_inputs_to_c(swaths, keep)
    info = _abi.MergedInfo()
    _check(ctx, lib().sd_calibrate_deburst_merge(ctx.handle, len(swaths), arr, None, None,
                                                 C.byref(info)), MergeError)
    ref = swaths[0].slc
    if out is None:
        out = (_empty_like_kind(ref, (info.lines, info.samples), "f4"),
               _empty_like_kind(ref, (info.lines, info.samples), "f4"))
    _check(ctx, lib().sd_calibrate_deburst_merge(ctx.handle, len(swaths), arr, T.ptr(out[0]),
                                                 T.ptr(out[1]), C.byref(info)), MergeError)
    return _merged_from_info(info, out[0], out[1])


# ── speckle ────────────────────────────────────────────────────────────────
def apply_speckle_filter(data, cols: int, rows: int, filter: SpeckleFilter,
                         ctx: Optional[Context] = None):
    """apply_speckle_filter (speckle.rs:131-180): returns a new array of the
    same shape; NaN is nodata."""
    ctx = _ctx(ctx)
    data = _prep(data, np.float32)
    n = T.numel(data)
    out = _empty_like_kind(data, tuple(data.shape), "f4")
    rc = lib().sd_speckle(ctx.handle, T.ptr(data), n, cols, rows, filter.kind, filter.window,
                          filter.enl, filter.damping, T.ptr(out))
    _check(ctx, rc, SpeckleError)
    return out


class SpeckleKernel:
    """The SpeckleKernel trait (speckle.rs:586-603)."""

    def apply(self, data, cols: int, rows: int):
        raise NotImplementedError


class GpuSpeckleKernel(SpeckleKernel):
    """SpeckleKernel implemented by the sm_100a filters."""

    def __init__(self, filter: SpeckleFilter, ctx: Optional[Context] = None):
        self.filter = filter
        self.ctx = ctx

    def apply(self, data, cols: int, rows: int):
        return apply_speckle_filter(data, cols, rows, self.filter, self.ctx)


def apply_speckle_step(data, cols: int, rows: int, kernel: Optional[SpeckleKernel]):
    """apply_speckle_step (run.rs:108-123): replaces the buffer when a kernel
    is given."""
    if kernel is None:
        return data
    return kernel.apply(data, cols, rows)


# ── output: dB conversion and Cloud-Optimised GeoTIFF ─────────────────────
def to_db_inplace(data, noise_floor_linear: float, ctx: Optional[Context] = None,
                  stats: bool = False):
    """to_db_inplace (export.rs:59-99) on the buffer itself (numpy or torch,
    host or device): returns (converted, noise_masked), and with stats=True
    also compute_db_stats (run.rs:63-97) of the result: (min, max, mean,
    median) of the finite dB values."""
    ctx = _ctx(ctx)
    if isinstance(data, np.ndarray) and (data.dtype != np.float32 or not data.flags.c_contiguous):
        raise TypeError("to_db_inplace works in place: pass a contiguous float32 array")
    if not isinstance(data, np.ndarray) and not data.is_contiguous():
        raise TypeError("to_db_inplace works in place: pass a contiguous float32 tensor")
    counts = (C.c_uint64 * 2)()
    st = (C.c_float * 4)()
    rc = lib().sd_to_db(ctx.handle, T.ptr(data), T.numel(data), float(noise_floor_linear), counts,
                        st if stats else None)
    _check(ctx, rc, ExportError)
    out = (int(counts[0]), int(counts[1]))
    return (out, tuple(float(x) for x in st)) if stats else out


def set_db_output(ctx: Context, enable: bool, noise_floor_linear: float = 0.0) -> None:
    """Makes terrain_correction and apply_speckle_filter on `ctx` write their
    raster in dB, converted in the producing kernel as to_db_inplace
    (export.rs:59-99) would convert it afterwards; db_result(ctx) returns
    the last such call's counts and compute_db_stats (run.rs:63-97)."""
    rc = lib().sd_ctx_set_db_output(ctx.handle, int(bool(enable)), float(noise_floor_linear))
    _check(ctx, rc, ExportError)


def db_result(ctx: Context):
    """((converted, noise_masked), (min, max, mean, median)) of the last call
    on `ctx` that wrote dB output."""
    counts = (C.c_uint64 * 2)()
    st = (C.c_float * 4)()
    _check(ctx, lib().sd_ctx_db_result(ctx.handle, counts, st))
    return (int(counts[0]), int(counts[1])), tuple(float(x) for x in st)


def downsample_2x(src, cols: int, rows: int, ctx: Optional[Context] = None):
    """downsample_2x (export.rs:362-392): ((rows+1)//2, (cols+1)//2) raster
    of 2x2 NaN-skipping f64 means."""
    ctx = _ctx(ctx)
    src = _prep(src, np.float32)
    out = _empty_like_kind(src, ((rows + 1) // 2, (cols + 1) // 2), "f4")
    rc = lib().sd_downsample_2x(ctx.handle, T.ptr(src), cols, rows, T.ptr(out))
    _check(ctx, rc, ExportError)
    return out


def write_cog_with_crs(path: str, data, cols: int, rows: int, geotransform, crs: OutputCrs,
                       tile_size: int = 512, ctx: Optional[Context] = None) -> None:
    """write_cog_with_crs (export.rs:329-355): single-band Float32 COG with
    overviews; data host or device."""
    ctx = _ctx(ctx)
    data = _prep(data, np.float32)
    gt = (C.c_double * 6)(*[float(x) for x in geotransform])
    rc = lib().sd_write_cog(ctx.handle, os.fsencode(path), T.ptr(data), cols, rows, gt, int(crs.kind),
                            int(getattr(crs, "zone", 0) or 0), int(tile_size))
    _check(ctx, rc, ExportError)


# ── SLC ingest ─────────────────────────────────────────────────────────────
class SlcReader:
    """SlcReader (slc_reader.rs:485-598) over a Sentinel-1 measurement TIFF;
    reads bursts into host arrays or straight into device tensors."""

    def __init__(self, path: str, ctx: Optional[Context] = None):
        self.ctx = _ctx(ctx)
        self._h = C.c_void_p()
        rc = lib().sd_slc_open(self.ctx.handle, os.fsencode(path), C.byref(self._h))
        _check(self.ctx, rc, SlcReadError)
        w, h, le = C.c_uint32(), C.c_uint32(), C.c_int32()
        lib().sd_slc_dims(self._h, C.byref(w), C.byref(h), C.byref(le))
        self.width, self.height, self.little_endian = int(w.value), int(h.value), bool(le.value)

    @classmethod
    def open(cls, path: str, ctx: Optional[Context] = None) -> "SlcReader":
        return cls(path, ctx)

    def read_burst_raw(self, first_line: int, line_count: int, out=None):
        """line_count rows from first_line as int16 [line_count, width, 2]
        ([I, Q] per pixel).  `out` (numpy, or a CUDA tensor the rows are
        streamed into) is filled and returned; by default a numpy array."""
        if out is None:
            out = np.empty((line_count, self.width, 2), np.int16)
        if T.numel(out) != line_count * self.width * 2:
            raise ValueError("out must hold line_count x width x 2 int16")
        rc = lib().sd_slc_read_burst_raw(self.ctx.handle, self._h, int(first_line), int(line_count), T.ptr(out))
        _check(self.ctx, rc, SlcReadError)
        return out

    def read_burst_complex(self, first_line: int, line_count: int):
        """read_burst_complex (585-598): the same rows as float32 [.., 2]."""
        return self.read_burst_raw(first_line, line_count).astype(np.float32)

    def close(self):
        if self._h:
            lib().sd_slc_close(self._h)
            self._h = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ── pre-TC multilook ───────────────────────────────────────────────────────
def apply_multilook(merged: MergedSigma0, range_looks: int, azimuth_looks: int,
                    azimuth_time_interval_s: float, ctx: Optional[Context] = None) -> MergedSigma0:
    """apply_multilook (scene_prep.rs:1060-1160): the boxcar on the device and
    the reference's geometry update.  R = A = 1 returns the input itself."""
    if range_looks == 1 and azimuth_looks == 1:
        return merged
    ctx = _ctx(ctx)
    if range_looks >= 1 and azimuth_looks > 1 and not (
            np.isfinite(azimuth_time_interval_s) and azimuth_time_interval_s > 0.0):
        raise SardineError(_abi.SD_ERR_INVALID_ARGUMENT, "InvalidArgument",
                           f"azimuth_time_interval_s must be > 0 when azimuth_looks > 1 "
                           f"(got {azimuth_time_interval_s})")
    ol = merged.lines // azimuth_looks if azimuth_looks else 0
    os_ = merged.samples // range_looks if range_looks else 0
    data = _prep(merged.data, np.float32)
    nesz = _prep(merged.nesz, np.float32)
    out = _empty_like_kind(data, (max(ol, 1), max(os_, 1)), "f4")
    onz = _empty_like_kind(data, (max(ol, 1), max(os_, 1)), "f4")
    rc = lib().sd_multilook(ctx.handle, T.ptr(data), T.ptr(nesz), merged.lines, merged.samples,
                            int(range_looks), int(azimuth_looks), T.ptr(out), T.ptr(onz))
    _check(ctx, rc)
    az0 = int(merged.azimuth_start_time_us)
    if azimuth_looks > 1:  # (A-1)/2 lines forward, truncated to whole microseconds (as i64)
        az0 += int((azimuth_looks - 1) / 2.0 * azimuth_time_interval_s * 1e6)
    return MergedSigma0(out, ol, os_,
                        merged.near_slant_range_time_s + (range_looks - 1) / 2.0 * merged.range_pixel_spacing_s,
                        merged.range_pixel_spacing_s * range_looks, merged.range_pixel_spacing_m * range_looks,
                        merged.cal_lut_extrapolation_gap_px, merged.noise_lut_extrapolation_gap_px, onz, az0)


# ── ground range ───────────────────────────────────────────────────────────
def _grd_grids(grids):
    keep, arr = [], (_abi.GrdSwathGrid * max(1, len(grids)))()
    for k, (sid, pts) in enumerate(grids):
        p = (_abi.GrdGridPoint * max(1, len(pts)))()
        for i, g in enumerate(pts):
            p[i].line = int(g.line)
            p[i].slant_range_time_s = float(g.slant_range_time_s)
            p[i].incidence_angle_deg = float(g.incidence_angle_deg)
        keep.append(p)
        arr[k].swath_id = int(str(sid)[-1]) if str(sid)[-1:].isdigit() else 0
        arr[k].points = C.cast(p, C.c_void_p)
        arr[k].n_points = len(pts)
    return arr, keep


def to_ground_range(merged: MergedSigma0, grids, target_spacing_m: float, azimuth_pixel_spacing_m: float,
                    ctx: Optional[Context] = None) -> T.GroundRangeImage:
    """to_ground_range (ground_range.rs:303-427): slant range -> ground range
    at target_spacing_m, then the azimuth looks; `grids` as for
    terrain_correction, with each point's line, slant_range_time_s and
    incidence_angle_deg."""
    ctx = _ctx(ctx)
    data = _prep(merged.data, np.float32)
    arr, keep = _grd_grids(grids)
    info = _abi.GrdInfo()
    args = (merged.lines, merged.samples, float(merged.near_slant_range_time_s),
            float(merged.range_pixel_spacing_s), float(merged.range_pixel_spacing_m), arr, len(grids),
            float(target_spacing_m), float(azimuth_pixel_spacing_m))
    rc = lib().sd_to_ground_range(ctx.handle, T.ptr(data), *args, None, C.byref(info))
    _check(ctx, rc, GroundRangeError)
    out = _empty_like_kind(data, (max(int(info.lines), 1), int(info.samples)), "f4")
    if info.lines:
        rc = lib().sd_to_ground_range(ctx.handle, T.ptr(data), *args, T.ptr(out), C.byref(info))
        _check(ctx, rc, GroundRangeError)
    return T.GroundRangeImage(out[: int(info.lines)], int(info.lines), int(info.samples),
                              info.range_pixel_spacing_m, info.azimuth_pixel_spacing_m, int(info.range_looks),
                              int(info.azimuth_looks))


# ── InSAR: TOPS deramping ──────────────────────────────────────────────────
def _dc_to_c(estimates):
    arr = (_abi.DcEstimateC * max(1, len(estimates)))()
    for k, e in enumerate(estimates):
        arr[k].azimuth_time_us = int(e.azimuth_time_us)
        arr[k].t0_s = float(e.t0_s)
        for j in range(3):
            arr[k].data_dc_poly[j] = float(e.data_dc_poly[j])
    return arr


def deramp_subswath(deburst: DeburstArray, swath: SubSwathMetadata, burst_start_us: int,
                    ctx: Optional[Context] = None) -> T.Deramped:
    """deramp_subswath (insar/deramp.rs:114-210): every CInt16 sample of the
    debursted sub-swath times exp(-j 2 pi f_DC(tau_c) t_az(l)), as complex
    f32 (lines, samples, 2) in the input's kind of memory.  burst_start_us is
    the UTC azimuth time (microseconds) of the first line."""
    ctx = _ctx(ctx)
    est = list(swath.dc_estimates or [])
    iq = _prep(deburst.data, np.int16)
    lines, samples = int(deburst.lines), int(deburst.samples)
    out = _empty_like_kind(iq, (lines, samples, 2), "f4")
    sid = int(str(swath.id)[-1]) if str(swath.id)[-1:].isdigit() else 0
    rc = lib().sd_deramp_subswath(ctx.handle, T.ptr(iq), lines, samples, int(deburst.valid_sample_offset),
                                  float(swath.slant_range_time_s), float(swath.range_pixel_spacing_m),
                                  float(swath.azimuth_time_interval_s), _dc_to_c(est), len(est),
                                  int(burst_start_us), sid, T.ptr(out))
    _check(ctx, rc, InsarError)
    return T.Deramped(out, lines, samples, int(deburst.valid_sample_offset))


# ── InSAR: co-registration resampling, interferogram and coherence ─────────
def resample_secondary(ref_lines: int, ref_samples: int, poly: T.CoregPoly, secondary: T.Deramped,
                       ctx: Optional[Context] = None) -> T.Deramped:
    """resample_secondary (insar/coreg.rs:230-264): the secondary sampled
    bilinearly at each reference pixel moved by the offset polynomials;
    zero outside the secondary."""
    ctx = _ctx(ctx)
    sec = _prep(secondary.data, np.float32)
    out = _empty_like_kind(sec, (int(ref_lines), int(ref_samples), 2), "f4")
    az = (C.c_double * 6)(*[float(v) for v in poly.az])
    rg = (C.c_double * 6)(*[float(v) for v in poly.rg])
    rc = lib().sd_resample_secondary(ctx.handle, T.ptr(sec), int(secondary.lines), int(secondary.samples),
                                     int(ref_lines), int(ref_samples), az, rg, T.ptr(out))
    _check(ctx, rc, InsarError)
    return T.Deramped(out, int(ref_lines), int(ref_samples), int(secondary.valid_sample_offset))


def form_interferogram(coreg: T.Coregistered, ref_swath: SubSwathMetadata, ref_orbit: OrbitData,
                       ref_first_us: int, sec_orbit: OrbitData, wavelength_m: float,
                       cfg: Optional[T.InterferogramConfig] = None,
                       ctx: Optional[Context] = None) -> T.Interferogram:
    """form_interferogram (insar/interferogram.rs:165-398): flat-earth phase,
    cross-product and windowed coherence (and the wrapped phase when
    cfg.compute_phase) in the reference's slant-range geometry."""
    ctx = _ctx(ctx)
    cfg = cfg or T.InterferogramConfig()
    r, s_ = coreg.ref_data, coreg.secondary_resampled
    ref = _prep(r.data, np.float32)
    sec = _prep(s_.data, np.float32)
    lines, samples = int(r.lines), int(r.samples)
    coh = _empty_like_kind(ref, (lines, samples), "f4")
    ph = _empty_like_kind(ref, (lines, samples), "f4") if cfg.compute_phase else None
    ro, so = ref_orbit.to_c(), sec_orbit.to_c()
    rc = lib().sd_form_interferogram(ctx.handle, T.ptr(ref), T.ptr(sec), lines, samples,
                                     int(r.valid_sample_offset), float(ref_swath.slant_range_time_s),
                                     float(ref_swath.range_pixel_spacing_m),
                                     float(ref_swath.azimuth_time_interval_s), ro, len(ref_orbit.times_us),
                                     int(ref_first_us), so, len(sec_orbit.times_us), float(wavelength_m),
                                     int(cfg.az_looks), int(cfg.rg_looks), T.ptr(coh), T.ptr(ph))
    _check(ctx, rc, InsarError)
    return T.Interferogram(coh, ph, lines, samples, int(cfg.az_looks), int(cfg.rg_looks))


def compute_coreg_offsets(ref_swath: SubSwathMetadata, ref_orbit: OrbitData, ref_first_us: int,
                          ref_deburst: DeburstArray, sec_swath: SubSwathMetadata, sec_orbit: OrbitData,
                          sec_first_us: int, ctx: Optional[Context] = None) -> T.CoregResult:
    """compute_coreg_offsets (insar/coreg.rs:128-223): the 20 x 50 sparse grid
    geocoded on the device, the degree-2 offset fits on the host."""
    ctx = _ctx(ctx)
    rc, r = _coreg_offsets_raw(ref_swath, ref_orbit, ref_first_us, ref_deburst, sec_swath, sec_orbit, sec_first_us,
                               ctx)
    _check(ctx, rc, InsarError)
    return T.CoregResult(T.CoregPoly(list(r.az_poly), list(r.rg_poly)), r.fit_residual_rms, int(r.n_valid))


def _coreg_offsets_raw(ref_swath, ref_orbit, ref_first_us, ref_deburst, sec_swath, sec_orbit, sec_first_us,
                       ctx: Context):
    """sd_coreg_offsets' status and result record; n_valid is set on the
    grid-too-small error too (the reference's error carries it,
    insar/coreg.rs:207-208)."""
    r = _abi.CoregResultC()
    rc = lib().sd_coreg_offsets(ctx.handle, ref_orbit.to_c(), len(ref_orbit.times_us), int(ref_first_us),
                                int(ref_deburst.lines), int(ref_deburst.samples),
                                int(ref_deburst.valid_sample_offset), float(ref_swath.azimuth_time_interval_s),
                                float(ref_swath.slant_range_time_s), float(ref_swath.range_pixel_spacing_m),
                                sec_orbit.to_c(), len(sec_orbit.times_us), int(sec_first_us),
                                float(sec_swath.azimuth_time_interval_s), float(sec_swath.slant_range_time_s),
                                float(sec_swath.range_pixel_spacing_m), int(sec_swath.first_sample), C.byref(r))
    return rc, r
