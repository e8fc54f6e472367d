"""Python mirrors of the reference data model on the hot path.

Each class follows a Rust type of SARdine (types.rs, calibration.rs,
apply_calibration.rs, deburst.rs, merge_subswaths.rs, terrain_correction.rs,
pipeline_options.rs, speckle.rs, geoid.rs, dem.rs, output_crs.rs) with the
same field names.  Arrays are numpy arrays (host) or torch tensors (host or
CUDA); the C ABI accepts either.  Times are int64 microseconds since a common
epoch.
"""
from __future__ import annotations

import ctypes as C
import enum
from dataclasses import dataclass, field
from typing import Any, List, Optional, Sequence, Tuple

import numpy as np

from . import _abi


def ptr(a: Any) -> int:
    """Address of a numpy array or torch tensor (contiguous)."""
    if a is None:
        return 0
    if isinstance(a, np.ndarray):
        if not a.flags["C_CONTIGUOUS"]:
            raise ValueError("array must be C-contiguous")
        return a.ctypes.data
    if hasattr(a, "data_ptr"):
        if not a.is_contiguous():
            raise ValueError("tensor must be contiguous")
        return a.data_ptr()
    raise TypeError(f"unsupported array type {type(a)!r}")


def numel(a: Any) -> int:
    return int(a.size) if isinstance(a, np.ndarray) else int(a.numel())


# ── enums ──────────────────────────────────────────────────────────────────
class ResamplingKernel(enum.IntEnum):
    """pipeline_options.rs:75-90"""
    Bilinear = _abi.RESAMPLE_BILINEAR
    Bicubic = _abi.RESAMPLE_BICUBIC
    Lanczos3 = _abi.RESAMPLE_LANCZOS3


@dataclass(frozen=True)
class OutputCrs:
    """output_crs.rs:70-96 (WGS84 lat/lon and UTM north/south)."""
    kind: int = _abi.CRS_WGS84
    zone: int = 0

    @staticmethod
    def wgs84() -> "OutputCrs":
        return OutputCrs(_abi.CRS_WGS84, 0)

    @staticmethod
    def utm_north(zone: int) -> "OutputCrs":
        return OutputCrs(_abi.CRS_UTM_NORTH, zone)

    @staticmethod
    def utm_south(zone: int) -> "OutputCrs":
        return OutputCrs(_abi.CRS_UTM_SOUTH, zone)

    @staticmethod
    def from_epsg(code: int) -> "OutputCrs":
        """OutputCrs::from_epsg (output_crs.rs:121-130), LAEA/WebMercator excluded."""
        if code == 4326:
            return OutputCrs.wgs84()
        if 32601 <= code <= 32660:
            return OutputCrs.utm_north(code - 32600)
        if 32701 <= code <= 32760:
            return OutputCrs.utm_south(code - 32700)
        raise ValueError(f"unsupported EPSG code {code}")

    @property
    def is_metric(self) -> bool:
        return self.kind != _abi.CRS_WGS84

    def epsg(self) -> int:
        if self.kind == _abi.CRS_WGS84:
            return 4326
        return (32600 if self.kind == _abi.CRS_UTM_NORTH else 32700) + self.zone


# ── orbit / scene ──────────────────────────────────────────────────────────
@dataclass
class OrbitData:
    """types.rs:157.  state_vectors: structured (n, 7) float64 [pos3, vel3]
    plus times_us int64 (n,)."""
    times_us: np.ndarray
    positions_m: np.ndarray
    velocities_m_s: np.ndarray

    def to_c(self) -> C.Array:
        n = len(self.times_us)
        arr = (_abi.StateVector * n)()
        for i in range(n):
            arr[i].time_us = int(self.times_us[i])
            for c in range(3):
                arr[i].position_m[c] = float(self.positions_m[i, c])
                arr[i].velocity_m_s[c] = float(self.velocities_m_s[i, c])
        return arr


@dataclass
class BoundingBox:
    """types.rs:227"""
    min_lat_deg: float
    max_lat_deg: float
    min_lon_deg: float
    max_lon_deg: float


@dataclass
class SubSwathMetadata:
    """types.rs:281 (fields used on the hot path)."""
    id: str
    burst_count: int
    lines_per_burst: int
    range_samples: int
    azimuth_time_interval_s: float
    range_pixel_spacing_m: float
    slant_range_time_s: float
    dc_estimates: list = None  # [DcEstimate]; deramp_subswath needs them
    first_sample: int = 0      # full-image column of the first valid pixel (compute_coreg_offsets)

    def to_c(self) -> _abi.SubSwath:
        return _abi.SubSwath(self.burst_count, self.lines_per_burst, self.azimuth_time_interval_s,
                             self.range_pixel_spacing_m, self.slant_range_time_s)


@dataclass
class BurstEntry:
    """types.rs:351"""
    subswath_id: str
    burst_index: int
    azimuth_time_us: int
    first_line: int
    last_line: int
    first_valid_sample: int
    last_valid_sample: int

    def to_c(self) -> _abi.Burst:
        return _abi.Burst(int(self.azimuth_time_us), self.burst_index, self.first_line,
                          self.last_line, self.first_valid_sample, self.last_valid_sample)


def bursts_to_c(bursts: Sequence[BurstEntry]) -> C.Array:
    arr = (_abi.Burst * max(1, len(bursts)))()
    for i, b in enumerate(bursts):
        arr[i] = b.to_c()
    return arr


@dataclass
class SceneMetadata:
    """types.rs:406 (the parts the hot path reads)."""
    sub_swaths: List[SubSwathMetadata]
    bursts: List[BurstEntry]
    orbit: OrbitData
    bounding_box: BoundingBox


@dataclass
class GeolocationGridPoint:
    """types.rs:171 (fields read by the terrain correction)."""
    azimuth_time_us: int
    latitude_deg: float
    longitude_deg: float = 0.0
    slant_range_time_s: float = 0.0
    line: int = 0                    # read by the ground-range projection
    incidence_angle_deg: float = 0.0


@dataclass
class DcEstimate:
    """types.rs:206-213: a Doppler-centroid polynomial f_DC(tau) = a0 + a1 (tau - t0)
    + a2 (tau - t0)^2 valid around azimuth_time_us (UTC microseconds)."""
    azimuth_time_us: int
    t0_s: float
    data_dc_poly: Sequence[float]


@dataclass
class Deramped:
    """insar/deramp.rs:73-84.  data: (lines, samples, 2) float32 [I, Q]."""
    data: Any
    lines: int
    samples: int
    valid_sample_offset: int


@dataclass
class CoregPoly:
    """insar/coreg.rs:73-90: offsets (dl, dc) = p0 + p1 l + p2 c + p3 l^2 + p4 l c + p5 c^2."""
    az: Sequence[float]
    rg: Sequence[float]


@dataclass
class CoregResult:
    """insar/coreg.rs:102-109."""
    poly: Any
    fit_residual_rms: float
    n_valid: int


@dataclass
class Coregistered:
    """insar/coreg.rs:93-98: reference and resampled secondary, both Deramped."""
    ref_data: Any
    secondary_resampled: Any


@dataclass
class InterferogramConfig:
    """insar/interferogram.rs:123-150 (defaults 10 x 40, no phase)."""
    az_looks: int = 10
    rg_looks: int = 40
    compute_phase: bool = False


@dataclass
class Interferogram:
    """insar/interferogram.rs:100-117.  phase is None unless requested."""
    coherence: Any
    phase: Any
    lines: int
    samples: int
    az_looks: int
    rg_looks: int


@dataclass
class GroundRangeImage:
    """ground_range.rs:60-85."""
    data: Any
    lines: int
    samples: int
    range_pixel_spacing_m: float
    azimuth_pixel_spacing_m: float
    range_looks: int
    azimuth_looks: int


def grid_to_c(points: Sequence[GeolocationGridPoint]) -> C.Array:
    arr = (_abi.GeoGridPoint * max(1, len(points)))()
    for i, p in enumerate(points):
        arr[i].azimuth_time_us = int(p.azimuth_time_us)
        arr[i].latitude_deg = float(p.latitude_deg)
    return arr


def pick_lut_grid(grids: Sequence[Tuple[str, Sequence[GeolocationGridPoint]]]):
    """build_azimuth_time_lut's choice (terrain_correction.rs:1086-1091): IW2,
    else the first sub-swath's grid."""
    for sid, pts in grids:
        if sid == "IW2":
            return pts
    return grids[0][1] if grids else []


# ── calibration LUTs ───────────────────────────────────────────────────────
@dataclass
class CalibrationVector:
    """calibration.rs:38-53 (sigma_nought only is used on this path)."""
    line: int
    pixels: np.ndarray  # uint32
    sigma_nought: np.ndarray  # float32


@dataclass
class SwathCalibration:
    """calibration.rs:57-69"""
    subswath_id: str
    vectors: List[CalibrationVector]


@dataclass
class NoiseRangeVector:
    """calibration.rs:73-82"""
    line: int
    pixels: np.ndarray
    noise_range_lut: np.ndarray


@dataclass
class NoiseAzimuthVector:
    """calibration.rs:86-96"""
    lines: np.ndarray  # int32
    noise_azimuth_lut: np.ndarray  # float32


@dataclass
class SwathNoise:
    """calibration.rs:100-107"""
    subswath_id: str
    range_vectors: List[NoiseRangeVector]
    azimuth_vectors: List[NoiseAzimuthVector] = field(default_factory=list)


class _Keep:
    """Holds references so ctypes pointers stay valid."""

    def __init__(self):
        self.refs: list = []

    def add(self, *objs):
        self.refs.extend(objs)
        return objs[0] if len(objs) == 1 else objs


def lut_vectors_to_c(vecs, keep: _Keep, values_attr: str) -> C.Array:
    arr = (_abi.LutVector * max(1, len(vecs)))()
    for i, v in enumerate(vecs):
        px = np.ascontiguousarray(v.pixels, dtype=np.uint32)
        vals = np.ascontiguousarray(getattr(v, values_attr), dtype=np.float32)
        keep.add(px, vals)
        arr[i].line = int(v.line)
        arr[i].pixels = px.ctypes.data
        arr[i].values = vals.ctypes.data
        arr[i].n = len(px)
    return arr


def noise_azimuth_to_c(noise: SwathNoise, keep: _Keep) -> _abi.NoiseAzimuth:
    na = _abi.NoiseAzimuth(0, 0, 0)
    if noise.azimuth_vectors:
        av = noise.azimuth_vectors[0]
        lines = np.ascontiguousarray(av.lines, dtype=np.int32)
        vals = np.ascontiguousarray(av.noise_azimuth_lut, dtype=np.float32)
        keep.add(lines, vals)
        na.lines, na.values, na.n = lines.ctypes.data, vals.ctypes.data, len(lines)
    return na


# ── rasters ────────────────────────────────────────────────────────────────
@dataclass
class DeburstArray:
    """deburst.rs:137-147.  data: (lines, samples, 2) int16."""
    data: Any
    lines: int
    samples: int
    valid_sample_offset: int


@dataclass
class Sigma0Array:
    """apply_calibration.rs:92-119"""
    data: Any
    lines: int
    samples: int
    valid_sample_offset: int
    cal_lut_extrapolation_gap_px: int
    noise_lut_extrapolation_gap_px: int
    nesz: Any


@dataclass
class SwathInput:
    """merge_subswaths.rs (SwathInput)"""
    sigma0: Sigma0Array
    swath: SubSwathMetadata
    azimuth_start_time_us: int


@dataclass
class MergedSigma0:
    """merge_subswaths.rs:106-162; also the RadarImage implementation used by
    the terrain correction (terrain_correction.rs:888-928)."""
    data: Any
    lines: int
    samples: int
    near_slant_range_time_s: float
    range_pixel_spacing_s: float
    range_pixel_spacing_m: float
    cal_lut_extrapolation_gap_px: int
    noise_lut_extrapolation_gap_px: int
    nesz: Any
    azimuth_start_time_us: int

    def to_c(self) -> _abi.RadarImage:
        return _abi.RadarImage(ptr(self.data), ptr(self.nesz), self.lines, self.samples,
                               int(self.azimuth_start_time_us), self.near_slant_range_time_s,
                               self.range_pixel_spacing_m)


@dataclass
class DemGrid:
    """A DemSource (dem.rs:829-842) backed by one raster.  kind
    DEM_GEOGRAPHIC follows Glo30Tile::elevation_at (dem.rs:351-371) inside a
    DemMosaic (longitude normalisation, dem.rs:697); kind DEM_PROJECTED_UTM
    applies the forward UTM projection first, then the same grid rules."""
    data: Any  # (height, width) float32
    origin_y: float
    origin_x: float
    pixel_size: float
    kind: int = _abi.DEM_GEOGRAPHIC
    utm_zone: int = 0
    utm_south: bool = False

    def to_c(self) -> _abi.Dem:
        h, w = (self.data.shape[0], self.data.shape[1])
        return _abi.Dem(self.kind, self.utm_zone, int(self.utm_south), 0, ptr(self.data), w, h,
                        self.origin_y, self.origin_x, self.pixel_size)


@dataclass
class GeoidModel:
    """geoid.rs:342-402: Zero or a 73x144 2.5-degree grid (Egm96/Egm2008)."""
    undulations_m: Optional[np.ndarray] = None

    @staticmethod
    def zero() -> "GeoidModel":
        return GeoidModel(None)

    def to_c(self, keep: _Keep) -> _abi.Geoid:
        if self.undulations_m is None:
            return _abi.Geoid(_abi.GEOID_ZERO, 0, 0)
        g = np.ascontiguousarray(self.undulations_m, dtype=np.float32).reshape(73 * 144)
        keep.add(g)
        return _abi.Geoid(_abi.GEOID_GRID, 0, g.ctypes.data)


class Precision:
    """Terrain-correction arithmetic: FP64 reproduces the reference; SPLIT
    keeps the FP64 orbit, Newton residuals and slant range (same converged
    times, mask and counters) and runs resampling, facet, LIA and flattening
    in FP32."""
    FP64 = _abi.PRECISION_FP64
    SPLIT = _abi.PRECISION_SPLIT


@dataclass
class TerrainCorrectionConfig:
    """terrain_correction.rs:100-236; TerrainCorrectionConfig::new defaults."""
    geoid: GeoidModel
    pixel_spacing_deg: float = 0.0001
    crs: OutputCrs = field(default_factory=OutputCrs.wgs84)
    max_newton_iterations: int = 10
    newton_tolerance_s: float = 1e-6
    flatten: bool = False
    compute_lia: bool = False
    noise_floor_margin_db: float = float("-inf")
    resampling: ResamplingKernel = ResamplingKernel.Bilinear
    precision: int = _abi.PRECISION_FP64

    def to_c(self, anchors: int) -> _abi.TcConfig:
        return _abi.TcConfig(self.pixel_spacing_deg, self.crs.kind, self.crs.zone,
                             self.max_newton_iterations, int(self.flatten),
                             self.newton_tolerance_s, int(self.compute_lia), int(self.resampling),
                             self.noise_floor_margin_db, anchors, self.precision, 0)


def scene_to_c(scene: SceneMetadata, keep: _Keep) -> _abi.Scene:
    svs = keep.add(scene.orbit.to_c())
    bb = scene.bounding_box
    ati = scene.sub_swaths[0].azimuth_time_interval_s if scene.sub_swaths else 0.0
    return _abi.Scene(ati, len(scene.sub_swaths), bb.min_lat_deg, bb.max_lat_deg, bb.min_lon_deg,
                      bb.max_lon_deg, C.addressof(svs), len(scene.orbit.times_us))


@dataclass
class GeocodedImage:
    """terrain_correction.rs:238-307"""
    data: Any
    rows: int
    cols: int
    origin_lat_deg: float
    origin_lon_deg: float
    pixel_spacing_lat_deg: float
    pixel_spacing_lon_deg: float
    total_pixel_count: int
    valid_pixel_count: int
    dem_missing_count: int
    outside_footprint_count: int
    non_converged_count: int
    degenerate_geometry_count: int
    flat_masked_count: int
    noise_masked_count: int
    geotransform: Tuple[float, ...]
    crs: OutputCrs
    cos_lia: Any
    mask: Any
    newton_iter_histogram: List[int]
    diag_exact_path_pixels: int = 0  # converged pixels computed on the row walk's exact path
    diag_fp64_redo_pixels: int = 0   # split precision: pixels recomputed in FP64
    diag_fp64_resampled: int = 0     # split precision: candidates re-sampled in FP64
    azimuth_time_us: Any = None      # converged zero-Doppler time per pixel (INT64_MIN: none)

    def valid_fraction(self) -> float:
        return self.valid_pixel_count / self.total_pixel_count

    @staticmethod
    def from_info(info: _abi.GeocodedInfo, crs: OutputCrs, data, cos_lia, mask) -> "GeocodedImage":
        return GeocodedImage(
            data=data, rows=int(info.rows), cols=int(info.cols),
            origin_lat_deg=info.origin_lat_deg, origin_lon_deg=info.origin_lon_deg,
            pixel_spacing_lat_deg=info.pixel_spacing, pixel_spacing_lon_deg=info.pixel_spacing,
            total_pixel_count=int(info.total_pixel_count),
            valid_pixel_count=int(info.valid_pixel_count),
            dem_missing_count=int(info.dem_missing_count),
            outside_footprint_count=int(info.outside_footprint_count),
            non_converged_count=int(info.non_converged_count),
            degenerate_geometry_count=int(info.degenerate_geometry_count),
            flat_masked_count=int(info.flat_masked_count),
            noise_masked_count=int(info.noise_masked_count),
            geotransform=tuple(info.geotransform), crs=crs, cos_lia=cos_lia, mask=mask,
            newton_iter_histogram=[int(x) for x in info.newton_iter_histogram],
            diag_exact_path_pixels=int(info.diag_exact_path_pixels),
            diag_fp64_redo_pixels=int(info.diag_fp64_redo_pixels),
            diag_fp64_resampled=int(info.diag_fp64_resampled))


# ── speckle ────────────────────────────────────────────────────────────────
@dataclass(frozen=True)
class SpeckleFilter:
    """speckle.rs:61-91.  Construct with the classmethods."""
    kind: int
    window: int = 7
    enl: float = 1.0
    damping: float = 0.0

    @classmethod
    def Boxcar(cls, window: int) -> "SpeckleFilter":
        return cls(_abi.SPECKLE_BOXCAR, window)

    @classmethod
    def Lee(cls, window: int, enl: float) -> "SpeckleFilter":
        return cls(_abi.SPECKLE_LEE, window, enl)

    @classmethod
    def Frost(cls, window: int, damping: float) -> "SpeckleFilter":
        return cls(_abi.SPECKLE_FROST, window, 1.0, damping)

    @classmethod
    def GammaMap(cls, window: int, enl: float) -> "SpeckleFilter":
        return cls(_abi.SPECKLE_GAMMA_MAP, window, enl)

    @classmethod
    def RefinedLee(cls, enl: float) -> "SpeckleFilter":
        return cls(_abi.SPECKLE_REFINED_LEE, 7, enl)
