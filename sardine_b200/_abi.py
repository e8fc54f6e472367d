"""ctypes mirrors of the structs in ``include/sardine_b200.h``.

These are plain data contracts; they carry no behaviour.  Field order and
types follow the header exactly (the header is the source of truth).
"""
from __future__ import annotations

import ctypes as C

SD_NEWTON_ITER_HIST_SIZE = 16

# status codes (sd_status)
SD_OK = 0
SD_ERR_INVALID_ARGUMENT = 1
SD_ERR_CUDA = 2
SD_ERR_OUT_OF_MEMORY = 3
SD_ERR_INTERNAL = 4
SD_ERR_TIMEOUT = 5
SD_ERR_BUSY = 6
SD_ERR_TC_ORBIT = 10
SD_ERR_TC_DEM = 11
SD_ERR_TC_NO_GRID_POINTS = 12
SD_ERR_TC_NO_SUBSWATHS = 13
SD_ERR_TC_CONFIG = 14
SD_ERR_TC_PROJECTION = 15
SD_ERR_SPECKLE_DIMENSION_MISMATCH = 20
SD_ERR_SPECKLE_BAD_WINDOW = 21
SD_ERR_SPECKLE_BAD_ENL = 22
SD_ERR_SPECKLE_BAD_DAMPING = 23
SD_ERR_CAL_NO_CALIBRATION_VECTORS = 30
SD_ERR_CAL_NO_NOISE_RANGE_VECTORS = 31
SD_ERR_CAL_LUT_RANGE_INSUFFICIENT = 32
SD_ERR_DEBURST_NO_BURSTS = 40
SD_ERR_DEBURST_BURST_COUNT_MISMATCH = 41
SD_ERR_DEBURST_TIFF_TOO_SMALL = 42
SD_ERR_DEBURST_EMPTY_VALID_WINDOW = 43
SD_ERR_DEBURST_INVALID_OVERLAP = 44
SD_ERR_DEBURST_IMPLAUSIBLE_OVERLAP = 45
SD_ERR_MERGE_EMPTY_INPUTS = 50
SD_ERR_MERGE_INCONSISTENT_PIXEL_SPACING = 51
SD_ERR_MERGE_EMPTY_SWATH = 52
SD_ERR_EXPORT_IO = 60
SD_ERR_EXPORT_INVALID_NOISE_FLOOR = 61
SD_ERR_EXPORT_INVALID_GEOTRANSFORM = 62
SD_ERR_EXPORT_INVALID_TILE_SIZE = 63
SD_ERR_SLC_IO = 70
SD_ERR_SLC_NOT_TIFF = 71
SD_ERR_SLC_BIGTIFF = 72
SD_ERR_SLC_MISSING_TAG = 73
SD_ERR_SLC_UNSUPPORTED_FORMAT = 74
SD_ERR_SLC_NON_CONTIGUOUS_STRIPS = 75
SD_ERR_SLC_LINE_OUT_OF_BOUNDS = 76
SD_ERR_GRD_NO_GRID_POINTS = 80
SD_ERR_GRD_EMPTY_IMAGE = 81
SD_ERR_GRD_INVALID_SPACING = 82
SD_ERR_GRD_INVALID_AZIMUTH_SPACING = 83
SD_ERR_GRD_INTERPOLATION_FAILED = 84
SD_ERR_INSAR_NO_DC_ESTIMATES = 90
SD_ERR_INSAR_AZIMUTH_TIME_BEFORE_DC = 91
SD_ERR_INSAR_INVALID_WINDOW_SIZE = 92
SD_ERR_INSAR_ORBIT = 93
SD_ERR_INSAR_COREG_GRID_TOO_SMALL = 94

RESAMPLE_BILINEAR, RESAMPLE_BICUBIC, RESAMPLE_LANCZOS3 = 0, 1, 2
CRS_WGS84, CRS_UTM_NORTH, CRS_UTM_SOUTH = 0, 1, 2
DEM_GEOGRAPHIC, DEM_PROJECTED_UTM = 0, 1
GEOID_ZERO, GEOID_GRID = 0, 1
SPECKLE_BOXCAR, SPECKLE_LEE, SPECKLE_FROST, SPECKLE_GAMMA_MAP, SPECKLE_REFINED_LEE = range(5)
PRECISION_FP64, PRECISION_SPLIT = 0, 1


class StateVector(C.Structure):
    _fields_ = [("time_us", C.c_int64), ("position_m", C.c_double * 3),
                ("velocity_m_s", C.c_double * 3)]


class RadarImage(C.Structure):
    _fields_ = [("data", C.c_void_p), ("nesz", C.c_void_p), ("lines", C.c_uint64),
                ("samples", C.c_uint64), ("azimuth_start_time_us", C.c_int64),
                ("near_slant_range_time_s", C.c_double), ("range_pixel_spacing_m", C.c_double)]


class Scene(C.Structure):
    _fields_ = [("azimuth_time_interval_s", C.c_double), ("n_sub_swaths", C.c_int32),
                ("min_lat_deg", C.c_double), ("max_lat_deg", C.c_double),
                ("min_lon_deg", C.c_double), ("max_lon_deg", C.c_double),
                ("state_vectors", C.c_void_p), ("n_state_vectors", C.c_uint64)]


class Dem(C.Structure):
    _fields_ = [("kind", C.c_int32), ("utm_zone", C.c_int32), ("utm_south", C.c_int32),
                ("_pad", C.c_int32), ("data", C.c_void_p), ("width", C.c_uint64),
                ("height", C.c_uint64), ("origin_y", C.c_double), ("origin_x", C.c_double),
                ("pixel_size", C.c_double)]


class Geoid(C.Structure):
    _fields_ = [("kind", C.c_int32), ("_pad", C.c_int32), ("undulations_m", C.c_void_p)]


class GeoGridPoint(C.Structure):
    _fields_ = [("azimuth_time_us", C.c_int64), ("latitude_deg", C.c_double)]


class GrdGridPoint(C.Structure):
    _fields_ = [("line", C.c_uint32), ("pad", C.c_uint32), ("slant_range_time_s", C.c_double),
                ("incidence_angle_deg", C.c_double)]


class GrdSwathGrid(C.Structure):
    _fields_ = [("swath_id", C.c_int32), ("pad", C.c_int32), ("points", C.c_void_p), ("n_points", C.c_uint64)]


class GrdInfo(C.Structure):
    _fields_ = [("lines", C.c_uint64), ("samples", C.c_uint64), ("range_pixel_spacing_m", C.c_double),
                ("azimuth_pixel_spacing_m", C.c_double), ("range_looks", C.c_uint64),
                ("azimuth_looks", C.c_uint64)]


class DcEstimateC(C.Structure):
    _fields_ = [("azimuth_time_us", C.c_int64), ("t0_s", C.c_double), ("data_dc_poly", C.c_double * 3)]


class CoregResultC(C.Structure):
    _fields_ = [("az_poly", C.c_double * 6), ("rg_poly", C.c_double * 6), ("fit_residual_rms", C.c_double),
                ("n_valid", C.c_uint64)]


class TcConfig(C.Structure):
    _fields_ = [("pixel_spacing", C.c_double), ("crs", C.c_int32), ("utm_zone", C.c_int32),
                ("max_newton_iterations", C.c_int32), ("flatten", C.c_int32),
                ("newton_tolerance_s", C.c_double), ("compute_lia", C.c_int32),
                ("resampling", C.c_int32), ("noise_floor_margin_db", C.c_float),
                ("projector_anchors", C.c_int32), ("precision", C.c_int32), ("_pad", C.c_int32)]


class GeocodedInfo(C.Structure):
    _fields_ = [("rows", C.c_uint64), ("cols", C.c_uint64), ("origin_lat_deg", C.c_double),
                ("origin_lon_deg", C.c_double), ("pixel_spacing", C.c_double),
                ("geotransform", C.c_double * 6), ("total_pixel_count", C.c_uint64),
                ("valid_pixel_count", C.c_uint64), ("dem_missing_count", C.c_uint64),
                ("outside_footprint_count", C.c_uint64), ("non_converged_count", C.c_uint64),
                ("degenerate_geometry_count", C.c_uint64), ("flat_masked_count", C.c_uint64),
                ("noise_masked_count", C.c_uint64),
                ("newton_iter_histogram", C.c_uint64 * SD_NEWTON_ITER_HIST_SIZE),
                ("diag_exact_path_pixels", C.c_uint64), ("diag_fp64_redo_pixels", C.c_uint64),
                ("diag_fp64_resampled", C.c_uint64)]

    COUNTERS = ("total_pixel_count", "valid_pixel_count", "dem_missing_count",
                "outside_footprint_count", "non_converged_count", "degenerate_geometry_count",
                "flat_masked_count", "noise_masked_count")

    def counters(self) -> dict:
        d = {k: int(getattr(self, k)) for k in self.COUNTERS}
        d["newton_iter_histogram"] = [int(x) for x in self.newton_iter_histogram]
        return d


class LutVector(C.Structure):
    _fields_ = [("line", C.c_int32), ("_pad", C.c_int32), ("pixels", C.c_void_p),
                ("values", C.c_void_p), ("n", C.c_uint64)]


class NoiseAzimuth(C.Structure):
    _fields_ = [("lines", C.c_void_p), ("values", C.c_void_p), ("n", C.c_uint64)]


class Burst(C.Structure):
    _fields_ = [("azimuth_time_us", C.c_int64), ("burst_index", C.c_uint64),
                ("first_line", C.c_uint64), ("last_line", C.c_uint64),
                ("first_valid_sample", C.c_uint64), ("last_valid_sample", C.c_uint64)]


class SubSwath(C.Structure):
    _fields_ = [("burst_count", C.c_uint64), ("lines_per_burst", C.c_uint64),
                ("azimuth_time_interval_s", C.c_double), ("range_pixel_spacing_m", C.c_double),
                ("slant_range_time_s", C.c_double)]


class SwathInput(C.Structure):
    _fields_ = [("slc_iq", C.c_void_p), ("tiff_width", C.c_uint64), ("tiff_height", C.c_uint64),
                ("sw", SubSwath), ("bursts", C.c_void_p), ("n_bursts", C.c_uint64),
                ("cal", C.c_void_p), ("n_cal", C.c_uint64), ("noise_range", C.c_void_p),
                ("n_noise_range", C.c_uint64), ("noise_azimuth", NoiseAzimuth)]


class MergedInfo(C.Structure):
    _fields_ = [("lines", C.c_uint64), ("samples", C.c_uint64),
                ("near_slant_range_time_s", C.c_double), ("range_pixel_spacing_s", C.c_double),
                ("range_pixel_spacing_m", C.c_double),
                ("cal_lut_extrapolation_gap_px", C.c_uint32),
                ("noise_lut_extrapolation_gap_px", C.c_uint32),
                ("azimuth_start_time_us", C.c_int64), ("n_swaths", C.c_int32), ("_pad", C.c_int32),
                ("swath_out_offset", C.c_int64 * 8), ("swath_seam", C.c_uint64 * 8),
                ("swath_lines", C.c_uint64 * 8), ("swath_valid_offset", C.c_uint64 * 8)]


class Tile(C.Structure):
    _fields_ = [("scene", C.c_void_p), ("cfg", TcConfig), ("origin_x", C.c_double),
                ("origin_y", C.c_double), ("rows", C.c_uint64), ("cols", C.c_uint64),
                ("speckle", C.c_int32), ("speckle_window", C.c_int32), ("enl", C.c_float),
                ("damping", C.c_float), ("out_data", C.c_void_p), ("out_cos_lia", C.c_void_p),
                ("out_mask", C.c_void_p)]
