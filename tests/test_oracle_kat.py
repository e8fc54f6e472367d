"""Pins the CPU oracle to the reference's own synthetic known-answer tests.

Each case restates one reference unit test (file:line in sardine/src/) with
the same inputs and the same acceptance bound, run against the oracle.  The
reference cannot be built here (Rust, crates not vendored), so these tests
are what anchors the oracle's parity.
"""
import math

import numpy as np
import pytest

import oracle
import sardine_b200 as sd
from sardine_b200 import _abi

WGS84_A = 6378137.0
WGS84_B = WGS84_A * (1.0 - 1.0 / 298.257223563)
C = 299792458.0
T0 = 1_601_917_680_000_000  # 2020-10-05T17:08:00Z in us


# ── geodesy.rs:141-221 ─────────────────────────────────────────────────────
def test_geodesy_equator_pole_london():
    e = oracle.geodetic_to_ecef(0.0, 0.0, 0.0)
    assert abs(e[0] - WGS84_A) < 1e-3 and abs(e[1]) < 1e-3 and abs(e[2]) < 1e-3
    p = oracle.geodetic_to_ecef(90.0, 0.0, 0.0)
    assert abs(p[0]) < 1e-3 and abs(p[1]) < 1e-3 and abs(p[2] - WGS84_B) < 1e-3
    l = oracle.geodetic_to_ecef(51.5, 0.0, 0.0)  # london_ecef
    assert abs(l[0] - 3_978_700.0) < 2000 and abs(l[1]) < 1 and abs(l[2] - 4_968_400.0) < 2000


# ── orbit.rs:984-1030, 1238-1275: a linear orbit is reproduced exactly ─────
def _linear_orbit():
    p0 = np.array([0.0, 0.0, 7_078_137.0])
    v = np.array([7_600.0, 10.0, -5.0])
    t = np.array([T0 + i * 10_000_000 for i in range(10)], np.int64)
    pos = np.stack([p0 + v * (i * 10.0) for i in range(10)])
    vel = np.tile(v, (10, 1))
    return sd.OrbitData(t, pos, vel), p0, v


def test_lagrange_exact_on_linear_orbit_and_zero_accel():
    orbit, p0, v = _linear_orbit()
    rc, pos, vel, acc = oracle.interpolate_orbit_and_accel(orbit, T0 + 45_000_000)
    assert rc == 0
    assert np.all(np.abs(pos - (p0 + v * 45.0)) < 1e-3)
    assert np.all(np.abs(vel - v) < 1e-9)
    assert np.all(np.abs(acc) < 1e-9)


def test_orbit_refuses_extrapolation():
    orbit, _, _ = _linear_orbit()
    rc, *_ = oracle.interpolate_orbit_and_accel(orbit, T0 - 1)
    assert rc == 2  # OutsideOrbitWindow
    rc, *_ = oracle.interpolate_orbit_and_accel(orbit, T0 + 90_000_001)
    assert rc == 2


# ── terrain_correction.rs:2185-2275: zero-Doppler on a circular orbit ──────
def _circular_test_orbit():
    """make_test_orbit (terrain_correction.rs:2185-2214)."""
    alt = 693_000.0
    r = 6_371_000.0 + alt
    v = math.sqrt(3.986_004_418e14 / r)
    t, pos, vel = [], [], []
    for i in range(30):
        ang = v * (i * 10.0) / r
        t.append(T0 + i * 10_000_000)
        pos.append([r * math.cos(ang), 0.0, r * math.sin(ang)])
        vel.append([-v * math.sin(ang), 0.0, v * math.cos(ang)])
    return sd.OrbitData(np.array(t, np.int64), np.array(pos), np.array(vel))


def test_zero_doppler_converges_at_nadir():
    orbit = _circular_test_orbit()
    s = orbit.positions_m[15]
    target = s * 6_371_000.0 / np.linalg.norm(s)
    st, t, it, res = oracle.solve_zero_doppler(target, orbit, int(orbit.times_us[15]), 10, 1e-6)
    assert st == 0
    assert abs(t - orbit.times_us[15]) < 100_000


def test_zero_doppler_reports_non_convergence():
    orbit = _circular_test_orbit()
    s, vv = orbit.positions_m[15], orbit.velocities_m_s[15]
    nadir = s * 6_371_000.0 / np.linalg.norm(s)
    target = nadir + vv / np.linalg.norm(vv) * 100_000.0
    st, *_ = oracle.solve_zero_doppler(target, orbit, int(orbit.times_us[15]), 1, 1e-12)
    assert st == 1  # NotConverged


# ── terrain_correction.rs:2278-2319: az-time LUT midpoint ───────────────────
def test_azimuth_time_lut_midpoint():
    pts = [sd.GeolocationGridPoint(T0, 52.0), sd.GeolocationGridPoint(T0 + 30_000_000, 50.0)]
    mid = oracle.guess_azimuth_time(pts, 51.0)
    assert abs(mid - (T0 + 15_000_000)) < 100_000


# ── terrain_correction.rs:1982-2183, 2558-2600: flattening geometry ─────────
def _flat_case(dx=500_000.0, dz=700_000.0, lat=50.0, lon=11.0, h=0.0):
    target = oracle.geodetic_to_ecef(lat, lon, h)
    return target, target + np.array([dx, 0.0, dz])


def test_flattening_nadir_is_unity():
    lat, lon, h = 50.0, 11.0, 300.0
    target = oracle.geodetic_to_ecef(lat, lon, h)
    sat = oracle.geodetic_to_ecef(lat, lon, h + 700_000.0)
    g, w, _ = oracle.terrain_geometry(lat, lon, h, h, h, h, sat, target, 1e-4)
    assert g == oracle.GEOM_VALID and abs(w - 1.0) < 1e-4


def test_flattening_side_looking_is_cos_theta():
    target, sat = _flat_case()
    sp = 1e-4
    fe = oracle.geodetic_to_ecef(50.0, 11.0 + sp, 0.0)
    fw = oracle.geodetic_to_ecef(50.0, 11.0 - sp, 0.0)
    fn = oracle.geodetic_to_ecef(50.0 + sp, 11.0, 0.0)
    fs = oracle.geodetic_to_ecef(50.0 - sp, 11.0, 0.0)
    n = np.cross(fe - fw, fn - fs)
    look = (sat - target) / np.linalg.norm(sat - target)
    cos_inc = n.dot(look) / np.linalg.norm(n)
    g, w, cl = oracle.terrain_geometry(50.0, 11.0, 0.0, 0.0, 0.0, 0.0, sat, target, sp)
    assert g == oracle.GEOM_VALID and abs(w - cos_inc) < 1e-6 and w < 1.0
    assert abs(w - cl) < 1e-9 and 0.5 < cl < 1.0  # flat: cos_lia == w (2558-2582)


def test_flattening_slope_layover_shadow_and_symmetry():
    target, sat = _flat_case()
    g, w, _ = oracle.terrain_geometry(50.0, 11.0, 1.0, -1.0, 0.0, 0.0, sat, target, 1e-4)
    assert g == oracle.GEOM_VALID and w > 1.0
    g, _, _ = oracle.terrain_geometry(50.0, 11.0, 100.0, -100.0, 0.0, 0.0, sat, target, 1e-4)
    assert g == oracle.GEOM_LAYOVER
    t2 = oracle.geodetic_to_ecef(50.0, 11.0, 0.0)
    sat2 = t2 + np.array([700_000.0, 0.0, 0.0])
    g, _, _ = oracle.terrain_geometry(50.0, 11.0, -5000.0, 5000.0, 0.0, 0.0, sat2, t2, 1e-4)
    assert g == oracle.GEOM_SHADOW
    wa = oracle.terrain_geometry(50.0, 11.0, 2.0, 0.0, 0.0, 0.0, sat, target, 1e-4)[1]
    wb = oracle.terrain_geometry(50.0, 11.0, 0.0, -2.0, 0.0, 0.0, sat, target, 1e-4)[1]
    wc = oracle.terrain_geometry(50.0, 11.0, 1.0, -1.0, 0.0, 0.0, sat, target, 1e-4)[1]
    assert max(abs(wa - wb), abs(wa - wc)) < 1e-4 * abs(wa)


# ── terrain_correction.rs:2322-2481: samplers and radar coordinates ─────────
def test_bilinear_values_and_nan():
    d = np.arange(1, 10, dtype=np.float32).reshape(3, 3)
    assert abs(oracle.sample(0, d, 1.0, 1.0) - 5.0) < 1e-6
    assert abs(oracle.sample(0, d, 0.5, 0.5) - 3.0) < 1e-6
    d2 = np.array([[1.0, np.nan, 3.0], [4.0, 5.0, 6.0]], np.float32)
    assert math.isnan(oracle.sample(0, d2, 0.0, 0.5))


def test_keys_weights_and_bicubic():
    assert abs(oracle.keys_weight(0.0) - 1.0) < 1e-12
    assert abs(oracle.keys_weight(1.0)) < 1e-12 and abs(oracle.keys_weight(-1.0)) < 1e-12
    assert oracle.keys_weight(2.0) == 0.0 and oracle.keys_weight(-2.5) == 0.0
    s = sum(oracle.keys_weight(li) * oracle.keys_weight(si) for li in range(-1, 3) for si in range(-1, 3))
    assert abs(s - 1.0) < 1e-12
    c = np.full((5, 5), 7.0, np.float32)
    for l, s_ in [(0.5, 0.5), (1.7, 2.3), (3.9, 3.9)]:
        assert abs(oracle.sample(1, c, l, s_) - 7.0) < 1e-4
    g = np.arange(16, dtype=np.float32).reshape(4, 4)
    assert abs(oracle.sample(1, g, 2.0, 3.0) - g[2, 3]) < 1e-4
    n = np.ones((4, 4), np.float32)
    n[1, 1] = np.nan
    assert math.isnan(oracle.sample(1, n, 1.5, 1.5))


def test_lanczos_weights_and_sampler():
    assert abs(oracle.lanczos_weight(0.0) - 1.0) < 1e-12
    for k in (-3, -2, -1, 1, 2, 3):
        assert abs(oracle.lanczos_weight(float(k))) < 1e-12
    c = np.full((8, 8), 5.0, np.float32)
    for l, s_ in [(2.5, 2.5), (3.7, 4.2)]:
        assert abs(oracle.sample(2, c, l, s_) - 5.0) < 0.25
    assert abs(oracle.sample(2, c, 4.0, 4.0) - 5.0) < 1e-4
    g = np.arange(25, dtype=np.float32).reshape(5, 5)
    assert abs(oracle.sample(2, g, 3.0, 4.0) - g[3, 4]) < 1e-3
    n = np.ones((8, 8), np.float32)
    n[4, 4] = np.nan
    assert math.isnan(oracle.sample(2, n, 3.5, 3.5))


def test_output_grid_extent_wgs84_snaps_outward():
    """terrain_correction.rs:1850-1871"""
    scene = sd.SceneMetadata([sd.SubSwathMetadata("IW1", 1, 1, 1, 2e-3, 2.33, 0.005)], [],
                             _linear_orbit()[0], sd.BoundingBox(47.123, 48.876, 11.234, 12.765))
    cfg = sd.TerrainCorrectionConfig(sd.GeoidModel.zero(), pixel_spacing_deg=0.01)
    rc, info = oracle.tc_output_grid(scene, cfg)
    assert rc == 0
    assert abs(info.origin_lat_deg - 48.88) < 1e-9 and abs(info.origin_lon_deg - 11.23) < 1e-9
    assert info.rows == round((48.88 - 47.12) / 0.01) and info.cols == round((12.77 - 11.23) / 0.01)


def test_output_grid_extent_utm_contains_projected_corners():
    """terrain_correction.rs:1877-1973"""
    bb = sd.BoundingBox(48.0, 48.5, 11.0, 12.0)
    scene = sd.SceneMetadata([sd.SubSwathMetadata("IW1", 1, 1, 1, 2e-3, 2.33, 0.005)], [],
                             _linear_orbit()[0], bb)
    for sp in (10.0, 50.0):
        cfg = sd.TerrainCorrectionConfig(sd.GeoidModel.zero(), pixel_spacing_deg=sp,
                                         crs=sd.OutputCrs.utm_north(32))
        rc, info = oracle.tc_output_grid(scene, cfg)
        assert rc == 0
        top, left = info.origin_lat_deg, info.origin_lon_deg
        bottom, right = top - info.rows * sp, left + info.cols * sp
        for lon, lat in [(11.0, 48.0), (11.0, 48.5), (12.0, 48.0), (12.0, 48.5)]:
            x, y = oracle.utm_lonlat_to_xy(32, False, lon, lat)
            assert left <= x <= right and bottom <= y <= top
        if sp == 10.0:
            assert 50_000 < right - left < 200_000 and 40_000 < top - bottom < 100_000


def test_mask_codes_stable():
    """terrain_correction.rs:2672-2683"""
    vals = dict(VALID=0, OUTSIDE_FOOTPRINT=1, DEM_MISSING=2, NON_CONVERGED=3, DEGENERATE_GEOMETRY=4,
                SHADOW=5, LAYOVER=6, FORESHORTENING=7, NOISE_MASKED=8, DEM_NEIGHBOUR_MISSING=9)
    hdr = open(__file__.replace("tests/test_oracle_kat.py", "include/sardine_b200.h")).read()
    for k, v in vals.items():
        assert f"SD_MASK_{k} = {v}" in hdr


# ── output_crs.rs:597-628, 688-790: UTM ─────────────────────────────────────
def test_utm32n_munich_round_trip():
    x, y = oracle.utm_lonlat_to_xy(32, False, 11.5755, 48.1374)
    assert abs(x - 691_603.03) < 1.0 and abs(y - 5_334_780.03) < 1.0
    lon, lat = oracle.utm_xy_to_lonlat(32, False, x, y)
    assert abs(lon - 11.5755) < 1e-7 and abs(lat - 48.1374) < 1e-7


def test_utm56s_sydney_round_trip():
    x, y = oracle.utm_lonlat_to_xy(56, True, 151.2153, -33.8568)
    lon, lat = oracle.utm_xy_to_lonlat(56, True, x, y)
    assert abs(lon - 151.2153) < 1e-7 and abs(lat + 33.8568) < 1e-7
    assert 100_000 < x < 900_000 and y > 5_000_000


@pytest.mark.parametrize("x_start,y", [(600_000.0, 5_334_780.0), (285_000.0, 5_540_000.0)])
def test_project_row_anchor_interpolation_within_1e6_deg(x_start, y):
    lon, lat = oracle.project_row(32, False, y, x_start, 10.0, 25_000, 256)
    for k in range(64):
        col = (k * 24_999) // 63
        lr, la = oracle.utm_xy_to_lonlat(32, False, x_start + col * 10.0, y)
        assert abs(lon[col] - lr) < 1e-6 and abs(lat[col] - la) < 1e-6


def test_project_row_single_pixel():
    lon, lat = oracle.project_row(32, False, 5_334_780.0, 691_603.0, 10.0, 1, 16)
    lr, la = oracle.utm_xy_to_lonlat(32, False, 691_603.0, 5_334_780.0)
    assert abs(lon[0] - lr) < 1e-12 and abs(lat[0] - la) < 1e-12


# ── geoid.rs:472-500 ────────────────────────────────────────────────────────
def test_egm96_synthetic_grid():
    g = np.zeros((73, 144), np.float32)
    g[0, 0], g[0, 1], g[1, 0], g[1, 1] = 40.0, 30.0, 20.0, 10.0
    m = sd.GeoidModel(g)
    assert abs(oracle.geoid_undulation(m, 90.0, 0.0) - 40.0) < 1e-4
    assert abs(oracle.geoid_undulation(m, 90.0, 1.25) - 35.0) < 1e-3
    assert abs(oracle.geoid_undulation(m, 88.75, 1.25) - 25.0) < 1e-3
    g5 = np.full((73, 144), 5.0, np.float32)
    assert abs(oracle.geoid_undulation(sd.GeoidModel(g5), 45.0, 0.0) -
               oracle.geoid_undulation(sd.GeoidModel(g5), 45.0, 360.0)) < 1e-9
    assert oracle.geoid_undulation(sd.GeoidModel.zero(), 45.0, 7.0) == 0.0


# ── dem.rs:999-1030: GLO-30 bilinear ramp ──────────────────────────────────
def test_glo30_linear_ramp():
    pix = 0.25
    data = np.tile(np.arange(4, dtype=np.float32) * 10.0, (4, 1))
    dem = sd.DemGrid(data, 51.0 - 0.5 * pix, 10.0 + 0.5 * pix, pix)
    assert abs(oracle.dem_elevation(dem, 50.5, 10.125)[1] - 0.0) < 1e-3
    assert abs(oracle.dem_elevation(dem, 50.5, 10.375)[1] - 10.0) < 1e-3
    assert abs(oracle.dem_elevation(dem, 50.5, 10.25)[1] - 5.0) < 1e-3
    assert oracle.dem_elevation(dem, 52.0, 10.5)[0] == 1  # outside -> Err


# ── deburst.rs:467-503 ──────────────────────────────────────────────────────
def test_overlap_errors():
    b0 = sd.BurstEntry("IW1", 0, T0, 0, 1000, 0, 100)
    b1 = sd.BurstEntry("IW1", 1, T0 + 100_000, 1000, 2000, 0, 100)
    assert oracle.compute_overlap_lines(b0, b1, 2e-3, 1000)[0] == _abi.SD_ERR_DEBURST_IMPLAUSIBLE_OVERLAP
    b2 = sd.BurstEntry("IW1", 1, T0 + 3_000_000, 1000, 2000, 0, 100)
    assert oracle.compute_overlap_lines(b0, b2, 2e-3, 1000)[0] == _abi.SD_ERR_DEBURST_INVALID_OVERLAP
    b3 = sd.BurstEntry("IW1", 1, T0 + 1_800_000, 1000, 2000, 0, 100)
    rc, ov = oracle.compute_overlap_lines(b0, b3, 2e-3, 1000)
    assert rc == 0 and ov == 100


# ── merge_subswaths.rs:554-725 ──────────────────────────────────────────────
RPS = 2.329562
DT = RPS * 2.0 / C


def _sw(t0):
    return sd.SubSwathMetadata("IW", 1, 1, 10, 2e-3, RPS, t0)


def _sig(vals, samples, voff, cg=0, ng=0):
    a = np.asarray(vals, np.float32).reshape(-1, samples)
    return sd.Sigma0Array(a, a.shape[0], samples, voff, cg, ng, np.zeros_like(a))


def _merge(*pairs):
    return oracle.merge_subswaths([sd.SwathInput(s, w, T0) for s, w in pairs])[0]


def test_merge_no_overlap_concatenated():
    m = _merge((_sig(range(1, 11), 10, 0), _sw(0.0)), (_sig(range(11, 21), 10, 0), _sw(10 * DT)))
    assert m.samples == 20 and m.lines == 1 and not np.isnan(m.data).any()
    assert m.data[0, 0] == 1.0 and m.data[0, 9] == 10.0 and m.data[0, 10] == 11.0 and m.data[0, 19] == 20.0


def test_merge_seam_at_midpoint():
    m = _merge((_sig([1.0] * 12, 12, 0), _sw(0.0)), (_sig([2.0] * 12, 12, 0), _sw(8 * DT)))
    assert m.samples == 20 and m.data[0, 9] == 1.0 and m.data[0, 10] == 2.0


def test_merge_min_lines_and_gap_max():
    m = _merge((_sig([1.0] * 50, 10, 0, 17, 0), _sw(0.0)), (_sig([2.0] * 30, 10, 0, 5, 42), _sw(10 * DT)))
    assert m.lines == 3
    assert m.cal_lut_extrapolation_gap_px == 17 and m.noise_lut_extrapolation_gap_px == 42


def test_merge_valid_offset_mapping():
    m = _merge((_sig(range(1, 11), 10, 5), _sw(0.0)), (_sig(range(101, 111), 10, 0), _sw(10 * DT)))
    assert m.samples == 15
    assert m.data[0, 0] == 1.0 and m.data[0, 6] == 7.0 and m.data[0, 7] == 103.0 and m.data[0, 14] == 110.0


def test_merge_near_range_time():
    m = _merge((_sig([1.0] * 10, 10, 3), _sw(0.005)), (_sig([2.0] * 10, 10, 0), _sw(0.005 + 15 * DT)))
    assert abs(m.near_slant_range_time_s - (0.005 + 3 * DT)) < 1e-15


def test_merge_errors():
    with pytest.raises(oracle.OracleError) as e:
        oracle.merge_subswaths([])
    assert e.value.code == _abi.SD_ERR_MERGE_EMPTY_INPUTS
    with pytest.raises(oracle.OracleError) as e:
        _merge((_sig([1.0] * 10, 10, 0), _sw(0.005)),
               (_sig([1.0] * 10, 10, 0), sd.SubSwathMetadata("IW", 1, 1, 10, 2e-3, 2.50, 0.006)))
    assert e.value.code == _abi.SD_ERR_MERGE_INCONSISTENT_PIXEL_SPACING


# ── apply_calibration.rs:583-765 ────────────────────────────────────────────
def _cal1(iq, k, noise, az=None):
    """Single-pixel calibration through the oracle's full apply_calibration."""
    deb = sd.DeburstArray(np.array(iq, np.int16).reshape(1, -1, 2), 1, len(iq), 0)
    n = deb.samples
    px = np.array([0, max(n, 1) + 10], np.uint32)
    cal = sd.SwathCalibration("IW1", [sd.CalibrationVector(0, px, np.array([k, k], np.float32))])
    nz = sd.SwathNoise("IW1", [sd.NoiseRangeVector(0, px, np.array([noise, noise], np.float32))],
                       [] if az is None else [sd.NoiseAzimuthVector(np.array([0, 10], np.int32),
                                                                    np.array([az, az], np.float32))])
    return oracle.apply_calibration(deb, cal, nz, 0)


def test_calibration_known_values():
    s = _cal1([[3, 4], [0, 0]], 10.0, 0.0)
    assert abs(s.data[0, 0] - 0.25) < 1e-7 and s.data[0, 1] == 0.0  # 25/100
    s = _cal1([[100, 200]], 300.0, 1000.0)
    assert abs(s.data[0, 0] - 49000.0 / 90000.0) < 1e-5
    s = _cal1([[10, 5]], 10.0, 25.0)  # power 125 -> sigma0 1.0, NESZ 0.25
    assert abs(s.data[0, 0] - 1.0) < 1e-5 and abs(s.nesz[0, 0] - 0.25) < 1e-5
    s = _cal1([[2, 1]], 10.0, 50.0)  # power 5 < noise: clamp to 0, NESZ 0.5
    assert s.data[0, 0] == 0.0 and abs(s.nesz[0, 0] - 0.5) < 1e-5
    s = _cal1([[10, 0]], 0.0, 10.0)  # k = 0 -> both outputs 0
    assert s.data[0, 0] == 0.0 and s.nesz[0, 0] == 0.0
    s = _cal1([[11, 3]], 10.0, 10.0, az=3.0)  # power 130, noise 30 -> 1.0, NESZ 0.3
    assert abs(s.data[0, 0] - 1.0) < 1e-5 and abs(s.nesz[0, 0] - 0.3) < 1e-5
    s = _cal1([[32767, 32767]], 1.0, 0.0)
    assert abs(s.data[0, 0] - float(np.float32(2 * 32767 * 32767))) < 1.0


def test_calibration_lut_interpolation():
    """interp_range_lut / lerp / bracket_azimuth (649-721) through full calls."""
    deb = sd.DeburstArray(np.full((3, 201, 2), [10, 0], np.int16), 3, 201, 0)
    px = np.array([0, 100, 200], np.uint32)
    cal = sd.SwathCalibration("IW1", [sd.CalibrationVector(0, px, np.array([1.0, 2.0, 3.0], np.float32)),
                                      sd.CalibrationVector(2, px, np.array([3.0, 4.0, 5.0], np.float32))])
    nz = sd.SwathNoise("IW1", [sd.NoiseRangeVector(0, px, np.zeros(3, np.float32))])
    s = oracle.apply_calibration(deb, cal, nz, 0)
    k = np.sqrt(100.0 / s.data)
    assert abs(k[0, 100] - 2.0) < 1e-5 and abs(k[0, 50] - 1.5) < 1e-5  # exact hit / midpoint
    assert abs(k[1, 100] - 3.0) < 1e-5  # azimuth midpoint between the two vectors
    assert abs(k[2, 200] - 5.0) < 1e-5


def test_calibration_errors():
    deb = sd.DeburstArray(np.zeros((1, 2000, 2), np.int16), 1, 2000, 0)
    px = np.array([0, 100], np.uint32)
    cal = sd.SwathCalibration("IW1", [sd.CalibrationVector(0, px, np.ones(2, np.float32))])
    nz = sd.SwathNoise("IW1", [sd.NoiseRangeVector(0, px, np.ones(2, np.float32))])
    with pytest.raises(oracle.OracleError) as e:
        oracle.apply_calibration(deb, cal, nz, 0)
    assert e.value.code == _abi.SD_ERR_CAL_LUT_RANGE_INSUFFICIENT
    with pytest.raises(oracle.OracleError) as e:
        oracle.apply_calibration(deb, sd.SwathCalibration("IW1", []), nz, 0)
    assert e.value.code == _abi.SD_ERR_CAL_NO_CALIBRATION_VECTORS


# ── speckle.rs:621-1000 ─────────────────────────────────────────────────────
F = sd.SpeckleFilter


def _spk(data, cols, rows, f):
    return oracle.apply_speckle_filter(np.asarray(data, np.float32), cols, rows, f)


def test_speckle_constant_fixed_point():
    data = np.full(11 * 9, 0.123, np.float32)
    for f in [F.Boxcar(3), F.Boxcar(7), F.Lee(5, 1.0), F.Lee(5, 4.0), F.Frost(5, 1.0), F.Frost(7, 2.0),
              F.GammaMap(5, 1.0), F.GammaMap(7, 4.0), F.RefinedLee(1.0), F.RefinedLee(4.0)]:
        out = _spk(data, 11, 9, f)
        assert np.all(np.abs(out - 0.123) <= 1e-6), f


def test_speckle_nan_centre():
    data = np.ones(81, np.float32)
    data[40] = np.nan
    for f in [F.Boxcar(3), F.Lee(3, 1.0), F.Frost(3, 1.0), F.GammaMap(3, 1.0), F.RefinedLee(1.0)]:
        out = _spk(data, 9, 9, f)
        assert np.isnan(out[40]) and np.isfinite(out[0])


def test_refined_lee_edge():
    data = np.where(np.arange(21)[None, :] < 10, 0.05, 0.50).repeat(21, 0).astype(np.float32)
    out = _spk(data.ravel(), 21, 21, F.RefinedLee(4.0)).reshape(21, 21)
    assert abs(out[10, 17] - 0.50) <= 1e-4
    assert abs(out[10, 11] - 0.50) < abs(out[10, 11] - 0.275)


def test_speckle_window_means():
    nan = np.nan
    out = _spk([nan, nan, nan, nan, 1.0, nan, nan, nan, nan], 3, 3, F.Boxcar(3))
    assert abs(out[4] - 1.0) <= 1e-6
    out = _spk(np.arange(1, 10), 3, 3, F.Boxcar(3))
    assert abs(out[4] - 5.0) <= 1e-6


def test_lee_enl_behaviour():
    data = np.full(25, 0.05, np.float32)
    data[12] = 0.50
    lo = _spk(data, 5, 5, F.Lee(3, 1.0))[12]
    hi = _spk(data, 5, 5, F.Lee(3, 10_000.0))[12]
    assert abs(hi - 0.5) < abs(lo - 0.5) and abs(hi - 0.5) < 0.005


def test_frost_zero_damping_is_boxcar():
    data = np.arange(1, 26, dtype=np.float32) * 0.01
    assert np.all(np.abs(_spk(data, 5, 5, F.Frost(3, 0.0)) - _spk(data, 5, 5, F.Boxcar(3))) <= 1e-6)


def test_gamma_map_regimes():
    data = np.array([0.10 + 0.0005 * ((i % 3) - 1.0) for i in range(25)], np.float32)
    assert abs(_spk(data, 5, 5, F.GammaMap(3, 1.0))[12] - 0.10) <= 1e-3
    pt = np.full(9, 0.01, np.float32)
    pt[4] = 100.0
    assert abs(_spk(pt, 3, 3, F.GammaMap(3, 4.0))[4] - 100.0) <= 1e-3
    q = [0.02, 0.18, 0.02, 0.18, 0.10, 0.18, 0.02, 0.18, 0.02]
    assert abs(_spk(q, 3, 3, F.GammaMap(3, 4.0))[4] - 0.11341) <= 5e-4


@pytest.mark.parametrize("f,code", [
    (F.Boxcar(4), _abi.SD_ERR_SPECKLE_BAD_WINDOW), (F.Boxcar(1), _abi.SD_ERR_SPECKLE_BAD_WINDOW),
    (F.Lee(3, 0.0), _abi.SD_ERR_SPECKLE_BAD_ENL), (F.Lee(3, float("nan")), _abi.SD_ERR_SPECKLE_BAD_ENL),
    (F.Lee(3, float("inf")), _abi.SD_ERR_SPECKLE_BAD_ENL), (F.RefinedLee(-1.0), _abi.SD_ERR_SPECKLE_BAD_ENL),
    (F.Frost(3, -0.1), _abi.SD_ERR_SPECKLE_BAD_DAMPING), (F.Frost(3, float("inf")), _abi.SD_ERR_SPECKLE_BAD_DAMPING),
])
def test_speckle_errors(f, code):
    with pytest.raises(oracle.OracleError) as e:
        _spk(np.full(25, 0.1), 5, 5, f)
    assert e.value.code == code


def test_speckle_dimension_mismatch():
    with pytest.raises(oracle.OracleError) as e:
        _spk(np.full(24, 0.1), 5, 5, F.Boxcar(3))
    assert e.value.code == _abi.SD_ERR_SPECKLE_DIMENSION_MISMATCH
