"""GPU terrain correction vs the CPU oracle on identical seeded scenes.

The oracle runs twice on every case: with the platform libm (glibc, which the
reference calls) and with correctly rounded sines and cosines
(oracle.libm("cr"); it also switches the forward UTM projection of DEM
lookups to the functions the device uses).  The GPU takes the sines and
cosines of its target ECEF coordinates from a correctly rounded function
and decides every DEM height as the exact projection would, so against the
second run the bar holds for every pixel: converged azimuth times, masks,
counters, the Newton histogram and the NaN pattern bit-exact, and
sigma0/gamma0 and cos(LIA) within 1e-4 relative.  Against the first run the
same bar holds outside the pixels where the two oracle runs differ, i.e.
where glibc's results are not correctly rounded; assert_tc_parity returns
their count.
"""
import numpy as np
import pytest

import oracle
import sardine_b200 as sd
from sardine_b200 import synth

pytestmark = pytest.mark.gpu

REL_TOL = 1e-4
COS_ABS = 1e-9  # cos(LIA) near zero: the facet is a chord expansion (~1e-11 m on 20 m chords)


def oracle_tc(*args, **kw):
    """The oracle with glibc's and with correctly rounded sines and cosines."""
    gl = oracle.terrain_correction(*args, **kw)
    with oracle.libm("cr"):
        cr = oracle.terrain_correction(*args, **kw)
    return gl, cr


def _neq(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return ~((a == b) | (np.isnan(a) & np.isnan(b)))


def libm_pixels(gl, cr):
    """Pixels where the glibc and the correctly rounded oracle runs differ."""
    d = _neq(gl.data, cr.data)
    if gl.mask is not None:
        d |= np.asarray(gl.mask) != np.asarray(cr.mask)
        d |= _neq(gl.cos_lia, cr.cos_lia)
    return d


def _rel(a, b):
    a = a.astype(np.float64)
    b = b.astype(np.float64)
    both = np.isfinite(a) & np.isfinite(b)
    d = np.zeros_like(a)
    d[both] = np.abs(a[both] - b[both]) / np.maximum(np.abs(b[both]), 1e-30)
    return d, both


def _bar(gpu, ref, compute_lia, keep):
    g = np.asarray(gpu.data)
    r = np.asarray(ref.data)
    k = np.ones(g.shape, bool) if keep is None else keep
    assert np.array_equal(np.isnan(g)[k], np.isnan(r)[k]), "NaN pattern differs"
    d, _ = _rel(g, r)
    n_bad = int((d[k] > REL_TOL).sum())
    assert n_bad == 0, f"{n_bad} pixels beyond {REL_TOL}, max {d[k].max()}"
    if compute_lia:
        gm, rm = np.asarray(gpu.mask), np.asarray(ref.mask)
        assert np.array_equal(gm[k], rm[k]), f"mask differs at {int((gm != rm)[k].sum())} px"
        gc, rc_ = np.asarray(gpu.cos_lia).astype(np.float64), np.asarray(ref.cos_lia).astype(np.float64)
        assert np.array_equal(np.isnan(gc)[k], np.isnan(rc_)[k])
        both = np.isfinite(gc) & np.isfinite(rc_) & k
        bad = np.abs(gc[both] - rc_[both]) > REL_TOL * np.abs(rc_[both]) + COS_ABS
        assert not bad.any(), f"cos(LIA) beyond the bar at {int(bad.sum())} px"


def _counters(gpu, ref):
    for k in ("valid_pixel_count", "dem_missing_count", "outside_footprint_count",
              "non_converged_count", "degenerate_geometry_count", "flat_masked_count",
              "noise_masked_count", "total_pixel_count"):
        assert getattr(gpu, k) == getattr(ref, k), k
    assert gpu.newton_iter_histogram == ref.newton_iter_histogram


def assert_tc_parity(gpu: sd.GeocodedImage, refs, compute_lia=True) -> int:
    """The bar against both oracle runs; returns the number of pixels where
    glibc's results are not correctly rounded."""
    gl, cr = refs
    assert (gpu.rows, gpu.cols) == (cr.rows, cr.cols)
    assert tuple(gpu.geotransform) == tuple(cr.geotransform)
    _counters(gpu, cr)
    _bar(gpu, cr, compute_lia, None)
    libm = libm_pixels(gl, cr)
    if not libm.any():
        _counters(gpu, gl)
    _bar(gpu, gl, compute_lia, ~libm)
    return int(libm.sum())


@pytest.mark.parametrize("resampling,flatten", [
    (sd.ResamplingKernel.Bilinear, False),
    (sd.ResamplingKernel.Bicubic, True),
    (sd.ResamplingKernel.Lanczos3, True),
])
def test_config1_shape_parity(ctx, resampling, flatten):
    sc = synth.config1_scene(seed=11, n_lines=1024, n_samples=2048, dem_n=256,
                             resampling=resampling, flatten=flatten)
    ref = oracle_tc(sc.merged, sc.scene, sc.dem, sc.grids, sc.config)
    gpu = sd.terrain_correction(sc.merged, sc.scene, sc.dem, sc.grids, sc.config, ctx=ctx)
    assert ref[0].valid_pixel_count > 0.5 * ref[0].total_pixel_count
    assert_tc_parity(gpu, ref)


def test_config1_full_shape_parity(ctx):
    """Plain terrain correction at its full stated shape: a 4096 x 8192
    sigma0 image, a 1024 x 1024 EPSG:4326 DEM, bilinear, LIA, no flattening."""
    sc = synth.config1_scene(seed=1)
    assert (sc.merged.lines, sc.merged.samples) == (4096, 8192)
    assert np.asarray(sc.dem.data).shape == (1024, 1024)
    assert sc.config.resampling == sd.ResamplingKernel.Bilinear and not sc.config.flatten
    ref = oracle_tc(sc.merged, sc.scene, sc.dem, sc.grids, sc.config)
    gpu = sd.terrain_correction(sc.merged, sc.scene, sc.dem, sc.grids, sc.config, ctx=ctx)
    assert ref[1].valid_pixel_count > 0.5 * ref[1].total_pixel_count
    assert_tc_parity(gpu, ref)


def test_config1_partial_footprint_and_voids(ctx):
    """DEM larger than the radar footprint (outside-footprint pixels) with
    NaN voids (DEM_MISSING and DEM_NEIGHBOUR_MISSING)."""
    sc = synth.config1_scene(seed=12, n_lines=256, n_samples=512, dem_n=320, flatten=True)
    dem = np.array(sc.dem.data)
    dem[40:60, 100:130] = np.nan
    dem[200, :] = np.nan
    sc.dem.data = dem
    ref = oracle_tc(sc.merged, sc.scene, sc.dem, sc.grids, sc.config)
    gpu = sd.terrain_correction(sc.merged, sc.scene, sc.dem, sc.grids, sc.config, ctx=ctx)
    assert ref[0].outside_footprint_count > 0 and ref[0].dem_missing_count > 0
    assert_tc_parity(gpu, ref)


def test_nesz_masking_and_nan_seams(ctx):
    sc = synth.config1_scene(seed=13, n_lines=512, n_samples=1024, dem_n=200)
    rng = np.random.default_rng(5)
    img = np.array(sc.merged.data)
    img[:, 300:310] = np.nan  # merge-seam gap
    nesz = rng.uniform(0.0, 0.06, size=img.shape).astype(np.float32)
    sc.merged.data = img
    sc.merged.nesz = nesz
    sc.config.noise_floor_margin_db = 0.0
    ref = oracle_tc(sc.merged, sc.scene, sc.dem, sc.grids, sc.config)
    gpu = sd.terrain_correction(sc.merged, sc.scene, sc.dem, sc.grids, sc.config, ctx=ctx)
    assert ref[0].noise_masked_count > 0
    assert_tc_parity(gpu, ref)


def test_small_max_iter_non_converged(ctx):
    sc = synth.config1_scene(seed=14, n_lines=256, n_samples=512, dem_n=96)
    sc.config.max_newton_iterations = 1
    ref = oracle_tc(sc.merged, sc.scene, sc.dem, sc.grids, sc.config)
    gpu = sd.terrain_correction(sc.merged, sc.scene, sc.dem, sc.grids, sc.config, ctx=ctx)
    assert ref[0].non_converged_count > 0
    assert_tc_parity(gpu, ref)


def test_loose_tolerance_generic_path(ctx):
    sc = synth.config1_scene(seed=15, n_lines=256, n_samples=512, dem_n=96)
    sc.config.newton_tolerance_s = 2e-4
    ref = oracle_tc(sc.merged, sc.scene, sc.dem, sc.grids, sc.config)
    gpu = sd.terrain_correction(sc.merged, sc.scene, sc.dem, sc.grids, sc.config, ctx=ctx)
    assert_tc_parity(gpu, ref)


def test_orbit_window_error(ctx):
    sc = synth.config1_scene(seed=16, n_lines=256, n_samples=512, dem_n=64)
    o = sc.scene.orbit
    sc.scene.orbit = sd.OrbitData(o.times_us[:9].copy(), o.positions_m[:9].copy(),
                                  o.velocities_m_s[:9].copy())
    with pytest.raises(oracle.OracleError) as e:
        oracle.terrain_correction(sc.merged, sc.scene, sc.dem, sc.grids, sc.config)
    with pytest.raises(sd.TerrainCorrectionError) as g:
        sd.terrain_correction(sc.merged, sc.scene, sc.dem, sc.grids, sc.config, ctx=ctx)
    assert g.value.kind == "Orbit" and e.value.code == g.value.code


def test_config2_shape_utm_parity(ctx):
    """UTM output grid, projected DEM, bicubic, gamma0 flattening + LIA."""
    sc = synth.config2_scene(seed=21, n_bursts=3, lines_per_burst=400, tiff_width=1500,
                             burst_step=300, swath_overlap=150, out_rows=None, out_cols=None,
                             lut_lines_step=150)
    swaths = sc.swaths
    merged_g = sd.calibrate_deburst_merge(swaths, ctx=ctx)
    # oracle chain: deburst -> calibrate -> merge
    inputs = []
    for s in swaths:
        deb = oracle.deburst_subswath(s.slc, s.sw, s.bursts)
        sig = oracle.apply_calibration(deb, s.cal, s.noise, s.bursts[0].first_line)
        inputs.append(sd.SwathInput(sig, s.sw, s.bursts[0].azimuth_time_us))
    merged_o, _ = oracle.merge_subswaths(inputs)
    assert np.array_equal(np.asarray(merged_g.data), merged_o.data, equal_nan=True)
    assert np.array_equal(np.asarray(merged_g.nesz), merged_o.nesz, equal_nan=True)
    ref = oracle_tc(merged_o, sc.scene, sc.dem, sc.grids, sc.config)
    gpu = sd.terrain_correction(merged_g, sc.scene, sc.dem, sc.grids, sc.config, ctx=ctx)
    assert ref[0].valid_pixel_count > 0
    assert_tc_parity(gpu, ref)


def test_device_resident_inputs(ctx):
    import torch
    sc = synth.config1_scene(seed=17, n_lines=512, n_samples=1024, dem_n=128)
    ref = oracle_tc(sc.merged, sc.scene, sc.dem, sc.grids, sc.config)
    sc.merged.data = torch.from_numpy(np.asarray(sc.merged.data)).cuda()
    sc.dem.data = torch.from_numpy(np.asarray(sc.dem.data)).cuda()
    gpu = sd.terrain_correction(sc.merged, sc.scene, sc.dem, sc.grids, sc.config, ctx=ctx)
    assert gpu.data.is_cuda
    gpu.data, gpu.cos_lia, gpu.mask = gpu.data.cpu().numpy(), gpu.cos_lia.cpu().numpy(), gpu.mask.cpu().numpy()
    assert_tc_parity(gpu, ref)


def test_row_bands_equal_whole_grid(ctx):
    """Row bands (the multi-GPU decomposition of one scene) reproduce the
    whole grid's rows exactly and their counters add up."""
    sc = synth.config1_scene(seed=18, n_lines=512, n_samples=1024, dem_n=128, flatten=True)
    whole = sd.terrain_correction(sc.merged, sc.scene, sc.dem, sc.grids, sc.config, ctx=ctx)
    bands = [(0, 37), (37, 90), (90, 0)]
    assert whole.rows > 90
    parts = [sd.terrain_correction(sc.merged, sc.scene, sc.dem, sc.grids, sc.config, ctx=ctx, row_range=b)
             for b in bands]
    assert np.array_equal(np.concatenate([p.data for p in parts]), whole.data, equal_nan=True)
    assert np.array_equal(np.concatenate([p.mask for p in parts]), whole.mask)
    assert sum(p.valid_pixel_count for p in parts) == whole.valid_pixel_count
    assert list(np.sum([p.newton_iter_histogram for p in parts], axis=0)) == whole.newton_iter_histogram


def test_orbit_window_polynomials_match_lagrange(ctx):
    """The GPU orbit (window polynomials) against the oracle's 8-point
    Lagrange at random microseconds and at the state-vector times themselves
    (where the reference's acceleration formula drops a term)."""
    import ctypes as C
    sc = synth.config1_scene(seed=19, n_lines=256, n_samples=512, dem_n=64)
    orb = sc.scene.orbit
    t = np.asarray(orb.times_us, np.int64)
    rng = np.random.default_rng(3)
    times = np.concatenate([rng.integers(t[0], t[-1] + 1, 4000), t, t[1:-1] - 1, t[1:-1] + 1]).astype(np.int64)
    out = np.empty((len(times), 9), np.float64)
    svs = orb.to_c()
    rc = sd.lib().sd_orbit_states(ctx.handle, svs, len(t), times.ctypes.data, len(times), out.ctypes.data)
    assert rc == 0, ctx.last_error()
    ref = np.array([np.concatenate(oracle.interpolate_orbit_and_accel(orb, int(x))[1:]) for x in times])
    assert np.abs(out[:, 0:3] - ref[:, 0:3]).max() < 1e-7        # m, of ~7e6 m
    assert np.abs(out[:, 3:6] - ref[:, 3:6]).max() < 1e-9        # m/s
    # far from a window's centre the reference's own acceleration sums carry
    # ~1e-7 m/s^2 of rounding; 2e-6 m/s^2 moves a Newton step by < 1e-13 s
    assert np.abs(out[:, 6:9] - ref[:, 6:9]).max() < 2e-6        # m/s^2
    bad = np.array([t[-1] + 1], np.int64)
    rc = sd.lib().sd_orbit_states(ctx.handle, svs, len(t), bad.ctypes.data, 1, out.ctypes.data)
    assert rc == 10


def test_config1_full_shape_parity(ctx):
    """Config 1 at its stated shape: 4096 x 8192 sigma0 (exponential, mean
    0.05), 1024^2 EPSG:4326 DEM at 1 arcsec, bilinear, LIA, no flattening;
    converged times per pixel included."""
    sc = synth.config1_scene(seed=1)
    assert (sc.merged.lines, sc.merged.samples) == (4096, 8192)
    (gl, gl_t, _), (cr, cr_t, _) = oracle_tc(sc.merged, sc.scene, sc.dem, sc.grids, sc.config,
                                             return_times=True)
    gpu = sd.terrain_correction(sc.merged, sc.scene, sc.dem, sc.grids, sc.config, ctx=ctx, return_times=True)
    assert gpu.total_pixel_count == 1024 * 1024
    assert gpu.valid_pixel_count > 0.5 * gpu.total_pixel_count
    assert np.array_equal(gpu.azimuth_time_us, cr_t)
    same = gl_t == cr_t
    assert np.array_equal(gpu.azimuth_time_us[same], gl_t[same])
    assert_tc_parity(gpu, (gl, cr))


def test_config2_shape_utm_times(ctx):
    """UTM grid on a projected DEM (the configuration where DEM positions are
    interpolated on the device): converged times equal the correctly rounded
    oracle's at every pixel."""
    sc = synth.config2_scene(seed=22, n_bursts=3, lines_per_burst=400, tiff_width=1500,
                             burst_step=300, swath_overlap=150, out_rows=None, out_cols=None,
                             lut_lines_step=150)
    merged = sd.calibrate_deburst_merge(sc.swaths, ctx=ctx)
    with oracle.libm("cr"):
        ref, ref_t, _ = oracle.terrain_correction(merged, sc.scene, sc.dem, sc.grids, sc.config,
                                                  return_times=True)
    gpu = sd.terrain_correction(merged, sc.scene, sc.dem, sc.grids, sc.config, ctx=ctx, return_times=True)
    assert ref.valid_pixel_count > 0
    assert np.array_equal(np.asarray(gpu.azimuth_time_us), ref_t)
    _bar(gpu, ref, True, None)


def test_device_cr_sincos_equals_host(ctx):
    """The device's correctly rounded sin/cos is the host's, bit for bit."""
    import torch
    g = torch.Generator(device="cuda").manual_seed(3)
    x = torch.cat([torch.empty(3_000_000, dtype=torch.float64, device="cuda").uniform_(-3.2, 3.2, generator=g),
                   torch.empty(500_000, dtype=torch.float64, device="cuda").uniform_(-10.0, 10.0, generator=g),
                   torch.empty(500_000, dtype=torch.float64, device="cuda").uniform_(-1e5, 1e5, generator=g)])
    s, c = torch.empty_like(x), torch.empty_like(x)
    rc = sd.lib().sd_cr_sincos(ctx.handle, x.data_ptr(), x.numel(), s.data_ptr(), c.data_ptr())
    assert rc == 0, ctx.last_error()
    torch.cuda.synchronize()
    hs, hc = oracle.cr_sincos(x.cpu().numpy())
    assert np.array_equal(s.cpu().numpy().view(np.uint64), hs.view(np.uint64))
    assert np.array_equal(c.cpu().numpy().view(np.uint64), hc.view(np.uint64))
