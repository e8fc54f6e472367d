"""Split-precision terrain correction (SD_PRECISION_SPLIT) vs the FP64 oracle.

The split path keeps every integer outcome of the FP64 path: converged
azimuth times (so geolocation error 0 px), masks, counters and the Newton
histogram are compared exactly.  sigma0/gamma0 and cos(LIA) come from FP32
resampling and an FP32 facet; their error against the oracle is measured per
output and must stay within 1e-4 relative (cos(LIA): 1e-5 absolute).
"""
import numpy as np
import pytest

import oracle
import sardine_b200 as sd
from sardine_b200 import synth
from sardine_b200.accuracy import compare_geocoded

pytestmark = pytest.mark.gpu

SPLIT = sd.Precision.SPLIT


def oracle_cr(*args, **kw):
    """The oracle with correctly rounded sines and cosines, the arithmetic of
    the device's target ECEF coordinates (the glibc run is compared with the
    FP64 path in test_gpu_tc.py)."""
    with oracle.libm("cr"):
        return oracle.terrain_correction(*args, **kw)


def _check(gpu, ref, ref_t, ati_s, compute_lia=True):
    rep = compare_geocoded(gpu, ref, gpu.azimuth_time_us, ref_t, ati_s)
    for k in ("valid_pixel_count", "dem_missing_count", "outside_footprint_count",
              "non_converged_count", "degenerate_geometry_count", "flat_masked_count",
              "noise_masked_count"):
        assert getattr(gpu, k) == getattr(ref, k), k
    assert gpu.newton_iter_histogram == ref.newton_iter_histogram
    assert rep["time_mismatch_px"] == 0, rep
    assert rep["geoloc_err_px_max"] == 0.0, rep
    assert rep["nan_pattern_equal"], rep
    assert rep["sigma_rel_over_1e-4_px"] == 0, rep
    if compute_lia:
        assert rep["mask_equal"], rep
        assert rep["cos_lia_abs_err_max"] <= 1e-5, rep
    return rep


@pytest.mark.parametrize("resampling,flatten", [
    (sd.ResamplingKernel.Bilinear, False),
    (sd.ResamplingKernel.Bicubic, True),
    (sd.ResamplingKernel.Lanczos3, True),
])
def test_split_config1_shape(ctx, resampling, flatten):
    sc = synth.config1_scene(seed=31, n_lines=1024, n_samples=2048, dem_n=256,
                             resampling=resampling, flatten=flatten)
    ref, ref_t, _ = oracle_cr(sc.merged, sc.scene, sc.dem, sc.grids, sc.config, return_times=True)
    sc.config.precision = SPLIT
    gpu = sd.terrain_correction(sc.merged, sc.scene, sc.dem, sc.grids, sc.config, ctx=ctx,
                                return_times=True)
    _check(gpu, ref, ref_t, sc.scene.sub_swaths[0].azimuth_time_interval_s)


def test_split_nesz_masking(ctx):
    """NESZ decisions near the threshold are settled in FP64: mask exact."""
    sc = synth.config1_scene(seed=33, n_lines=512, n_samples=1024, dem_n=200)
    rng = np.random.default_rng(7)
    img = np.array(sc.merged.data)
    nesz = rng.uniform(0.0, 0.06, size=img.shape).astype(np.float32)
    sc.merged.nesz = nesz
    sc.config.noise_floor_margin_db = 0.0
    ref, ref_t, _ = oracle_cr(sc.merged, sc.scene, sc.dem, sc.grids, sc.config, return_times=True)
    sc.config.precision = SPLIT
    gpu = sd.terrain_correction(sc.merged, sc.scene, sc.dem, sc.grids, sc.config, ctx=ctx,
                                return_times=True)
    assert ref.noise_masked_count > 0
    _check(gpu, ref, ref_t, sc.scene.sub_swaths[0].azimuth_time_interval_s)


def test_split_config2_shape_lanczos(ctx):
    """Config-3 processing (lanczos3, flatten, LIA, UTM) on a reduced IW scene."""
    sc = synth.config2_scene(seed=41, n_bursts=3, lines_per_burst=400, tiff_width=1500,
                             burst_step=300, swath_overlap=150, out_rows=None, out_cols=None,
                             lut_lines_step=150, resampling=sd.ResamplingKernel.Lanczos3)
    merged = sd.calibrate_deburst_merge(sc.swaths, ctx=ctx)
    ref, ref_t, _ = oracle_cr(merged, sc.scene, sc.dem, sc.grids, sc.config, return_times=True)
    sc.config.precision = SPLIT
    gpu = sd.terrain_correction(merged, sc.scene, sc.dem, sc.grids, sc.config, ctx=ctx,
                                return_times=True)
    assert ref.valid_pixel_count > 0
    rep = _check(gpu, ref, ref_t, sc.scene.sub_swaths[0].azimuth_time_interval_s)
    assert rep["sigma_db_err_p99"] <= 4.4e-4


def test_fp64_times_match_oracle(ctx):
    """The FP64 path's converged times equal the oracle's, pixel for pixel:
    all of them against the correctly rounded run, and against the glibc run
    wherever that run's times equal the correctly rounded run's."""
    sc = synth.config1_scene(seed=35, n_lines=512, n_samples=1024, dem_n=160, flatten=True)
    ref, ref_t, _ = oracle_cr(sc.merged, sc.scene, sc.dem, sc.grids, sc.config, return_times=True)
    gpu = sd.terrain_correction(sc.merged, sc.scene, sc.dem, sc.grids, sc.config, ctx=ctx,
                                return_times=True)
    _, gl_t, _ = oracle.terrain_correction(sc.merged, sc.scene, sc.dem, sc.grids, sc.config, return_times=True)
    assert np.array_equal(gpu.azimuth_time_us, ref_t)
    same = gl_t == ref_t
    assert np.array_equal(gpu.azimuth_time_us[same], gl_t[same])


def test_bad_precision_mode(ctx):
    sc = synth.config1_scene(seed=36, n_lines=128, n_samples=256, dem_n=64)
    sc.config.precision = 7
    with pytest.raises(sd.TerrainCorrectionError) as e:
        sd.terrain_correction(sc.merged, sc.scene, sc.dem, sc.grids, sc.config, ctx=ctx)
    assert e.value.kind == "Config"


@pytest.mark.parametrize("resampling", [sd.ResamplingKernel.Bilinear, sd.ResamplingKernel.Bicubic,
                                        sd.ResamplingKernel.Lanczos3])
def test_split_zero_clipped_sigma0(ctx, resampling):
    """Calibrated sigma0 is clipped at zero by the noise subtraction: values
    interpolated between zeros and non-zeros keep 1e-4 relative (plain
    relative error, every pixel)."""
    sc = synth.config1_scene(seed=37, n_lines=1024, n_samples=2048, dem_n=256, resampling=resampling,
                             flatten=True)
    img = np.array(sc.merged.data)
    rng = np.random.default_rng(9)
    img[rng.uniform(size=img.shape) < 0.35] = 0.0
    sc.merged.data = img
    ref, ref_t, _ = oracle_cr(sc.merged, sc.scene, sc.dem, sc.grids, sc.config, return_times=True)
    sc.config.precision = SPLIT
    gpu = sd.terrain_correction(sc.merged, sc.scene, sc.dem, sc.grids, sc.config, ctx=ctx,
                                return_times=True)
    rep = compare_geocoded(gpu, ref, gpu.azimuth_time_us, ref_t, sc.scene.sub_swaths[0].azimuth_time_interval_s)
    assert rep["nan_pattern_equal"] and rep["mask_equal"], rep
    assert rep["time_mismatch_px"] == 0, rep
    assert rep["sigma_rel_over_1e-4_px"] == 0, rep


@pytest.mark.parametrize("resampling", [sd.ResamplingKernel.Bilinear, sd.ResamplingKernel.Bicubic,
                                        sd.ResamplingKernel.Lanczos3])
def test_split_matches_fp64_path_zero_clipped_full_shape(ctx, resampling):
    """Split vs the FP64 path on the config-1 shape (4096 x 8192 sigma0,
    1024^2 DEM) geocoded at a quarter of the DEM posting (4096^2 output px),
    flattening on, with 35 % of the sigma0 samples clipped to zero as the
    noise subtraction does.  Both paths share the microsecond chain, so
    times, masks, counters and the NaN pattern are equal, and every
    sigma0/gamma0 is within 1e-4 relative of the FP64 value: no pixel is
    excepted and no noise-floor metric is used."""
    sc = synth.config1_scene(seed=39, resampling=resampling, flatten=True)
    img = np.array(sc.merged.data)
    rng = np.random.default_rng(10)
    img[rng.uniform(size=img.shape) < 0.35] = 0.0
    sc.merged.data = img
    sc.config.pixel_spacing_deg = sc.config.pixel_spacing_deg / 4
    ref = sd.terrain_correction(sc.merged, sc.scene, sc.dem, sc.grids, sc.config, ctx=ctx, return_times=True)
    sc.config.precision = SPLIT
    gpu = sd.terrain_correction(sc.merged, sc.scene, sc.dem, sc.grids, sc.config, ctx=ctx, return_times=True)
    rep = compare_geocoded(gpu, ref, gpu.azimuth_time_us, ref.azimuth_time_us,
                           sc.scene.sub_swaths[0].azimuth_time_interval_s)
    assert rep["compared_px"] > 4_000_000, rep
    assert rep["time_mismatch_px"] == 0, rep
    assert rep["nan_pattern_equal"] and rep["mask_equal"], rep
    assert rep["sigma_rel_over_1e-4_px"] == 0, rep
    assert rep["cos_lia_abs_err_max"] <= 1e-5, rep
    assert gpu.newton_iter_histogram == ref.newton_iter_histogram
    assert gpu.valid_pixel_count == ref.valid_pixel_count
