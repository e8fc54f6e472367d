"""GPU speckle filters, deburst, calibration and merge vs the CPU oracle."""
import numpy as np
import pytest

import oracle
import sardine_b200 as sd
from sardine_b200 import synth

pytestmark = pytest.mark.gpu

FILTERS = [
    sd.SpeckleFilter.Boxcar(5),
    sd.SpeckleFilter.Lee(7, 4.4),
    sd.SpeckleFilter.Frost(5, 2.0),
    sd.SpeckleFilter.GammaMap(5, 4.4),
    sd.SpeckleFilter.RefinedLee(4.4),
    sd.SpeckleFilter.Boxcar(3),
    sd.SpeckleFilter.GammaMap(9, 1.0),
    sd.SpeckleFilter.Lee(3, 1.0),
    sd.SpeckleFilter.Boxcar(15),
]


# 301 columns: rows not 16-byte aligned, the window is staged with loads;
# 300 and 40: aligned rows, staged by one tensor-memory copy per block (40 x
# 20 is smaller than one block's window, so the fill covers every side)
@pytest.mark.parametrize("shape", [(173, 301), (173, 300), (20, 40)], ids=lambda s: f"{s[0]}x{s[1]}")
@pytest.mark.parametrize("flt", FILTERS, ids=lambda f: f"k{f.kind}w{f.window}")
def test_speckle_parity(ctx, flt, shape):
    rng = np.random.default_rng(3)
    rows, cols = shape
    img = rng.exponential(0.05, size=(rows, cols)).astype(np.float32)
    img[10:14, 20:40] = np.nan  # slices clip to small shapes
    img[150:, 290:] = 0.0
    # negative zeros: a window of -0.0 alone sums to +0.0 in the reference's
    # loop, and skipped taps must not change any sum's sign
    img[60:75, 100:118] = -0.0
    img[62:63, 130:140] = -0.0
    img[100:101, 7:8] = np.inf
    img[80:81, 200:201] = -np.inf
    img[5:7, 3:9] = -0.0
    img[0, :] = np.nan  # a void edge row
    ref = oracle.apply_speckle_filter(img, cols, rows, flt).reshape(rows, cols)
    out = np.asarray(sd.apply_speckle_filter(img, cols, rows, flt, ctx=ctx)).reshape(rows, cols)
    assert np.array_equal(np.isnan(out), np.isnan(ref))
    m = np.isfinite(ref)
    if flt.kind == sd._abi.SPECKLE_FROST:  # f32 exp: CUDA vs libm ulps
        rel = np.abs(out[m] - ref[m]) / np.maximum(np.abs(ref[m]), 1e-30)
        assert rel.max() < 1e-5
    else:
        assert np.array_equal(out[m], ref[m]), "bit-exact expected (same f64 sums, same f32 ops)"
        # the same bits, signed zeros included
        assert np.array_equal(out[m].view(np.uint32), ref[m].view(np.uint32))


@pytest.mark.parametrize("kind,window,enl,damp,code", [
    (0, 4, 1.0, 0.0, "BadWindow"), (0, 1, 1.0, 0.0, "BadWindow"), (1, 5, 0.0, 0.0, "BadEnl"),
    (3, 5, float("nan"), 0.0, "BadEnl"), (2, 5, 1.0, -1.0, "BadDamping"),
    (2, 5, 1.0, float("inf"), "BadDamping"), (4, 2, -1.0, 0.0, "BadEnl"),
])
def test_speckle_errors(ctx, kind, window, enl, damp, code):
    img = np.ones((8, 8), np.float32)
    with pytest.raises(sd.SpeckleError) as e:
        sd.apply_speckle_filter(img, 8, 8, sd.SpeckleFilter(kind, window, enl, damp), ctx=ctx)
    assert e.value.kind == code
    with pytest.raises(sd.SpeckleError) as e:
        sd.apply_speckle_filter(img, 7, 8, sd.SpeckleFilter.Boxcar(3), ctx=ctx)
    assert e.value.kind == "DimensionMismatch"


def test_speckle_trait_object(ctx):
    k = sd.GpuSpeckleKernel(sd.SpeckleFilter.RefinedLee(4.4), ctx=ctx)
    img = np.full((16, 16), 0.25, np.float32)
    out = sd.apply_speckle_step(img, 16, 16, k)
    assert np.allclose(out, 0.25, rtol=1e-6)
    assert sd.apply_speckle_step(img, 16, 16, None) is img


def _small_iw(seed=31):
    return synth.config2_scene(seed=seed, n_bursts=3, lines_per_burst=400, tiff_width=1200,
                               burst_step=300, swath_overlap=100, out_rows=64, out_cols=64,
                               lut_lines_step=130)


def test_deburst_calibrate_merge_bit_exact(ctx):
    sc = _small_iw()
    inputs_o, inputs_g = [], []
    for s in sc.swaths:
        deb_o = oracle.deburst_subswath(s.slc, s.sw, s.bursts)
        deb_g = sd.deburst_subswath(s.slc, s.sw, s.bursts, ctx=ctx)
        assert (deb_g.lines, deb_g.samples, deb_g.valid_sample_offset) == \
               (deb_o.lines, deb_o.samples, deb_o.valid_sample_offset)
        assert np.array_equal(np.asarray(deb_g.data), deb_o.data)
        sig_o = oracle.apply_calibration(deb_o, s.cal, s.noise, s.bursts[0].first_line)
        sig_g = sd.apply_calibration(deb_g, s.cal, s.noise, s.bursts[0].first_line, ctx=ctx)
        assert np.array_equal(np.asarray(sig_g.data), sig_o.data)
        assert np.array_equal(np.asarray(sig_g.nesz), sig_o.nesz)
        assert (sig_g.cal_lut_extrapolation_gap_px, sig_g.noise_lut_extrapolation_gap_px) == \
               (sig_o.cal_lut_extrapolation_gap_px, sig_o.noise_lut_extrapolation_gap_px)
        inputs_o.append(sd.SwathInput(sig_o, s.sw, s.bursts[0].azimuth_time_us))
        inputs_g.append(sd.SwathInput(sig_g, s.sw, s.bursts[0].azimuth_time_us))
    m_o, info = oracle.merge_subswaths(inputs_o)
    m_g = sd.merge_subswaths(inputs_g, ctx=ctx)
    assert (m_g.lines, m_g.samples) == (m_o.lines, m_o.samples)
    assert m_g.near_slant_range_time_s == m_o.near_slant_range_time_s
    assert m_g.azimuth_start_time_us == m_o.azimuth_start_time_us
    assert np.array_equal(np.asarray(m_g.data), m_o.data, equal_nan=True)
    assert np.array_equal(np.asarray(m_g.nesz), m_o.nesz, equal_nan=True)
    fused = sd.calibrate_deburst_merge(sc.swaths, ctx=ctx)
    assert np.array_equal(np.asarray(fused.data), m_o.data, equal_nan=True)
    assert np.array_equal(np.asarray(fused.nesz), m_o.nesz, equal_nan=True)


def test_deburst_errors(ctx):
    sc = _small_iw()
    s = sc.swaths[0]
    with pytest.raises(sd.DeburstError) as e:
        sd.deburst_subswath(s.slc, s.sw, [], ctx=ctx)
    assert e.value.kind == "NoBursts"
    b = [sd.BurstEntry(**vars(x)) for x in s.bursts]
    b[1].azimuth_time_us = b[0].azimuth_time_us + int(390 * synth.ATI * 1e6)
    with pytest.raises(sd.DeburstError) as e:
        sd.deburst_subswath(s.slc, s.sw, b, ctx=ctx)
    assert e.value.kind == "ImplausibleOverlap"
