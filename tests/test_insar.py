"""InSAR after deramping: co-registration resampling (resample_secondary,
insar/coreg.rs:230-264) and interferogram + coherence (form_interferogram,
insar/interferogram.rs:165-398).  The oracle against the reference's own
tests (coreg.rs:639-768, interferogram.rs:496-693) and a plain-Python
restatement, then the GPU kernels against the oracle."""
import math

import numpy as np
import pytest

import oracle
import sardine_b200 as sd
from sardine_b200 import _abi
from sardine_b200.types import (CoregPoly, Coregistered, Deramped, InterferogramConfig, OrbitData,
                                SubSwathMetadata)

T0_US = 1_548_221_628_000_000
WGS84_A, WGS84_B = 6_378_137.0, 6_356_752.314245


def _deramped(lines, samples, val=None, data=None, off=0):
    if data is None:
        data = np.tile(np.array(val, np.float32), (lines, samples, 1))
    if isinstance(data, np.ndarray):  # device tensors pass through as they are
        data = np.ascontiguousarray(data, np.float32)
    return Deramped(data, lines, samples, off)


def _orbit_at(x, y, z):
    """make_orbit_at (interferogram.rs:508-521): a fixed position, 11 vectors 10 s apart."""
    t = np.array([T0_US + int(i * 10.0 * 1e6) for i in range(-5, 6)], np.int64)
    return OrbitData(t, np.tile([x, y, z], (11, 1)).astype(np.float64),
                     np.tile([0.0, 7600.0, 0.0], (11, 1)).astype(np.float64))


def _minimal_swath():
    """minimal_swath (interferogram.rs:523-543)."""
    return SubSwathMetadata("IW1", 1, 10, 20, 2.056e-3, 2.33, 5.35e-3)


def _circular_orbit(baseline=(0.0, 0.0, 0.0)):
    """A circular, 98-degree inclined orbit 700 km up, 15 vectors 10 s apart from
    T0 - 20 s; `baseline` shifts every position (a secondary pass)."""
    r = WGS84_A + 700_000.0
    w = math.sqrt(3.986004418e14 / r ** 3)
    inc = math.radians(98.0)
    e2 = np.array([0.0, math.cos(inc), math.sin(inc)])
    ts, ps, vs = [], [], []
    for i in range(15):
        t = -20.0 + 10.0 * i
        th = 0.7 + w * t
        ts.append(T0_US + int(t * 1e6))
        ps.append(r * (math.cos(th) * np.array([1.0, 0.0, 0.0]) + math.sin(th) * e2) + np.array(baseline))
        vs.append(r * w * (-math.sin(th) * np.array([1.0, 0.0, 0.0]) + math.cos(th) * e2))
    return OrbitData(np.array(ts, np.int64), np.array(ps), np.array(vs))


def _geo_swath(lines, samples):
    """Near range 709 km at 20 m spacing: the reference's 10-iteration flat-earth
    solve converges from its nadir start only up to ~722 km for this orbit, so
    the image holds both converged pixels and pixels left at zero phase."""
    return SubSwathMetadata("IW1", 1, lines, samples, 2.055556e-3, 20.0, 2.0 * 709_000.0 / 299_792_458.0)


def _py_coherence(ig_re, ig_im, rp, sp, az, rg, phase=False):
    """interferogram.rs:334-383 in plain Python floats (sequential f64 sums)."""
    lines, samples = ig_re.shape
    ah, rh = az // 2, rg // 2
    coh = np.zeros((lines, samples), np.float32)
    ph = np.zeros((lines, samples), np.float32)
    for l in range(lines):
        for c in range(samples):
            s = [0.0, 0.0, 0.0, 0.0]
            for wl in range(max(l - ah, 0), min(l + ah + 1, lines)):
                for wc in range(max(c - rh, 0), min(c + rh + 1, samples)):
                    s[0] += float(ig_re[wl, wc])
                    s[1] += float(ig_im[wl, wc])
                    s[2] += float(rp[wl, wc])
                    s[3] += float(sp[wl, wc])
            den = math.sqrt(s[2] * s[3])
            coh[l, c] = min(math.sqrt(s[0] * s[0] + s[1] * s[1]) / den, 1.0) if den > 0 else 0.0
            ph[l, c] = math.atan2(s[1], s[0])
    return coh, ph


# ── oracle vs the reference's co-registration tests ─────────────────────────
def test_oracle_forward_geocoding_converges_on_ellipsoid():
    # coreg.rs:638-681
    p, v, rng = (4_750_000.0, 2_600_000.0, 4_540_000.0), (3_640.0, -6_664.0, 0.0), 700_000.0
    t = oracle.ecef_from_slant_range_doppler(p, v, rng, 20, 1e-3)
    assert t is not None
    tx, ty, tz = t
    assert abs(tx * tx / WGS84_A ** 2 + ty * ty / WGS84_A ** 2 + tz * tz / WGS84_B ** 2 - 1.0) < 1e-6
    assert abs(math.dist(t, p) - rng) < 1.0
    assert abs(((tx - p[0]) * v[0] + (ty - p[1]) * v[1] + (tz - p[2]) * v[2]) / rng) < 1.0


def _sec9():
    return _deramped(3, 3, data=np.array([[i, i + 1] for i in range(9)], np.float32).reshape(3, 3, 2))


def test_oracle_bilinear_integer_and_out_of_bounds():
    # coreg.rs:709-744, observed through resample_secondary with constant offsets
    sec = _sec9()
    at = lambda dl, dc, s=sec: oracle.resample_secondary(1, 1, CoregPoly([dl, 0, 0, 0, 0, 0],
                                                                         [dc, 0, 0, 0, 0, 0]), s).data[0, 0]
    assert list(at(0.0, 0.0)) == [0.0, 1.0] and list(at(1.0, 1.0)) == [4.0, 5.0]
    two = _deramped(2, 2, (1.0, 2.0))
    for dl, dc in ((-1.0, 0.0), (0.0, 5.0), (5.0, 0.0)):
        assert list(at(dl, dc, two)) == [0.0, 0.0]
    assert np.isnan(at(float("nan"), 0.0, sec)).all()  # `NaN as usize` is 0: the weights carry the NaN


def test_oracle_resample_with_zero_offset_is_identity():
    # coreg.rs:746-767
    sec = _sec9()
    r = oracle.resample_secondary(2, 2, CoregPoly([0.0] * 6, [0.0] * 6), sec)
    assert np.array_equal(r.data, sec.data[:2, :2])


# ── oracle vs the reference's interferogram tests ───────────────────────────
def _igram(ref_val, sec_val, lines, samples, cfg):
    orb = _orbit_at(7_071_000.0, 0.0, 0.0)
    co = Coregistered(_deramped(lines, samples, ref_val), _deramped(lines, samples, sec_val))
    return oracle.form_interferogram(co, _minimal_swath(), orb, T0_US, orb, 0.0555, cfg)


def test_oracle_same_scene_coherence_is_unity():
    # interferogram.rs:545-575
    rc, g = _igram((1.0, 0.0), (1.0, 0.0), 40, 80, InterferogramConfig(4, 8, False))
    assert rc == 0 and (g.lines, g.samples) == (40, 80) and g.phase is None
    assert np.all(np.abs(g.coherence[4:-4, 8:-8] - 1.0) < 1e-4)


def test_oracle_zero_secondary_gives_zero_coherence():
    # interferogram.rs:577-600
    rc, g = _igram((1.0, 0.0), (0.0, 0.0), 20, 40, InterferogramConfig())
    assert rc == 0 and np.all(g.coherence == 0.0)


def test_oracle_phase_output_populated_when_requested():
    # interferogram.rs:602-628
    rc, g = _igram((1.0, 0.0), (0.0, 1.0), 10, 20, InterferogramConfig(2, 4, True))
    assert rc == 0 and g.phase.shape == (10, 20)
    assert abs(g.phase[5, 10] + math.pi / 2) < 0.1


def test_oracle_zero_window_and_orbit_errors():
    # interferogram.rs:630-645; a line time outside the orbit is InsarError::Orbit
    assert _igram((1.0, 0.0), (1.0, 0.0), 10, 20, InterferogramConfig(0, 4))[0] == \
        _abi.SD_ERR_INSAR_INVALID_WINDOW_SIZE
    orb = _orbit_at(7_071_000.0, 0.0, 0.0)
    co = Coregistered(_deramped(4, 4, (1.0, 0.0)), _deramped(4, 4, (1.0, 0.0)))
    assert oracle.form_interferogram(co, _minimal_swath(), orb, T0_US + 60_000_000, orb, 0.0555)[0] == \
        _abi.SD_ERR_INSAR_ORBIT


def test_oracle_flat_earth_phase_is_zero_same_orbit():
    # interferogram.rs:647-667
    rc, g = _igram((1.0, 0.0), (1.0, 0.0), 8, 16, InterferogramConfig(2, 4, True))
    assert rc == 0 and abs(g.phase[4, 8]) < 0.01


def test_oracle_coherence_equals_python_restatement():
    """The reference tests' geometry (802 km range from a 700 km altitude): the
    10-iteration flat-earth solve does not converge from its nadir start, so
    the flat-earth phase is zero and the igram is ref conj(sec)."""
    rng = np.random.default_rng(7)
    lines, samples = 14, 23
    ref = rng.normal(0, 30, (lines, samples, 2)).astype(np.float32)
    sec = (ref + rng.normal(0, 15, ref.shape)).astype(np.float32)
    orb = _orbit_at(7_071_000.0, 0.0, 0.0)
    co = Coregistered(_deramped(lines, samples, data=ref), _deramped(lines, samples, data=sec))
    rc, g = oracle.form_interferogram(co, _minimal_swath(), orb, T0_US, orb, 0.0555, InterferogramConfig(5, 7, True))
    assert rc == 0
    r64, s64 = ref.astype(np.float64), sec.astype(np.float64)
    ig_re = (r64[..., 0] * s64[..., 0] + r64[..., 1] * s64[..., 1]).astype(np.float32)
    ig_im = (r64[..., 1] * s64[..., 0] - r64[..., 0] * s64[..., 1]).astype(np.float32)
    rp = ref[..., 0] * ref[..., 0] + ref[..., 1] * ref[..., 1]
    sp = sec[..., 0] * sec[..., 0] + sec[..., 1] * sec[..., 1]
    coh, ph = _py_coherence(ig_re, ig_im, rp, sp, 5, 7)
    assert np.array_equal(g.coherence, coh) and np.array_equal(g.phase, ph)


# ── GPU vs oracle ────────────────────────────────────────────────────────────
def _pair(lines, samples, seed, noise=20.0):
    rng = np.random.default_rng(seed)
    ref = rng.normal(0, 40, (lines, samples, 2)).astype(np.float32)
    sec = (ref + rng.normal(0, noise, ref.shape)).astype(np.float32)
    return ref, sec


@pytest.mark.gpu
@pytest.mark.parametrize("lines,samples,sl,ss", [(2, 2, 3, 3), (417, 1203, 430, 1250), (64, 300, 70, 290)])
def test_gpu_resample_bit_exact(ctx, lines, samples, sl, ss):
    import torch
    rng = np.random.default_rng(lines)
    sec = _deramped(sl, ss, data=rng.normal(0, 50, (sl, ss, 2)).astype(np.float32), off=11)
    poly = CoregPoly([0.37, 1.2e-4, -3e-5, 2e-8, -1e-9, 3e-9], [-0.81, 2e-5, 4.1e-4, -1e-9, 2e-9, 1e-8])
    if lines == 2:
        poly = CoregPoly([0.0] * 6, [0.0] * 6)
    want = oracle.resample_secondary(lines, samples, poly, sec)
    for kind in ("host", "device"):
        src = sec if kind == "host" else _deramped(sl, ss, data=torch.from_numpy(sec.data).cuda(), off=11)
        got = sd.resample_secondary(lines, samples, poly, src, ctx=ctx)
        assert got.valid_sample_offset == 11
        gd = got.data if kind == "host" else got.data.cpu().numpy()
        assert np.array_equal(np.asarray(gd).view(np.uint32), want.data.view(np.uint32))


def _close(got, want, rtol, atol=0.0, frac=0.99):
    """Equal except where CUDA's and the C library's FP64 sincos (or atan2)
    differ in the last bit and that survives the f32 rounding of a term."""
    got = np.asarray(got)
    assert np.all(np.abs(got.astype(np.float64) - want) <= atol + rtol * np.abs(want))
    assert np.mean(got == want) >= frac


@pytest.mark.gpu
@pytest.mark.parametrize("lines,samples,az,rg,phase", [(40, 80, 4, 8, False), (300, 1000, 10, 40, True),
                                                       (150, 260, 80, 40, True), (37, 129, 3, 300, False)])
def test_gpu_interferogram_matches_oracle(ctx, lines, samples, az, rg, phase):
    """Realistic geometry: an inclined circular orbit and a secondary 100-200 m
    away, so the flat-earth phase has dense fringes.  (150, 260, 80, 40) and
    (37, 129, 3, 300) have windows too large for the shared-memory tile."""
    import torch
    ref, sec = _pair(lines, samples, lines + samples)
    sw = _geo_swath(lines, samples)
    ro, so = _circular_orbit(), _circular_orbit((110.0, -60.0, 150.0))
    co = Coregistered(_deramped(lines, samples, data=ref, off=57), _deramped(lines, samples, data=sec, off=57))
    cfg = InterferogramConfig(az, rg, phase)
    rc, want = oracle.form_interferogram(co, sw, ro, T0_US, so, 0.05546576, cfg)
    assert rc == 0
    for kind in ("host", "device"):
        c2 = co if kind == "host" else Coregistered(
            _deramped(lines, samples, data=torch.from_numpy(ref).cuda(), off=57),
            _deramped(lines, samples, data=torch.from_numpy(sec).cuda(), off=57))
        got = sd.form_interferogram(c2, sw, ro, T0_US, so, 0.05546576, cfg, ctx=ctx)
        gc = got.coherence if kind == "host" else got.coherence.cpu().numpy()
        _close(gc, want.coherence, rtol=2e-6, atol=1e-7)
        if phase:
            gp = got.phase if kind == "host" else got.phase.cpu().numpy()
            _close(gp, want.phase, rtol=0.0, atol=1e-5)
        else:
            assert got.phase is None


@pytest.mark.gpu
def test_gpu_flat_earth_phase_matches_oracle(ctx):
    """A unit pair and a 1 x 1 window: the phase output is the wrapped
    flat-earth phase of every pixel (the Newton solve on the device)."""
    lines, samples = 50, 700
    sw = _geo_swath(lines, samples)
    ro, so = _circular_orbit(), _circular_orbit((110.0, -60.0, 150.0))
    co = Coregistered(_deramped(lines, samples, (1.0, 0.0)), _deramped(lines, samples, (1.0, 0.0)))
    cfg = InterferogramConfig(1, 1, True)
    rc, want = oracle.form_interferogram(co, sw, ro, T0_US, so, 0.05546576, cfg)
    assert rc == 0 and np.ptp(want.phase) > 6.0 and 0.1 < np.mean(want.phase == 0.0) < 0.9  # fringes wrap
    got = sd.form_interferogram(co, sw, ro, T0_US, so, 0.05546576, cfg, ctx=ctx)
    _close(got.phase, want.phase, rtol=0.0, atol=2e-6)
    _close(got.coherence, want.coherence, rtol=1.2e-7)


@pytest.mark.gpu
def test_gpu_interferogram_reference_cases_and_errors(ctx):
    orb = _orbit_at(7_071_000.0, 0.0, 0.0)
    co = Coregistered(_deramped(40, 80, (1.0, 0.0)), _deramped(40, 80, (1.0, 0.0)))
    g = sd.form_interferogram(co, _minimal_swath(), orb, T0_US, orb, 0.0555, InterferogramConfig(4, 8), ctx=ctx)
    assert np.all(np.abs(g.coherence[4:-4, 8:-8] - 1.0) < 1e-4)
    co0 = Coregistered(_deramped(20, 40, (1.0, 0.0)), _deramped(20, 40, (0.0, 0.0)))
    assert np.all(sd.form_interferogram(co0, _minimal_swath(), orb, T0_US, orb, 0.0555, ctx=ctx).coherence == 0)
    with pytest.raises(sd.InsarError) as e:
        sd.form_interferogram(co, _minimal_swath(), orb, T0_US, orb, 0.0555, InterferogramConfig(0, 4), ctx=ctx)
    assert e.value.kind == "InvalidWindowSize"
    with pytest.raises(sd.InsarError) as e:
        sd.form_interferogram(co, _minimal_swath(), orb, T0_US + 60_000_000, orb, 0.0555, ctx=ctx)
    assert e.value.kind == "Orbit"


# ── sparse co-registration offsets (compute_coreg_offsets) ──────────────────
def test_oracle_poly_fit_recovers_linear_offset():
    # coreg.rs:683-706
    pts = [(i * 10.0, j * 50.0, 0.5, 0.0) for i in range(100) for j in range(10)]
    rc, coef, rms = oracle.fit_poly6(pts, 2)
    assert rc == 0 and abs(coef[0] - 0.5) < 1e-9 and rms < 1e-10


def _coreg_case(realistic=False, lines=1500, samples=4000):
    """realistic: the inclined circular orbits (200 m baseline), secondary
    0.31 s later.  Otherwise the reference tests' fixed-position orbit for
    both passes (interferogram.rs:508-521, moved off the equator), where the zero-Doppler residual
    after forward geocoding is far below 1 ns, so every point converges."""
    if realistic:
        sw = SubSwathMetadata("IW1", 1, lines, samples, 2.055556e-3, 20.0, 2.0 * 712_000.0 / 299_792_458.0)
        ro, so, ts = _circular_orbit(), _circular_orbit((110.0, -60.0, 150.0)), T0_US + 310_000
    else:
        sw = SubSwathMetadata("IW1", 1, lines, samples, 2.055556e-3, 20.0, 2.0 * 712_000.0 / 299_792_458.0)
        ro = so = _orbit_at(6_000_000.0, 0.0, 3_741_857.0)  # 7071 km out, off the equator
        ts = T0_US
    sec_sw = SubSwathMetadata("IW1", 1, lines, samples, sw.azimuth_time_interval_s, 20.0, sw.slant_range_time_s,
                              first_sample=3)
    return sw, ro, T0_US, Deramped(None, lines, samples, 5), sec_sw, so, ts


def test_oracle_coreg_offsets_fixed_orbit():
    """Same fixed state for every line of both passes: the secondary line is
    0, so dl = -l, and dc = ref offset - first_sample; the fit recovers them."""
    rc, r = oracle.compute_coreg_offsets(*_coreg_case())
    assert rc == 0 and r.n_valid == 1000
    assert np.allclose(r.poly.az, [0, -1, 0, 0, 0, 0], atol=1e-6) and abs(r.poly.rg[0] - 2.0) < 1e-3
    assert r.fit_residual_rms < 1e-6


def test_oracle_coreg_offsets_realistic_orbit_fails_like_the_reference():
    """solve_zero_doppler steps in whole microseconds (terrain_correction.rs
    :1066) but asks for |delta| < 1e-9 s (coreg.rs:381), so on real orbits a
    point converges only when its zero-Doppler time lies within 1 ns of a
    whole microsecond: the grid comes out too small."""
    rc, _ = oracle.compute_coreg_offsets(*_coreg_case(realistic=True))
    assert rc == _abi.SD_ERR_INSAR_COREG_GRID_TOO_SMALL
    assert oracle.coreg_n_valid(*_coreg_case(realistic=True)) == (rc, 4)


@pytest.mark.gpu
def test_gpu_coreg_offsets_match_oracle(ctx):
    case = _coreg_case()
    rc, want = oracle.compute_coreg_offsets(*case)
    assert rc == 0
    got = sd.compute_coreg_offsets(*case, ctx=ctx)
    assert got.n_valid == want.n_valid
    assert got.poly.az == want.poly.az and got.poly.rg == want.poly.rg
    assert got.fit_residual_rms == want.fit_residual_rms


@pytest.mark.gpu
def test_gpu_coreg_grid_too_small(ctx):
    """The error kind and the number of grid points that converged before it:
    on the realistic orbit the microsecond stepping lets 4 of 1000 converge,
    and the device must find the same 4."""
    from sardine_b200 import _coreg_offsets_raw
    for case, n in ((_coreg_case(realistic=True), 4),
                    (_coreg_case()[:2] + (T0_US + 500_000_000,) + _coreg_case()[3:], 0)):
        rc, n_oracle = oracle.coreg_n_valid(*case)
        assert rc == _abi.SD_ERR_INSAR_COREG_GRID_TOO_SMALL and n_oracle == n
        with pytest.raises(sd.InsarError) as e:
            sd.compute_coreg_offsets(*case, ctx=ctx)
        assert e.value.kind == "CoregGridTooSmall"
        rc, r = _coreg_offsets_raw(*case, ctx)
        assert rc == _abi.SD_ERR_INSAR_COREG_GRID_TOO_SMALL
        assert int(r.n_valid) == n_oracle
