"""Ground-range projection (to_ground_range, ground_range.rs:303-427): the
oracle against the reference's own tests (ground_range.rs:533-748) and a
numpy restatement, then the fused GPU kernel against the oracle bit for bit."""
import math

import numpy as np
import pytest

import oracle
import sardine_b200 as sd
from sardine_b200 import _abi
from sardine_b200.types import GeolocationGridPoint as GP

C_LIGHT = 299_792_458.0


def _merged(data, near=5.0e-3, rps_m=2.33):
    data = np.asarray(data, np.float32) if isinstance(data, (list, np.ndarray)) else data
    lines, samples = data.shape
    return sd.MergedSigma0(data, lines, samples, near, rps_m * 2.0 / C_LIGHT, rps_m, 0, 0, data, 0)


def _grid_one_swath(near, rps_s, n_cols, lines=(0, 50, 99), inc0=30.0, inc1=36.0, step=50):
    """ground_range.rs:640-660: 3 azimuth rows x 5 points, incidence linear in pixel
    (points every `step` pixels; the reference's test uses 50 over 200 columns)."""
    pts = []
    for line in lines:
        for i in range(5):
            pixel = i * step
            frac = pixel / (n_cols - 1)
            pts.append(GP(0, 50.0, 8.0, near + pixel * rps_s, line, inc0 + frac * (inc1 - inc0)))
    return [("IW1", pts)]


def _grids_three_swaths(near, rps_s, samples):
    """Three overlapping sub-swaths over the merged columns (IW seams), incidence 30-46 deg."""
    out = []
    bounds = [(0, samples * 0.40), (samples * 0.33, samples * 0.72), (samples * 0.66, samples - 1)]
    for k, (c0, c1) in enumerate(bounds):
        pts = []
        for line in (0, 400, 800, 1200):
            for i in range(21):
                c = c0 + (c1 - c0) * i / 20
                inc = 30.0 + 16.0 * c / samples + 0.01 * (line / 1200.0)
                pts.append(GP(0, 0.0, 0.0, near + c * rps_s, line, inc))
        out.append((f"IW{k + 1}", pts[::-1]))  # unsorted on purpose
    return out


def _numpy_grd(m, grids, target, az_sp):
    """A numpy restatement for a single-swath grid (no seams, no extrapolation)."""
    (_, pts), = grids
    lines = sorted({p.line for p in pts})
    mid = lines[len(lines) // 2]
    row = sorted([(p.slant_range_time_s, p.incidence_angle_deg) for p in pts if p.line == mid])
    t = np.array([r[0] for r in row])
    a = np.array([r[1] for r in row])
    st = m.near_slant_range_time_s + np.arange(m.samples) * m.range_pixel_spacing_s
    ang = []
    for s in st:
        i = int(np.searchsorted(t, s, "left"))
        if i < len(t) and t[i] == s:
            ang.append(a[i])
        else:
            f = (s - t[i - 1]) / (t[i] - t[i - 1])
            ang.append(a[i - 1] + f * (a[i] - a[i - 1]))
    gs = [m.range_pixel_spacing_m / math.sin(x * (math.pi / 180.0)) for x in ang]
    cum = [0.0]
    acc = 0.0
    for i in range(1, m.samples):
        acc += (gs[i - 1] + gs[i]) / 2.0
        cum.append(acc)
    os_ = int(math.floor(cum[-1] / target))
    al = int(max(round(target / az_sp), 1.0))
    cum = np.array(cum)
    proj = np.full((m.lines, os_), np.nan, np.float32)
    d = np.asarray(m.data, np.float32)
    for j in range(os_):
        tg = j * target
        i = int(np.searchsorted(cum, tg, "left"))
        if i < len(cum) and cum[i] == tg:
            proj[:, j] = d[:, i]
        elif i >= len(cum):
            proj[:, j] = d[:, -1]
        else:
            f = np.float32((tg - cum[i - 1]) / (cum[i] - cum[i - 1]))
            v0, v1 = d[:, i - 1], d[:, i]
            proj[:, j] = np.where(np.isnan(v0) | np.isnan(v1), np.float32(np.nan), v0 + (v1 - v0) * f)
    ol = m.lines // al
    out = np.full((ol, os_), np.nan, np.float32)
    for o in range(ol):
        blk = proj[o * al:(o + 1) * al].astype(np.float64)
        cnt = (~np.isnan(blk)).sum(0)
        s = np.zeros(os_)
        for k in range(al):  # sequential f64 sums, line order
            s = s + np.where(np.isnan(blk[k]), 0.0, blk[k])
        out[o] = np.where(cnt > 0, (s / np.maximum(cnt, 1)).astype(np.float32), np.float32(np.nan))
    return out


# ── oracle ───────────────────────────────────────────────────────────────────
def test_oracle_synthetic_uniform():
    # ground_range.rs:621-683
    m = _merged(np.full((100, 200), 0.1))
    rc, g = oracle.to_ground_range(m, _grid_one_swath(5.0e-3, m.range_pixel_spacing_s, 200), 10.0, 14.08)
    assert rc == 0
    assert 0 < g.samples < 200 and g.lines > 0 and g.range_pixel_spacing_m == 10.0
    valid = g.data[~np.isnan(g.data)]
    assert valid.size and abs(valid.astype(np.float64).mean() - 0.1) < 0.001


def test_oracle_rejects():
    # ground_range.rs:686-748
    m = _merged(np.ones((10, 10)))
    assert oracle.to_ground_range(sd.MergedSigma0(np.zeros(0, np.float32), 0, 0, 5e-3, 1e-8, 2.33, 0, 0,
                                                  np.zeros(0, np.float32), 0), [], 10.0, 14.08)[0] \
        == _abi.SD_ERR_GRD_EMPTY_IMAGE
    assert oracle.to_ground_range(m, [], -10.0, 14.08)[0] == _abi.SD_ERR_GRD_INVALID_SPACING
    for az in (0.0, -1.0, float("nan")):
        assert oracle.to_ground_range(m, [], 10.0, az)[0] == _abi.SD_ERR_GRD_INVALID_AZIMUTH_SPACING
    assert oracle.to_ground_range(m, [], 10.0, 14.08)[0] == _abi.SD_ERR_GRD_INTERPOLATION_FAILED
    assert oracle.to_ground_range(m, [("IW2", [])], 10.0, 14.08)[0] == _abi.SD_ERR_GRD_NO_GRID_POINTS


def test_oracle_interpolator_points():
    # ground_range.rs:560-604: 5.0 ms -> 30 deg, 6.0 ms -> 36 deg, midpoint 33 deg; observed through the
    # ground spacing of a 3-column image whose columns sit exactly on those times
    pts = [GP(0, 50.0, 8.0, 5.0e-3, 100, 30.0), GP(0, 50.0, 9.0, 6.0e-3, 100, 36.0)]
    m = sd.MergedSigma0(np.ones((1, 3), np.float32), 1, 3, 5.0e-3, 0.5e-3, 2.33, 0, 0, np.ones((1, 3), np.float32), 0)
    rc, g = oracle.to_ground_range(m, [("IW1", pts)], 1.0, 1.0)
    gs = [2.33 / math.sin(a * (math.pi / 180.0)) for a in (30.0, 33.0, 36.0)]
    assert rc == 0 and g.samples == math.floor((gs[0] + gs[1]) / 2.0 + (gs[1] + gs[2]) / 2.0)
    # outside the grid's range (beyond the 1 % extrapolation band): interpolation fails
    m2 = sd.MergedSigma0(np.ones((1, 3), np.float32), 1, 3, 6.5e-3, 0.5e-3, 2.33, 0, 0, np.ones((1, 3), np.float32), 0)
    assert oracle.to_ground_range(m2, [("IW1", pts)], 1.0, 1.0)[0] == _abi.SD_ERR_GRD_INTERPOLATION_FAILED


def test_oracle_equals_numpy_restatement():
    rng = np.random.default_rng(4)
    d = rng.exponential(0.05, (37, 260)).astype(np.float32)
    d[rng.random(d.shape) < 0.1] = np.nan
    m = _merged(d)
    grids = _grid_one_swath(5.0e-3, m.range_pixel_spacing_s, 260, lines=(0, 10, 20, 30), step=65)
    rc, g = oracle.to_ground_range(m, grids, 7.5, 2.6)
    assert rc == 0
    want = _numpy_grd(m, grids, 7.5, 2.6)
    assert np.array_equal(g.data.view(np.uint32), want.view(np.uint32))


# ── GPU vs oracle ────────────────────────────────────────────────────────────
@pytest.mark.gpu
@pytest.mark.parametrize("lines,samples,target,az", [(100, 200, 10.0, 14.08), (1203, 4001, 10.0, 2.3),
                                                     (64, 901, 4.0, 13.9)])
def test_gpu_grd_bit_exact(ctx, lines, samples, target, az):
    import torch
    rng = np.random.default_rng(lines)
    d = rng.exponential(0.05, (lines, samples)).astype(np.float32)
    d[rng.random(d.shape) < 0.15] = np.nan
    d[:, :3] = np.nan
    m = _merged(d)
    grids = (_grid_one_swath(5.0e-3, m.range_pixel_spacing_s, samples) if samples == 200
             else _grids_three_swaths(5.0e-3, m.range_pixel_spacing_s, samples))
    rc, g = oracle.to_ground_range(m, grids, target, az)
    assert rc == 0
    for kind in ("host", "device"):
        src = m if kind == "host" else _merged(torch.from_numpy(d).cuda())
        got = sd.to_ground_range(src, grids, target, az, ctx=ctx)
        assert (got.lines, got.samples, got.azimuth_looks, got.range_looks) == \
            (g.lines, g.samples, g.azimuth_looks, g.range_looks)
        assert got.azimuth_pixel_spacing_m == g.azimuth_pixel_spacing_m
        gd = got.data if kind == "host" else got.data.cpu().numpy()
        assert np.array_equal(np.ascontiguousarray(gd).view(np.uint32), g.data.view(np.uint32))


@pytest.mark.gpu
def test_gpu_grd_errors(ctx):
    m = _merged(np.ones((10, 10)))
    cases = [((m, [], -10.0, 14.08), "InvalidSpacing"), ((m, [], 10.0, 0.0), "InvalidAzimuthSpacing"),
             ((m, [], 10.0, 14.08), "InterpolationFailed"), ((m, [("IW2", [])], 10.0, 14.08), "NoGridPoints")]
    for args, kind in cases:
        with pytest.raises(sd.GroundRangeError) as e:
            sd.to_ground_range(*args, ctx=ctx)
        assert e.value.kind == kind
