"""Pre-TC multilook (apply_multilook, scene_prep.rs:1060-1160): the oracle
against the reference's own tests (run.rs:1451-1595), the GPU boxcar
against the oracle bit for bit, and the geometry update."""
import numpy as np
import pytest

import oracle
import sardine_b200 as sd

RPS_S = 2.329562 / 299_792_458.0 * 2.0


def _merged(data, nesz=None, lines=None, samples=None):
    if isinstance(data, (list, np.ndarray)):  # torch tensors pass through as they are
        data = np.asarray(data, np.float32)
        nesz = np.full_like(data, 0.01) if nesz is None else np.asarray(nesz, np.float32)
    lines = lines or data.shape[0]
    samples = samples or data.shape[1]
    return sd.MergedSigma0(data, lines, samples, 0.005300, RPS_S, 2.329562, 0, 0, nesz, 1_548_221_628_000_000)


def test_oracle_multilook_kats():
    # run.rs:1483-1526
    rc, d, _ = oracle.multilook(np.array([[1, 1, 5, 5]], np.float32), np.full((1, 4), 0.01, np.float32), 1, 4, 2, 1)
    assert rc == 0 and np.allclose(d, [[1.0, 5.0]])
    rc, d, _ = oracle.multilook(np.array([[1, 3, 5, 7], [2, 4, 6, 8]], np.float32),
                                np.full((2, 4), 0.01, np.float32), 2, 4, 2, 1)
    assert np.array_equal(d, np.array([[2, 6], [3, 7]], np.float32))
    rc, d, n = oracle.multilook(np.array([[np.nan, 4.0]], np.float32), np.array([[np.nan, 0.1]], np.float32),
                                1, 2, 2, 1)
    assert d[0, 0] == np.float32(4.0) and abs(n[0, 0] - 0.1) < 1e-6
    rc, d, _ = oracle.multilook(np.full((1, 2), np.nan, np.float32), np.full((1, 2), 0.01, np.float32), 1, 2, 2, 1)
    assert np.isnan(d[0, 0])
    # run.rs:1573-1594: zero and oversized factors are errors
    assert oracle.multilook(np.ones((2, 4), np.float32), np.ones((2, 4), np.float32), 2, 4, 0, 1)[0] != 0
    assert oracle.multilook(np.ones((2, 4), np.float32), np.ones((2, 4), np.float32), 2, 4, 8, 1)[0] != 0


@pytest.mark.gpu
def test_gpu_multilook_kats_and_geometry(ctx):
    m = _merged(np.full((4, 8), 2.0))
    assert sd.apply_multilook(m, 1, 1, 0.0, ctx=ctx) is m                      # run.rs:1472-1481
    out = sd.apply_multilook(_merged([[1, 3, 5, 7], [2, 4, 6, 8]]), 2, 1, 0.0, ctx=ctx)
    assert np.array_equal(out.data, np.array([[2, 6], [3, 7]], np.float32))
    out = sd.apply_multilook(_merged([[np.nan, 4.0]], [[np.nan, 0.1]]), 2, 1, 0.0, ctx=ctx)
    assert out.data[0, 0] == 4.0 and abs(out.nesz[0, 0] - 0.1) < 1e-6
    m = _merged(np.ones((2, 8)))
    out = sd.apply_multilook(m, 4, 1, 0.0, ctx=ctx)                            # run.rs:1533-1551
    assert (out.samples, out.lines) == (2, 2)
    assert abs(out.range_pixel_spacing_s - 4 * m.range_pixel_spacing_s) < 1e-25
    assert abs(out.range_pixel_spacing_m - 4 * m.range_pixel_spacing_m) < 1e-12
    assert abs(out.near_slant_range_time_s - (m.near_slant_range_time_s + 1.5 * m.range_pixel_spacing_s)) < 1e-25
    m = _merged(np.ones((4, 2)))
    out = sd.apply_multilook(m, 1, 2, 2.055e-3, ctx=ctx)                       # run.rs:1555-1569
    assert (out.lines, out.samples) == (2, 2)
    assert out.azimuth_start_time_us == m.azimuth_start_time_us + int(0.5 * 2.055e-3 * 1e6)
    for r, a in ((0, 1), (8, 1)):                                              # run.rs:1573-1594
        with pytest.raises(sd.SardineError) as e:
            sd.apply_multilook(_merged(np.ones((2, 4))), r, a, 0.0, ctx=ctx)
        assert "multilook" in str(e.value)


@pytest.mark.gpu
@pytest.mark.parametrize("lines,samples,r,a", [(257, 1031, 4, 1), (301, 499, 5, 3), (64, 64, 1, 7)])
def test_gpu_multilook_bit_exact(ctx, lines, samples, r, a):
    import torch
    rng = np.random.default_rng(lines + samples)
    d = rng.exponential(0.05, (lines, samples)).astype(np.float32)
    d[rng.random((lines, samples)) < 0.2] = np.nan
    d[:, : 2 * r] = np.nan  # whole NaN blocks at the swath edge
    n = rng.uniform(0.001, 0.02, (lines, samples)).astype(np.float32)
    rc, rd, rn = oracle.multilook(d, n, lines, samples, r, a)
    assert rc == 0
    for kind in ("host", "device"):
        src = _merged(d, n) if kind == "host" else _merged(torch.from_numpy(d).cuda(), torch.from_numpy(n).cuda(),
                                                           lines, samples)
        out = sd.apply_multilook(src, r, a, 2.055e-3, ctx=ctx)
        od = out.data if kind == "host" else out.data.cpu().numpy()
        on = out.nesz if kind == "host" else out.nesz.cpu().numpy()
        assert np.array_equal(od.view(np.uint32), rd.view(np.uint32))
        assert np.array_equal(on.view(np.uint32), rn.view(np.uint32))
