"""Output path: dB conversion with the run's dB statistics, overview
downsampling and the Cloud-Optimised GeoTIFF writer.

CPU tests pin the oracle to the reference's own tests (export.rs:1227-1727);
GPU tests compare the sm_100a path with the oracle: counts, NaN pattern and
file bytes exactly, dB values within 4 ulps (CUDA log10f against glibc
log10f, both within 2 ulps of the exact value)."""
import os
import struct

import numpy as np
import pytest

import oracle
import sardine_b200 as sd

WGS = sd.OutputCrs.wgs84()
GT = [8.0, 0.0001, 0.0, 52.0, 0.0, -0.0001]


def _ulps(a, b):
    """|a - b| in units of the float32 spacing at the larger magnitude."""
    a = np.asarray(a, np.float32)
    b = np.asarray(b, np.float32)
    sp = np.spacing(np.maximum(np.abs(a), np.abs(b)).astype(np.float32))
    return np.abs(a.astype(np.float64) - b.astype(np.float64)) / sp.astype(np.float64)


def _ifd_tags(buf, off):
    n = struct.unpack_from("<H", buf, off)[0]
    tags = {}
    for k in range(n):
        tag, typ, cnt, val = struct.unpack_from("<HHII", buf, off + 2 + 12 * k)
        tags[tag] = (typ, cnt, val)
    nxt = struct.unpack_from("<I", buf, off + 2 + 12 * n)[0]
    return n, tags, nxt


def _raster(rows, cols, seed):
    rng = np.random.default_rng(seed)
    d = rng.exponential(0.05, size=(rows, cols)).astype(np.float32)
    d[rng.random((rows, cols)) < 0.07] = np.nan
    d[rng.random((rows, cols)) < 0.05] = 0.0
    d[: rows // 7, : cols // 5] = np.nan  # an all-NaN corner (whole overview patches)
    return d


# ── oracle vs the reference's known answers ─────────────────────────────────
def test_oracle_to_db_kats():
    # export.rs:1227-1275
    d = np.array([1.0, 10.0], np.float32)
    assert oracle.to_db_inplace(d, 0.0) == (2, 0)
    assert abs(d[0]) < 1e-5 and abs(d[1] - 10.0) < 1e-5
    d = np.array([0.0, -0.001, 0.5], np.float32)
    assert oracle.to_db_inplace(d, 0.0) == (1, 2)
    assert np.isnan(d[0]) and np.isnan(d[1]) and np.isfinite(d[2])
    d = np.array([0.005, 0.05], np.float32)
    assert oracle.to_db_inplace(d, 0.01) == (1, 1)
    assert np.isnan(d[0]) and np.isfinite(d[1])
    d = np.array([np.nan, 1.0], np.float32)
    assert oracle.to_db_inplace(d, 0.0) == (1, 0) and np.isnan(d[0])
    with pytest.raises(oracle.OracleError):
        oracle.to_db_inplace(np.array([1.0], np.float32), -0.001)


def test_oracle_downsample_kats():
    # export.rs:1695-1727
    d = oracle.downsample_2x(np.arange(16, dtype=np.float32), 4, 4)
    assert np.array_equal(d, np.array([[2.5, 4.5], [10.5, 12.5]], np.float32))
    s = np.full(4, np.nan, np.float32)
    s[0] = 1.0
    assert oracle.downsample_2x(s, 2, 2)[0, 0] == 1.0
    assert np.isnan(oracle.downsample_2x(np.full(4, np.nan, np.float32), 2, 2)[0, 0])


def test_oracle_db_stats_restated():
    # run.rs:63-97, restated in numpy on a raster with more than 100000 finite values
    rng = np.random.default_rng(1)
    d = (rng.normal(-12, 4, 250_001)).astype(np.float32)
    d[rng.random(d.size) < 0.1] = np.nan
    d[5] = np.inf
    fin = d[np.isfinite(d)]
    stride = max(fin.size // 100000, 1)
    sample = np.sort(fin[::stride])
    mn, mx, mean, med = oracle.db_stats(d)
    assert mn == fin.min() and mx == fin.max() and med == sample[sample.size // 2]
    assert mean == np.float32(np.sum(fin.astype(np.float64)) / fin.size) or abs(mean - fin.mean()) < 1e-5
    assert all(np.isnan(oracle.db_stats(np.full(3, np.nan, np.float32))))


def test_oracle_cog_rejects(tmp_path):
    # export.rs:1583-1604
    d = np.ones(4, np.float32)
    for ts in (100, 32, 8192):
        assert oracle.write_cog(str(tmp_path / "a.tif"), d, 2, 2, GT, WGS, ts) == sd._abi.SD_ERR_EXPORT_INVALID_TILE_SIZE
    bad = [8.0, 0.0, 0.0, 52.0, 0.0, -0.0001]
    assert oracle.write_cog(str(tmp_path / "b.tif"), d, 2, 2, bad, WGS, 512) == sd._abi.SD_ERR_EXPORT_INVALID_GEOTRANSFORM


def test_oracle_cog_header_and_ramp(tmp_path):
    # export.rs:1606-1693
    rows, cols = 512, 1024
    data = (np.arange(rows * cols, dtype=np.float32) * np.float32(0.001)).reshape(rows, cols)
    p = str(tmp_path / "h.tif")
    assert oracle.write_cog(p, data, cols, rows, GT, WGS, 512) == 0
    buf = open(p, "rb").read()
    assert buf[:4] == b"II\x2a\x00"
    off = struct.unpack_from("<I", buf, 4)[0]
    assert 0 < off < len(buf) and struct.unpack_from("<H", buf, off)[0] == 17

    ramp = np.arange(64 * 64, dtype=np.float32).reshape(64, 64)
    p = str(tmp_path / "r.tif")
    assert oracle.write_cog(p, ramp, 64, 64, [0.0, 0.001, 0.0, 1.0, 0.0, -0.001], WGS, 64) == 0
    buf = open(p, "rb").read()
    n0, t0, ifd1 = _ifd_tags(buf, struct.unpack_from("<I", buf, 4)[0])
    assert t0[256][2] == 32 and t0[257][2] == 32  # the one overview level, 32 x 32
    n1, t1, nxt = _ifd_tags(buf, ifd1)
    assert n1 == 17 and nxt == 0 and t1[256][2] == 64
    tile_at = struct.unpack_from("<I", buf, t1[324][2])[0]  # TileOffsets points to a 1-entry array
    tile = np.frombuffer(buf, np.float32, 64 * 64, tile_at)
    assert tile[0] == 0.0 and tile[64] == 64.0 and tile[-1] == 4095.0
    # the overview tile: the 32 x 32 means in the top-left corner, NaN padding elsewhere
    ov_at = struct.unpack_from("<I", buf, t0[324][2])[0]
    ov = np.frombuffer(buf, np.float32, 64 * 64, ov_at).reshape(64, 64)
    assert np.array_equal(ov[:32, :32], oracle.downsample_2x(ramp, 64, 64))
    assert np.isnan(ov[32:, :]).all() and np.isnan(ov[:, 32:]).all()


def test_oracle_cog_utm_geokeys(tmp_path):
    # output_crs.rs:265-287: projected layout, EPSG in key 3072, metres in 3076
    p = str(tmp_path / "u.tif")
    assert oracle.write_cog(p, np.ones((70, 90), np.float32), 90, 70, [500000.0, 10.0, 0.0, 5.2e6, 0.0, -10.0],
                            sd.OutputCrs.utm_south(33), 64) == 0
    buf = open(p, "rb").read()
    off = struct.unpack_from("<I", buf, 4)[0]
    while True:
        n, tags, nxt = _ifd_tags(buf, off)
        if nxt == 0:
            break
        off = nxt
    typ, cnt, at = tags[34735]
    keys = struct.unpack_from(f"<{cnt}H", buf, at)
    assert cnt == 20 and keys[3] == 4 and keys[12] == 3072 and keys[15] == 32733 and keys[19] == 9001
    scale = struct.unpack_from("<3d", buf, tags[33550][2])
    tie = struct.unpack_from("<6d", buf, tags[33922][2])
    assert scale == (10.0, 10.0, 0.0) and tie == (0.0, 0.0, 0.0, 500000.0, 5.2e6, 0.0)


# ── GPU path vs the oracle ──────────────────────────────────────────────────
@pytest.mark.gpu
def test_gpu_to_db_kats(ctx):
    d = np.array([1.0, 10.0, 0.0, -0.001, 0.5, np.nan, 0.005, 0.05], np.float32)
    ref = d.copy()
    assert sd.to_db_inplace(d, 0.01, ctx=ctx) == oracle.to_db_inplace(ref, 0.01) == (4, 3)
    assert np.array_equal(np.isnan(d), np.isnan(ref))
    assert abs(d[0]) < 1e-5 and abs(d[1] - 10.0) < 1e-5
    with pytest.raises(sd.ExportError) as e:
        sd.to_db_inplace(np.ones(3, np.float32), -0.001, ctx=ctx)
    assert e.value.kind == "InvalidNoiseFloor"


@pytest.mark.gpu
@pytest.mark.parametrize("n,floor", [(1, 0.0), (4097, 0.0), (3_000_017, 0.01)])
def test_gpu_to_db_and_stats_match_oracle(ctx, n, floor):
    import torch
    rng = np.random.default_rng(n)
    d = rng.exponential(0.05, n).astype(np.float32)
    d[rng.random(n) < 0.1] = np.nan
    d[rng.random(n) < 0.05] = 0.0
    d[rng.random(n) < 0.01] = -1.0
    ref = d.copy()
    cref = oracle.to_db_inplace(ref, floor)
    sref = oracle.db_stats(ref)
    host = d.copy()
    (c1, s1) = sd.to_db_inplace(host, floor, ctx=ctx, stats=True)  # host buffer
    dev = torch.from_numpy(d.copy()).cuda()
    (c2, s2) = sd.to_db_inplace(dev, floor, ctx=ctx, stats=True)   # device buffer, in place
    dev = dev.cpu().numpy()
    for got, cs, st in ((host, c1, s1), (dev, c2, s2)):
        assert cs == cref
        assert np.array_equal(np.isnan(got), np.isnan(ref))
        fin = np.isfinite(ref)
        assert _ulps(got[fin], ref[fin]).max() <= 4
        if n > 1:
            assert _ulps(st[0], sref[0]) <= 4 and _ulps(st[1], sref[1]) <= 4 and _ulps(st[3], sref[3]) <= 4
            assert abs(st[2] - sref[2]) <= 1e-6 * abs(sref[2])


@pytest.mark.gpu
@pytest.mark.parametrize("rows,cols", [(1, 1), (7, 5), (513, 1031)])
def test_gpu_downsample_bit_exact(ctx, rows, cols):
    src = _raster(rows, cols, rows * cols)
    got = sd.downsample_2x(src, cols, rows, ctx=ctx)
    ref = oracle.downsample_2x(src, cols, rows)
    assert got.shape == ref.shape
    assert np.array_equal(got.view(np.uint32), ref.view(np.uint32))


@pytest.mark.gpu
@pytest.mark.parametrize("rows,cols,ts,crs", [
    (1000, 1300, 256, WGS),                       # three overview levels, ragged edge tiles
    (64, 64, 64, WGS),                            # the reference's ramp case
    (300, 700, 128, sd.OutputCrs.utm_north(32)),  # projected GeoKeys
    (5, 3, 64, sd.OutputCrs.utm_south(59)),       # smaller than one tile
])
def test_gpu_cog_file_equals_oracle(ctx, tmp_path, rows, cols, ts, crs):
    import torch
    data = _raster(rows, cols, rows + cols)
    gt = [500000.0, 10.0, 0.0, 5.2e6, 0.0, -10.0] if crs.is_metric else GT
    pref = str(tmp_path / "ref.tif")
    assert oracle.write_cog(pref, data, cols, rows, gt, crs, ts) == 0
    want = open(pref, "rb").read()
    p1 = str(tmp_path / "host.tif")
    sd.write_cog_with_crs(p1, data, cols, rows, gt, crs, ts, ctx=ctx)
    assert open(p1, "rb").read() == want
    p2 = str(tmp_path / "dev.tif")
    sd.write_cog_with_crs(p2, torch.from_numpy(data).cuda(), cols, rows, gt, crs, ts, ctx=ctx)
    assert open(p2, "rb").read() == want


@pytest.mark.gpu
def test_gpu_cog_errors(ctx, tmp_path):
    d = np.ones((2, 2), np.float32)
    with pytest.raises(sd.ExportError) as e:
        sd.write_cog_with_crs(str(tmp_path / "a.tif"), d, 2, 2, GT, WGS, 100, ctx=ctx)
    assert e.value.kind == "InvalidTileSize"
    with pytest.raises(sd.ExportError) as e:
        sd.write_cog_with_crs(str(tmp_path / "b.tif"), d, 2, 2, [8.0, 0.0001, 0.0, 52.0, 0.0, 0.0001], WGS, 512,
                              ctx=ctx)
    assert e.value.kind == "InvalidGeotransform"
    with pytest.raises(sd.ExportError) as e:
        sd.write_cog_with_crs(str(tmp_path / "no_such_dir" / "c.tif"), d, 2, 2, GT, WGS, 512, ctx=ctx)
    assert e.value.kind == "Io"
    assert not os.path.exists(str(tmp_path / "no_such_dir"))


def _fused_vs_separate(ctx, run, floor):
    """run() on ctx with dB output fused into its last kernel, against run()
    in linear followed by to_db_inplace on the same context: the same bits,
    counts and statistics (both convert with the same device function)."""
    lin = np.array(run(), dtype=np.float32)
    c_sep, s_sep = sd.to_db_inplace(lin, floor, ctx=ctx, stats=True)
    sd.set_db_output(ctx, True, floor)
    try:
        fused = np.array(run(), dtype=np.float32)
        c_f, s_f = sd.db_result(ctx)
    finally:
        sd.set_db_output(ctx, False)
    assert np.array_equal(fused.view(np.uint32), lin.view(np.uint32)), "fused dB raster differs"
    assert c_f == c_sep
    assert np.array_equal(np.array(s_f, np.float32).view(np.uint32), np.array(s_sep, np.float32).view(np.uint32))
    assert c_f[0] > 0 and c_f[1] > 0
    return fused


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "split"])
def test_gpu_db_fused_into_terrain_correction(ctx, precision):
    """to_db_inplace fused into the terrain correction's last kernels
    (k_cand, and k_resample / k_redo in split precision)."""
    from sardine_b200 import synth
    sc = synth.config1_scene(seed=21, n_lines=512, n_samples=1024, dem_n=160, flatten=True,
                             resampling=sd.ResamplingKernel.Lanczos3)
    if precision == "split":
        sc.config.precision = sd.Precision.SPLIT
    floor = 0.02

    def run():
        return sd.terrain_correction(sc.merged, sc.scene, sc.dem, sc.grids, sc.config, ctx=ctx).data

    fused = _fused_vs_separate(ctx, run, floor)
    # and against the oracle's to_db of the same linear raster
    lin = np.array(run(), dtype=np.float32)
    ref = lin.copy()
    oracle.to_db_inplace(ref, floor)
    fin = np.isfinite(ref)
    assert np.array_equal(np.isnan(fused), np.isnan(ref))
    assert _ulps(fused[fin], ref[fin]).max() <= 4


@pytest.mark.gpu
@pytest.mark.parametrize("flt", [sd.SpeckleFilter.RefinedLee(4.4), sd.SpeckleFilter.GammaMap(5, 4.4)],
                         ids=["refined_lee", "gamma_map"])
def test_gpu_db_fused_into_speckle(ctx, flt):
    rng = np.random.default_rng(8)
    rows, cols = 301, 257
    img = rng.exponential(0.05, size=(rows, cols)).astype(np.float32)
    img[5:9, 30:60] = np.nan
    img[200:230, 100:140] = 0.0

    def run():
        return sd.apply_speckle_filter(img, cols, rows, flt, ctx=ctx)

    _fused_vs_separate(ctx, run, 0.01)


@pytest.mark.gpu
def test_gpu_db_output_errors(ctx):
    with pytest.raises(sd.ExportError) as e:
        sd.set_db_output(ctx, True, -1.0)
    assert e.value.kind == "InvalidNoiseFloor"
    fresh = sd.Context(ctx.device)
    with pytest.raises(sd.SardineError):
        sd.db_result(fresh)
    fresh.close()
