"""Batched tiles over device-resident scenes (sd_scene_* / sd_tc_tiles_*).

Each tile is terrain_correction on the tile's own output grid: checked
against the oracle run on that grid (same bar as the single-scene parity
tests).  A speckle-filtered tile is geocoded with a halo of half a window,
filtered and cropped: checked against the oracle geocoding the widened grid,
the oracle filter, then the crop.  A tile's result does not depend on the
batch around it, with or without CUDA graphs.
"""
import copy

import numpy as np
import pytest

import oracle
import sardine_b200 as sd
from sardine_b200 import synth, tiles
from sardine_b200.accuracy import compare_geocoded
from tests.test_gpu_tc import assert_tc_parity

pytestmark = pytest.mark.gpu

K = sd.ResamplingKernel


def _scene(ctx, seed, **kw):
    sc = synth.config1_scene(seed=seed, n_lines=1024, n_samples=2048, dem_n=256, flatten=True, **kw)
    rs = tiles.ResidentScene(sc.merged, sc.scene, sc.dem, sc.grids, sc.config.geoid, ctx)
    _, g = oracle.tc_output_grid(sc.scene, sc.config)
    return sc, rs, g


def _req(sc, rs, g, r0, c0, rows, cols, kernel=K.Bilinear, speckle=None, precision=sd.Precision.FP64):
    cfg = copy.copy(sc.config)
    cfg.resampling = kernel
    cfg.precision = precision
    sp = cfg.pixel_spacing_deg
    return tiles.TileRequest(rs, cfg, g.origin_lon_deg + c0 * sp, g.origin_lat_deg - r0 * sp, rows, cols,
                             speckle)


def _host(res):
    res.data = res.data.cpu().numpy()
    if res.cos_lia is not None:
        res.cos_lia = res.cos_lia.cpu().numpy()
        res.mask = res.mask.cpu().numpy()
    return res


def _oracle_tile(sc, req, halo=0):
    """The oracle on the tile's grid, with glibc's and with correctly rounded
    sines and cosines (see test_gpu_tc)."""
    sp = req.config.pixel_spacing_deg

    def run():
        return oracle.terrain_correction_grid(sc.merged, sc.scene, sc.dem, sc.grids, req.config,
                                              req.origin_x - halo * sp, req.origin_y + halo * sp,
                                              req.rows + 2 * halo, req.cols + 2 * halo)
    gl = run()
    with oracle.libm("cr"):
        cr = run()
    return gl, cr


def test_tiles_match_oracle(ctx):
    sc, rs, g = _scene(ctx, 51)
    reqs = [_req(sc, rs, g, 0, 0, 64, 96, K.Bilinear),
            _req(sc, rs, g, 17, 40, 100, 33, K.Bicubic),
            _req(sc, rs, g, 120, 5, 80, 200, K.Lanczos3),
            _req(sc, rs, g, 3, 150, 31, 57, K.Bicubic),
            _req(sc, rs, g, 200, 200, 1, 1, K.Bilinear)]
    res = tiles.tc_tiles(reqs, ctx)
    for req, r in zip(reqs, res):
        ref = _oracle_tile(sc, req)
        assert r.total_pixel_count == req.rows * req.cols
        assert_tc_parity(_host(r), ref)
    rs.close()


def test_tiles_two_scenes_split_precision(ctx):
    sc1, rs1, g1 = _scene(ctx, 52)
    sc2, rs2, g2 = _scene(ctx, 53, center_lat_deg=-20.0)
    reqs = [_req(sc1, rs1, g1, 10, 10, 70, 90, K.Lanczos3, precision=sd.Precision.SPLIT),
            _req(sc2, rs2, g2, 30, 60, 64, 64, K.Bicubic),
            _req(sc2, rs2, g2, 90, 0, 50, 120, K.Lanczos3, precision=sd.Precision.SPLIT)]
    res = tiles.tc_tiles(reqs, ctx)
    for (sc, req), r in zip([(sc1, reqs[0]), (sc2, reqs[1]), (sc2, reqs[2])], res):
        ref = _oracle_tile(sc, req)
        r = _host(r)
        if req.config.precision == sd.Precision.SPLIT:
            rep = compare_geocoded(r, ref[1])
            assert rep["nan_pattern_equal"] and rep["mask_equal"], rep
            assert rep["sigma_rel_over_1e-4_px"] == 0, rep
            assert r.newton_iter_histogram == ref[1].newton_iter_histogram
        else:
            assert_tc_parity(r, ref)
    rs1.close()
    rs2.close()


@pytest.mark.parametrize("filt,halo", [(sd.SpeckleFilter.RefinedLee(4.4), 3),
                                       (sd.SpeckleFilter.GammaMap(5, 4.4), 2)])
def test_tiles_speckle_halo_crop(ctx, filt, halo):
    sc, rs, g = _scene(ctx, 54)
    req = _req(sc, rs, g, 40, 50, 90, 120, K.Bicubic, speckle=filt)
    assert req.halo() == halo
    r = _host(tiles.tc_tiles([req], ctx)[0])
    big = _oracle_tile(sc, req, halo)[1]
    rows, cols = req.rows + 2 * halo, req.cols + 2 * halo
    ref = oracle.apply_speckle_filter(big.data, cols, rows, filt)
    crop = np.asarray(ref).reshape(rows, cols)[halo:halo + req.rows, halo:halo + req.cols]
    assert np.array_equal(np.isnan(r.data), np.isnan(crop))
    ok = np.isfinite(crop)
    rel = np.abs(r.data[ok].astype(np.float64) - crop[ok]) / np.maximum(np.abs(crop[ok]), 1e-30)
    assert (rel > 1e-4).sum() == 0, rel.max()
    assert np.array_equal(r.mask, big.mask[halo:halo + req.rows, halo:halo + req.cols])
    rs.close()


def test_tiles_same_alone_and_in_mix(ctx):
    sc1, rs1, g1 = _scene(ctx, 55)
    sc2, rs2, g2 = _scene(ctx, 56)
    a = _req(sc1, rs1, g1, 20, 30, 77, 91, K.Bicubic, speckle=sd.SpeckleFilter.RefinedLee(4.4))
    mix = [_req(sc2, rs2, g2, 0, 0, 150, 150, K.Lanczos3),
           a,
           _req(sc1, rs1, g1, 100, 100, 40, 300, K.Bilinear, speckle=sd.SpeckleFilter.GammaMap(5, 4.4)),
           _req(sc2, rs2, g2, 5, 7, 64, 64, K.Bicubic, precision=sd.Precision.SPLIT)]
    alone = _host(tiles.tc_tiles([a], ctx)[0])
    inmix = _host(tiles.tc_tiles(mix, ctx)[1])
    assert np.array_equal(alone.data, inmix.data, equal_nan=True)
    assert np.array_equal(alone.mask, inmix.mask)
    assert alone.newton_iter_histogram == inmix.newton_iter_histogram
    rs1.close()
    rs2.close()


def test_tiles_graph_replay(ctx):
    sc, rs, g = _scene(ctx, 57)
    b1 = [_req(sc, rs, g, 0, 0, 60, 80, K.Bicubic), _req(sc, rs, g, 70, 10, 33, 120, K.Lanczos3)]
    b2 = [_req(sc, rs, g, 11, 12, 90, 45, K.Bilinear, speckle=sd.SpeckleFilter.RefinedLee(4.4))]
    plain = [_host(r) for r in tiles.tc_tiles(b1, ctx)] + [_host(r) for r in tiles.tc_tiles(b2, ctx)]
    tiles.set_graphs(ctx, True)
    try:
        for _ in range(2):
            got = [_host(r) for r in tiles.tc_tiles(b1, ctx)] + [_host(r) for r in tiles.tc_tiles(b2, ctx)]
            for x, y in zip(plain, got):
                assert np.array_equal(x.data, y.data, equal_nan=True)
                assert np.array_equal(x.mask, y.mask)
                assert x.valid_pixel_count == y.valid_pixel_count
    finally:
        tiles.set_graphs(ctx, False)
    rs.close()


def test_tiles_async_and_errors(ctx):
    sc, rs, g = _scene(ctx, 58)
    batch = tiles.TileBatch(ctx, [_req(sc, rs, g, 0, 0, 64, 64)]).launch()
    with pytest.raises(sd.SardineError) as e:
        tiles.TileBatch(ctx, [_req(sc, rs, g, 0, 0, 8, 8)]).launch()
    assert e.value.kind == "Busy"
    while not batch.done():
        pass
    assert batch.finish()[0].total_pixel_count == 64 * 64
    with pytest.raises(sd.SpeckleError) as e:
        tiles.tc_tiles([_req(sc, rs, g, 0, 0, 8, 8, speckle=sd.SpeckleFilter.GammaMap(4, 4.4))], ctx)
    assert e.value.kind == "BadWindow"
    bad = _req(sc, rs, g, 0, 0, 8, 8)
    bad.config.pixel_spacing_deg = 0.0
    with pytest.raises(sd.TerrainCorrectionError) as e:
        tiles.tc_tiles([bad], ctx)
    assert e.value.kind == "Config"
    rs.close()


def test_tiles_launch_shapes_do_not_change_results(ctx):
    """Every launch shape the autotuner may pick (speckle block, persistent
    CTAs per SM, per-tile parameter launches) gives bit-identical tiles."""
    from sardine_b200 import autotune
    sc, rs, g = _scene(ctx, 59)
    reqs = [_req(sc, rs, g, 0, 0, 60, 80, K.Bicubic, speckle=sd.SpeckleFilter.GammaMap(5, 4.4)),
            _req(sc, rs, g, 70, 10, 33, 120, K.Lanczos3, precision=sd.Precision.SPLIT),
            _req(sc, rs, g, 11, 12, 90, 45, K.Bilinear, speckle=sd.SpeckleFilter.RefinedLee(4.4))]
    base = [_host(r) for r in tiles.tc_tiles(reqs, ctx)]
    try:
        for shape in ([64, 4], [16, 16], [128, 2]):
            for cps in (0, 2, -1):
                autotune.apply(ctx, {"speckle": shape, "main_cps": cps})
                got = [_host(r) for r in tiles.tc_tiles(reqs, ctx)]
                for x, y in zip(base, got):
                    assert np.array_equal(x.data, y.data, equal_nan=True), (shape, cps)
                    assert np.array_equal(x.mask, y.mask)
                    assert x.newton_iter_histogram == y.newton_iter_histogram
    finally:
        autotune.apply(ctx, autotune.DEFAULT)
    rs.close()
