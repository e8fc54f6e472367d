"""The served loop on the GPU: two real slots (contexts with their own
streams), requests arriving while other batches are on the device, so that
batches of the two slots overlap.  Every result equals the same request run
alone (bit for bit), whatever batch it landed in; a cancelled request has no
result and does not disturb the others."""
import copy
import time

import numpy as np
import pytest

import sardine_b200 as sd
from sardine_b200 import synth, tiles
from sardine_b200.serve import Cancelled, GeocodingServer

pytestmark = pytest.mark.gpu

K = sd.ResamplingKernel


def _scene(ctx, seed):
    import oracle
    sc = synth.config1_scene(seed=seed, n_lines=1024, n_samples=2048, dem_n=256, flatten=True)
    rs = tiles.ResidentScene(sc.merged, sc.scene, sc.dem, sc.grids, sc.config.geoid, ctx)
    _, g = oracle.tc_output_grid(sc.scene, sc.config)
    return sc, rs, g


def _requests(scenes, rng, n):
    out = []
    for _ in range(n):
        sc, rs, g = scenes[int(rng.integers(0, len(scenes)))]
        rows, cols = (int(x) for x in rng.integers(16, 160, 2))
        r0 = int(rng.integers(0, g.rows - rows))
        c0 = int(rng.integers(0, g.cols - cols))
        cfg = copy.copy(sc.config)
        cfg.resampling = [K.Bilinear, K.Bicubic, K.Lanczos3][int(rng.integers(0, 3))]
        cfg.precision = [sd.Precision.FP64, sd.Precision.SPLIT][int(rng.integers(0, 2))]
        filt = [None, sd.SpeckleFilter.RefinedLee(4.4), sd.SpeckleFilter.GammaMap(5, 4.4)][int(rng.integers(0, 3))]
        sp = cfg.pixel_spacing_deg
        out.append(tiles.TileRequest(rs, cfg, g.origin_lon_deg + c0 * sp, g.origin_lat_deg - r0 * sp, rows, cols,
                                     filt))
    return out


def _saver(saved, host=False):
    def on_done(t):
        r = t.result
        assert r.data.is_cuda != host  # host_results: the planes arrive in pinned host memory
        saved[id(t)] = (r.data.cpu().numpy().copy(), None if r.mask is None else r.mask.cpu().numpy().copy(),
                        r.valid_pixel_count, list(r.newton_iter_histogram))
    return on_done


def _alone(req, ctx):
    a = tiles.tc_tiles([req], ctx)[0]
    return (a.data.cpu().numpy(), None if a.mask is None else a.mask.cpu().numpy(), a.valid_pixel_count,
            list(a.newton_iter_histogram))


def _same(x, y):
    assert np.array_equal(x[0], y[0], equal_nan=True)
    assert (x[1] is None and y[1] is None) or np.array_equal(x[1], y[1])
    assert x[2] == y[2] and x[3] == y[3]


@pytest.mark.parametrize("host", [False, True], ids=["device_results", "host_results"])
def test_served_results_equal_alone_with_overlapping_slots(ctx, host):
    scenes = [_scene(ctx, 61), _scene(ctx, 62)]
    rng = np.random.default_rng(3)
    reqs = _requests(scenes, rng, 40)
    saved = {}
    srv = GeocodingServer(0, hbm_budget=2 << 30, slots=2, max_batch=6, graphs=True, on_done=_saver(saved, host),
                          host_results=host)
    # a burst fills both slots, then Poisson arrivals at ~2000 req/s while
    # batches are on the device
    tickets = [srv.submit(r) for r in reqs[:12]]
    srv.step()
    overlap = sum(s.batch is not None for s in srv.slots)
    arrivals = np.cumsum(rng.exponential(1.0 / 2000.0, len(reqs) - 12))
    t0 = time.perf_counter()
    i = 12
    while i < len(reqs) or srv.busy():
        now = time.perf_counter() - t0
        while i < len(reqs) and arrivals[i - 12] <= now:
            tickets.append(srv.submit(reqs[i]))
            i += 1
        srv.step()
        overlap = max(overlap, sum(s.batch is not None for s in srv.slots))
    assert overlap == 2, "the two slots' batches never overlapped"
    assert all(t.error is None and t.done for t in tickets)
    alone_ctx = sd.Context(0)
    for t in tickets:
        _same(saved[id(t)], _alone(t.request, alone_ctx))
    srv.close()
    alone_ctx.close()
    for _, rs, _ in scenes:
        rs.close()


def test_served_cancel_on_device(ctx):
    scenes = [_scene(ctx, 63)]
    rng = np.random.default_rng(4)
    reqs = _requests(scenes, rng, 10)
    saved = {}
    srv = GeocodingServer(0, hbm_budget=1 << 30, slots=1, max_batch=4, graphs=False, on_done=_saver(saved))
    tickets = [srv.submit(r) for r in reqs]
    srv.step()                              # four in flight, six queued
    in_flight, queued = tickets[1], tickets[6]
    assert srv.cancel(in_flight) and srv.cancel(queued)
    assert queued.done and isinstance(queued.error, Cancelled)
    srv.drain()
    assert isinstance(in_flight.error, Cancelled) and in_flight.result is None and id(in_flight) not in saved
    alone_ctx = sd.Context(0)
    for t in tickets:
        if t in (in_flight, queued):
            continue
        assert t.error is None
        _same(saved[id(t)], _alone(t.request, alone_ctx))
    srv.close()
    alone_ctx.close()
    scenes[0][1].close()
