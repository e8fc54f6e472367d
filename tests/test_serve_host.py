"""Host logic of the served-geocoding loop (no GPU): HBM-budget admission,
continuous batching over slots, FIFO order, latency accounting; and the
tile geometry helpers."""
import copy

import numpy as np

import oracle
import sardine_b200 as sd
from sardine_b200 import synth
from sardine_b200.serve import Cancelled, GeocodingServer, latency_summary
from sardine_b200.tiles import TileRequest


class FakeReq:
    def __init__(self, name, nbytes, rows=10, cols=10):
        self.name, self.nbytes, self.rows, self.cols = name, nbytes, rows, cols

    def device_bytes(self):
        return self.nbytes


class FakeBatch:
    """Finishes after `polls` calls of done()."""

    def __init__(self, reqs, polls):
        self.reqs, self.left = reqs, polls

    def done(self):
        self.left -= 1
        return self.left <= 0

    def finish(self):
        return [("result", r.name) for r in self.reqs]


class FakeSlot:
    def __init__(self, cap, polls=2):
        self.capacity, self.polls = cap, polls
        self.batch, self.tickets, self.bytes = None, [], 0
        self.launched = []

    def launch(self, reqs):
        self.launched.append([r.name for r in reqs])
        return FakeBatch(reqs, self.polls)

    def close(self):
        pass


class Clock:
    def __init__(self):
        self.t = 0.0

    def __call__(self):
        self.t += 1.0
        return self.t


def _server(budget, slots=2, max_batch=64, polls=2):
    made = []

    def factory(cap):
        s = FakeSlot(cap, polls)
        made.append(s)
        return s
    srv = GeocodingServer(hbm_budget=budget, slots=slots, max_batch=max_batch, clock=Clock(),
                          slot_factory=factory)
    return srv, made


def test_admission_respects_budget_and_max_batch():
    srv, slots = _server(budget=200, slots=2, max_batch=3)  # 100 B per slot
    for i in range(6):
        srv.submit(FakeReq(f"r{i}", 40))
    srv.step()
    # each slot takes what fits its 100 B share: two 40 B requests
    assert slots[0].launched == [["r0", "r1"]] and slots[1].launched == [["r2", "r3"]]
    assert [t.request.name for t in srv.queue] == ["r4", "r5"]
    srv.drain()
    assert sorted(t.request.name for t in srv.completed) == [f"r{i}" for i in range(6)]
    assert all(t.result == ("result", t.request.name) for t in srv.completed)


def test_continuous_batching_admits_while_other_slot_busy():
    srv, slots = _server(budget=200, slots=2, polls=3)
    srv.submit(FakeReq("a", 90))
    srv.step()                       # a -> slot 0
    srv.submit(FakeReq("b", 90))     # arrives while a is on the GPU
    srv.step()                       # b -> slot 1 at once, not after a
    assert slots[0].launched == [["a"]] and slots[1].launched == [["b"]]
    srv.submit(FakeReq("c", 90))
    srv.drain()
    names = [t.request.name for t in srv.completed]
    assert names.index("a") < names.index("c")
    assert sum(len(x) for x in slots[0].launched + slots[1].launched) == 3


def test_fifo_head_of_line_and_oversize():
    srv, slots = _server(budget=100, slots=1, max_batch=8)
    big = srv.submit(FakeReq("big", 500))
    assert big.done and isinstance(big.error, MemoryError)
    srv.submit(FakeReq("x", 70))
    srv.submit(FakeReq("y", 70))   # does not fit beside x: waits for the next batch
    srv.submit(FakeReq("z", 10))   # FIFO: not admitted ahead of y
    srv.step()
    assert slots[0].launched == [["x"]]
    srv.drain()
    assert slots[0].launched == [["x"], ["y", "z"]]


def test_cancel_queued_and_in_flight():
    srv, slots = _server(budget=100, slots=1, max_batch=1, polls=3)
    a = srv.submit(FakeReq("a", 50))
    b = srv.submit(FakeReq("b", 50))
    c = srv.submit(FakeReq("c", 50))
    srv.step()                       # a in flight, b and c queued
    assert srv.cancel(a) and srv.cancel(b)
    assert b.done and b.cancelled and not a.done
    srv.drain()
    assert a.cancelled and a.result is None       # ran with its batch, result dropped
    assert c.result == ("result", "c") and c.error is None
    assert slots[0].launched == [["a"], ["c"]]     # b never launched
    assert not srv.cancel(c)                      # already completed
    s = latency_summary(srv.completed)
    assert s["completed"] == 1 and s["failed"] == 2


def test_deadline_expires_in_queue():
    srv, slots = _server(budget=100, slots=1, max_batch=1, polls=5)
    srv.submit(FakeReq("a", 50))
    late = srv.submit(FakeReq("late", 50), deadline_s=2.0)   # the fake clock ticks 1 per call
    ok = srv.submit(FakeReq("ok", 50), deadline_s=1e9)
    srv.drain()
    assert isinstance(late.error, Cancelled) and late.result is None
    assert ok.result == ("result", "ok")
    assert ["late"] not in slots[0].launched


def test_latency_summary():
    srv, _ = _server(budget=1000, slots=1, polls=1)
    for i in range(4):
        srv.submit(FakeReq(f"r{i}", 10, rows=2, cols=3))
    srv.drain()
    s = latency_summary(srv.completed)
    assert s["completed"] == 4 and s["px"] == 24
    assert s["p50_ms"] > 0 and s["p99_ms"] >= s["p50_ms"]


def test_tile_request_halo_and_budget():
    sc = synth.config1_scene(seed=5, n_lines=128, n_samples=256, dem_n=48)
    r0 = TileRequest(None, sc.config, 0.0, 0.0, 100, 50)
    r1 = TileRequest(None, sc.config, 0.0, 0.0, 100, 50, sd.SpeckleFilter.RefinedLee(4.4))
    r2 = TileRequest(None, sc.config, 0.0, 0.0, 100, 50, sd.SpeckleFilter.GammaMap(5, 4.4))
    assert (r0.halo(), r1.halo(), r2.halo()) == (0, 3, 2)
    # per-pixel target, facet, pair bases, codes, selection and halo'd
    # outputs: 78 B per halo'd pixel
    assert r1.device_bytes() >= 106 * 56 * 78 and r1.device_bytes() > r0.device_bytes()


def test_oracle_explicit_grid_equals_scene_grid():
    """The tile oracle on the scene's own grid reproduces terrain_correction."""
    sc = synth.config1_scene(seed=6, n_lines=256, n_samples=512, dem_n=64, flatten=True)
    _, g = oracle.tc_output_grid(sc.scene, sc.config)
    full = oracle.terrain_correction(sc.merged, sc.scene, sc.dem, sc.grids, sc.config)
    same = oracle.terrain_correction_grid(sc.merged, sc.scene, sc.dem, sc.grids, sc.config,
                                          g.origin_lon_deg, g.origin_lat_deg, g.rows, g.cols)
    assert np.array_equal(full.data, same.data, equal_nan=True)
    assert np.array_equal(full.mask, same.mask)
    assert full.newton_iter_histogram == same.newton_iter_histogram
