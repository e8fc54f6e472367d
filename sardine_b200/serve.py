"""Served geocoding: a device-resident request loop with continuous batching.

Scenes stay resident in HBM (`tiles.ResidentScene`).  Tile requests arrive
at any time; each scheduler step

  1. collects every slot whose batch has finished (its requests complete,
     their scratch leaves the HBM budget),
  2. admits queued requests, oldest first, into a batch for a free slot while
     the batch fits the slot's share of the HBM budget and `max_batch`,
  3. launches that batch asynchronously (one persistent launch per stage,
     replayed from a CUDA graph).

A request can be cancelled (`cancel`): a queued one leaves the queue, an
in-flight one still runs with its batch but its result is dropped when the
batch is collected.  A request submitted with a deadline that has passed by
the time a slot could take it is cancelled the same way (`Cancelled`).

A slot is a context (CUDA stream + reserved scratch arena); with two or more
slots, a batch admitted while another is on the GPU runs concurrently with
it.  Requests never wait for a batch boundary longer than one in-flight
batch per slot.  A request's result does not depend on the batch it lands in
(each tile is an independent job of the launch).
"""
from __future__ import annotations

import ctypes as C
import time
from collections import deque
from dataclasses import dataclass, field
from typing import Callable, Deque, List, Optional

from ._lib import Context, lib
from .tiles import TileBatch, TileRequest


class Cancelled(Exception):
    """The request was cancelled (by `cancel` or its deadline) and has no result."""


@dataclass
class Ticket:
    """One submitted request and, once done, its result and timings."""
    request: TileRequest
    t_submit: float
    t_launch: float = 0.0
    t_done: float = 0.0
    result: object = None
    error: Optional[BaseException] = None
    deadline: float = float("inf")  # latest admission time (the clock's units)
    cancel_requested: bool = False

    @property
    def cancelled(self) -> bool:
        return isinstance(self.error, Cancelled)

    @property
    def latency_s(self) -> float:
        return self.t_done - self.t_submit

    @property
    def done(self) -> bool:
        return self.t_done > 0.0


def output_bytes(req: TileRequest) -> int:
    """Device bytes of a tile's results (f32 data, f32 cos(LIA), u8 mask),
    each plane 256 B aligned."""
    n = req.rows * req.cols
    al = lambda x: (x + 255) // 256 * 256
    return al(4 * n) + (al(4 * n) + al(n) if req.config.compute_lia else 0)


class _Slot:
    """A context (stream) with its scratch arena reserved up front and a
    result arena the batch's outputs are carved from."""

    def __init__(self, device: int, arena_bytes: int, graphs: bool, out_bytes: int, host: bool = False):
        import torch
        self.ctx = Context(device)
        self.device = device
        self.capacity = arena_bytes
        self.out_capacity = out_bytes
        lib().sd_ctx_set_graphs(self.ctx.handle, int(graphs))
        if arena_bytes:
            rc = lib().sd_ctx_reserve(self.ctx.handle, C.c_uint64(arena_bytes))
            if rc != 0:
                raise MemoryError(self.ctx.last_error())
        self.out_arena = torch.empty(out_bytes, dtype=torch.uint8, device=f"cuda:{device}")
        # host delivery: a pinned mirror of the result arena, filled by one
        # copy on the slot's stream behind each batch's kernels
        self.host_arena = torch.empty(out_bytes, dtype=torch.uint8, pin_memory=True) if host else None
        self.host_views = None
        self.batch: Optional[TileBatch] = None
        self.tickets: List[Ticket] = []
        self.bytes = 0

    def launch(self, requests):
        import torch
        outs, hviews, off = [], [], 0
        for r in requests:
            n = r.rows * r.cols
            views, hv = [], []
            for k, (dt, esz) in enumerate(((torch.float32, 4), (torch.float32, 4), (torch.uint8, 1))):
                if k > 0 and not r.config.compute_lia:
                    views.append(None)
                    hv.append(None)
                    continue
                views.append(self.out_arena[off:off + esz * n].view(dt).view(r.rows, r.cols))
                if self.host_arena is not None:
                    hv.append(self.host_arena[off:off + esz * n].view(dt).view(r.rows, r.cols))
                off += (esz * n + 255) // 256 * 256
            outs.append(tuple(views))
            hviews.append(tuple(hv))
        batch = TileBatch(self.ctx, requests, outs).launch()
        self.host_views = None
        if self.host_arena is not None and off:
            # one copy behind the batch on its stream (the library's, so no
            # torch stream bookkeeping outlives the context); the batch is
            # done once the copy has landed
            rc = lib().sd_tc_tiles_copy_out(self.ctx.handle, C.c_void_p(self.host_arena.data_ptr()),
                                            C.c_void_p(self.out_arena.data_ptr()), C.c_uint64(off))
            if rc != 0:
                raise RuntimeError(f"sd_tc_tiles_copy_out: {self.ctx.last_error()}")
            self.host_views = hviews
        return batch

    def close(self):
        # the result arenas go before the context whose stream filled them
        self.host_views = None
        self.host_arena = None
        self.out_arena = None
        self.ctx.close()


class GeocodingServer:
    """Continuous-batching request loop over resident scenes on one GPU.

    hbm_budget: device bytes the in-flight batches may hold for tile scratch
    (split evenly over `slots`; each slot reserves its share up front, so the
    loop itself never allocates device memory for scratch).
    """

    def __init__(self, device: int = 0, hbm_budget: int = 8 << 30, slots: int = 2,
                 max_batch: int = 64, graphs: bool = True,
                 clock: Callable[[], float] = time.perf_counter, slot_factory=None,
                 on_done: Optional[Callable[[Ticket], None]] = None, keep_results: bool = False,
                 host_results: bool = False):
        """hbm_budget covers each slot's scratch arena (4/5 of its share) and
        result arena (1/5).  Results live in the slot's result arena until
        that slot's next batch: `on_done(ticket)` runs as each request
        completes (copy out what must outlive it); unless keep_results, the
        completed ticket keeps only counters and timings.  host_results:
        results are delivered in pinned host memory (the slot's host mirror,
        copied behind the batch on its stream, so the transfer overlaps the
        other slots' kernels); a request completes when its results are on
        the host."""
        if slots < 1:
            raise ValueError("slots must be >= 1")
        self.clock = clock
        self.max_batch = max_batch
        self.on_done = on_done
        self.keep_results = keep_results
        share = hbm_budget // slots
        make = slot_factory or (lambda cap: _Slot(device, cap * 4 // 5, graphs, cap // 5, host_results))
        self.slots = [make(share) for _ in range(slots)]
        self.queue: Deque[Ticket] = deque()
        self.completed: List[Ticket] = []

    # ── client side ──
    def submit(self, req: TileRequest, deadline_s: Optional[float] = None) -> Ticket:
        """Queues a request; with deadline_s it is cancelled if no slot has
        taken it within deadline_s of its submission."""
        t = Ticket(req, self.clock())
        if deadline_s is not None:
            t.deadline = t.t_submit + deadline_s
        out_cap = getattr(self.slots[0], "out_capacity", None)
        if req.device_bytes() > self.slots[0].capacity or \
                (out_cap is not None and output_bytes(req) > out_cap):
            t.error = MemoryError(f"tile needs {req.device_bytes()} B, above a slot's "
                                  f"{self.slots[0].capacity} B share of the HBM budget")
            t.t_done = t.t_submit
            self.completed.append(t)
            return t
        self.queue.append(t)
        return t

    def cancel(self, t: Ticket) -> bool:
        """Cancels a request that has not completed: a queued one is removed
        at once; an in-flight one runs on with its batch and its result is
        dropped at collection.  Returns False when it had already completed."""
        if t.done:
            return False
        try:
            self.queue.remove(t)
        except ValueError:  # in flight
            t.cancel_requested = True
            return True
        t.error = Cancelled("cancelled before launch")
        t.t_done = self.clock()
        self.completed.append(t)
        return True

    # ── scheduler ──
    def step(self) -> int:
        """One scheduler pass; returns the number of requests that completed."""
        n_done = 0
        for s in self.slots:
            if s.batch is not None and s.batch.done():
                n_done += self._collect(s)
        for s in self.slots:
            if s.batch is None and self.queue:
                self._admit(s)
        return n_done

    def _collect(self, s: _Slot) -> int:
        now = None
        try:
            results = s.batch.finish()
            now = self.clock()
            host = getattr(s, "host_views", None)
            for k, (t, r) in enumerate(zip(s.tickets, results)):
                if host is not None and hasattr(r, "data"):  # the planes as they landed on the host
                    r.data, r.cos_lia, r.mask = host[k]
                t.t_done = now
                if t.cancel_requested:  # ran with its batch; the result is dropped
                    t.error = Cancelled("cancelled in flight")
                    continue
                t.result = r
                if self.on_done is not None:
                    self.on_done(t)
                if not self.keep_results and hasattr(r, "data"):
                    r.data = r.cos_lia = r.mask = None
        except Exception as e:  # the whole batch failed: report it on every ticket
            now = self.clock()
            for t in s.tickets:
                t.error = e
                t.t_done = now
        self.completed.extend(s.tickets)
        n = len(s.tickets)
        s.batch, s.tickets, s.bytes = None, [], 0
        return n

    def _admit(self, s: _Slot) -> None:
        take: List[Ticket] = []
        used = used_out = 0
        out_cap = getattr(s, "out_capacity", float("inf"))
        now = self.clock()
        while self.queue and self.queue[0].deadline < now:  # expired before any slot took it
            t = self.queue.popleft()
            t.error = Cancelled("deadline passed before launch")
            t.t_done = now
            self.completed.append(t)
        while self.queue and len(take) < self.max_batch:
            need = self.queue[0].request.device_bytes()
            need_out = output_bytes(self.queue[0].request) if out_cap != float("inf") else 0
            if used + need > s.capacity or used_out + need_out > out_cap:
                break
            used += need
            used_out += need_out
            take.append(self.queue.popleft())
        if not take:
            return
        now = self.clock()
        for t in take:
            t.t_launch = now
        s.tickets, s.bytes = take, used
        s.batch = s.launch([t.request for t in take])

    def busy(self) -> bool:
        return bool(self.queue) or any(s.batch is not None for s in self.slots)

    def drain(self) -> None:
        while self.busy():
            self.step()

    def close(self) -> None:
        self.drain()
        for s in self.slots:
            s.close()


def latency_summary(tickets: List[Ticket]) -> dict:
    import numpy as np
    ok = [t for t in tickets if t.error is None and t.done]
    if not ok:
        return {"completed": 0}
    lat = np.array([t.latency_s for t in ok]) * 1e3
    px = sum(t.request.rows * t.request.cols for t in ok)
    t0 = min(t.t_submit for t in ok)
    t1 = max(t.t_done for t in ok)
    return {"completed": len(ok), "failed": len(tickets) - len(ok), "p50_ms": float(np.percentile(lat, 50)),
            "p99_ms": float(np.percentile(lat, 99)), "mean_ms": float(lat.mean()),
            "px": int(px), "span_s": t1 - t0, "px_per_s": px / max(t1 - t0, 1e-9)}
