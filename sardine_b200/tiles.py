"""Device-resident scenes and batched tile geocoding (sd_scene_* / sd_tc_tiles_*).

A `ResidentScene` uploads one radar scene (merged sigma0 + NESZ, DEM, geoid,
orbit, geolocation-grid LUT, FP64 orbit table) once.  A batch of
`TileRequest`s (output windows of any size over any resident scene, each with
its own resampling kernel, precision and optional speckle filter) is then
geocoded by one launch per stage.  Each tile equals `terrain_correction` run
on that tile's own output grid; with a speckle filter the tile is geocoded
with a halo of half a window and filtered before cropping.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from typing import List, Optional, Sequence

import numpy as np

from . import _abi
from . import types as T
from ._lib import Context, lib


def _check(ctx: Context, rc: int):
    if rc != 0:
        from . import TerrainCorrectionError, _check as check
        check(ctx, rc, TerrainCorrectionError)


def _prep(a, dtype):
    if a is None:
        return None
    if isinstance(a, np.ndarray):
        return np.ascontiguousarray(a, dtype=dtype)
    return a


class ResidentScene:
    """sd_scene_create: the scene's inputs and orbit table kept in HBM.

    Host arrays are copied; CUDA tensors are borrowed (kept referenced here)."""

    def __init__(self, merged: T.MergedSigma0, scene: T.SceneMetadata, dem: T.DemGrid, grids,
                 geoid: T.GeoidModel, ctx: Context):
        self.ctx = ctx
        keep = T._Keep()
        self._refs = []
        data = _prep(merged.data, np.float32)
        nesz = _prep(merged.nesz, np.float32) if merged.nesz is not None else None
        dem_data = _prep(dem.data, np.float32)
        self._refs += [data, nesz, dem_data]
        img = _abi.RadarImage(T.ptr(data), T.ptr(nesz), merged.lines, merged.samples,
                              int(merged.azimuth_start_time_us), merged.near_slant_range_time_s,
                              merged.range_pixel_spacing_m)
        sc = T.scene_to_c(scene, keep)
        d = _abi.Dem(dem.kind, dem.utm_zone, int(dem.utm_south), 0, T.ptr(dem_data),
                     dem_data.shape[1], dem_data.shape[0], dem.origin_y, dem.origin_x, dem.pixel_size)
        geo = geoid.to_c(keep)
        pts = T.pick_lut_grid(grids)
        g = T.grid_to_c(pts)
        h = C.c_void_p()
        _check(ctx, lib().sd_scene_create(ctx.handle, C.byref(img), C.byref(sc), C.byref(d),
                                          C.byref(geo), g, len(pts), C.byref(h)))
        self.handle = h
        self.lines, self.samples = merged.lines, merged.samples

    @property
    def device_bytes(self) -> int:
        return int(lib().sd_scene_device_bytes(self.handle)) if self.handle else 0

    def close(self):
        if self.handle:
            lib().sd_scene_destroy(self.handle)
            self.handle = None
            self._refs = []

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


@dataclass
class TileRequest:
    """One output window: `origin_x`/`origin_y` are the west/north edges in
    the config's CRS (degrees for WGS84, metres for UTM)."""
    scene: ResidentScene
    config: T.TerrainCorrectionConfig
    origin_x: float
    origin_y: float
    rows: int
    cols: int
    speckle: Optional[T.SpeckleFilter] = None

    def halo(self) -> int:
        if self.speckle is None:
            return 0
        w = 7 if self.speckle.kind == _abi.SPECKLE_REFINED_LEE else self.speckle.window
        return w // 2

    def device_bytes(self) -> int:
        """Device scratch this tile needs inside a batch (admission budget):
        per-pixel target (24 B) and facet (32 B, with flattening or LIA),
        pair base / time (8 B), codes (4 B), selection (1 B) and halo'd
        outputs (9 B) over the halo'd grid, plus per-row state and the final
        rasters when they are staged."""
        h = self.halo()
        r, c = self.rows + 2 * h, self.cols + 2 * h
        anchors = min(256, c) + 1 if self.config.crs.kind != _abi.CRS_WGS84 else 0
        per_row = 8 + 8 + 17 * 8 + (16 + 64) * anchors
        extra = 0
        if self.config.precision == T.Precision.SPLIT:
            # FP64 re-sample queue: per k_cand item (256 px) a count and 64 x 24 B
            extra = -(-(r * c) // 256) * (4 + 64 * 24) + 512
        geom = 32 if (self.config.flatten or self.config.compute_lia) else 0
        return r * c * (24 + geom + 8 + 4 + 1 + 9) + r * per_row + self.rows * self.cols * 9 + 8192 + extra


def _tile_to_c(req: TileRequest, outs, anchors: int) -> _abi.Tile:
    data, cos, mask = outs
    sp = req.speckle
    return _abi.Tile(req.scene.handle, req.config.to_c(anchors), float(req.origin_x),
                     float(req.origin_y), int(req.rows), int(req.cols),
                     -1 if sp is None else int(sp.kind), 7 if sp is None else int(sp.window),
                     1.0 if sp is None else float(sp.enl), 0.0 if sp is None else float(sp.damping),
                     T.ptr(data), T.ptr(cos), T.ptr(mask))


def _alloc_outputs(req: TileRequest, device):
    import torch
    shape = (req.rows, req.cols)
    data = torch.empty(shape, dtype=torch.float32, device=device)
    cos = torch.empty(shape, dtype=torch.float32, device=device) if req.config.compute_lia else None
    mask = torch.empty(shape, dtype=torch.uint8, device=device) if req.config.compute_lia else None
    return data, cos, mask


class TileBatch:
    """One batch in flight on a context: launch(), poll(), finish()."""

    def __init__(self, ctx: Context, requests: Sequence[TileRequest], outputs=None,
                 anchors: int = 256):
        self.ctx = ctx
        self.requests = list(requests)
        if outputs is None:
            dev = f"cuda:{ctx.device}"
            outputs = [_alloc_outputs(r, dev) for r in self.requests]
        self.outputs = outputs
        arr = (_abi.Tile * len(self.requests))()
        for i, (r, o) in enumerate(zip(self.requests, outputs)):
            arr[i] = _tile_to_c(r, o, anchors)
        self._arr = arr
        self.launched = False

    def launch(self) -> "TileBatch":
        _check(self.ctx, lib().sd_tc_tiles_launch(self.ctx.handle, self._arr, len(self.requests)))
        self.launched = True
        return self

    def done(self) -> bool:
        rc = lib().sd_tc_tiles_poll(self.ctx.handle)
        if rc == 0:
            return True
        if rc == _abi.SD_ERR_BUSY:
            return False
        _check(self.ctx, rc)
        return False

    def finish(self) -> List[T.GeocodedImage]:
        n = len(self.requests)
        infos = (_abi.GeocodedInfo * n)()
        _check(self.ctx, lib().sd_tc_tiles_finish(self.ctx.handle, infos, n))
        res = []
        for r, o, f in zip(self.requests, self.outputs, infos):
            res.append(T.GeocodedImage.from_info(f, r.config.crs, o[0], o[1], o[2]))
        return res


def tc_tiles(requests: Sequence[TileRequest], ctx: Context, outputs=None) -> List[T.GeocodedImage]:
    """Geocodes a batch of tiles (synchronous)."""
    return TileBatch(ctx, requests, outputs).launch().finish()


def set_graphs(ctx: Context, on: bool) -> None:
    """Replay the tile stages as CUDA graphs of persistent kernels."""
    lib().sd_ctx_set_graphs(ctx.handle, int(on))
