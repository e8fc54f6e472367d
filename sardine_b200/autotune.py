"""Autotuner for the launch shapes of the tile stages.

Two knobs change speed and never results: the block shape of the speckle /
crop stage (a wider block shares its halo over more outputs; a taller one
re-reads fewer rows) and the CTAs per SM of the persistent geocoding kernel.
`tune` times the candidates on the caller's own batch with CUDA events
around each stage, keeps the fastest, and caches the choice per device and
batch signature in a JSON file.
"""
from __future__ import annotations

import json
import math
import os
from typing import Dict, List, Optional, Sequence, Tuple

from ._lib import Context, lib
from .tiles import TileRequest, tc_tiles

SPECKLE_SHAPES: List[Tuple[int, int]] = [(32, 8), (32, 4), (64, 4), (32, 16), (16, 16), (128, 2)]
# 0: persistent over all tiles, as many CTAs as fit; 3, 2: fewer per SM;
# -1: one parameter-form launch per tile over four streams
MAIN_CTAS_PER_SM: List[int] = [0, 3, -1]
DEFAULT = {"speckle": [32, 8], "main_cps": 0}


def cache_path() -> str:
    return os.environ.get("SARDINE_B200_TUNE_CACHE",
                          os.path.join(os.path.expanduser("~"), ".cache", "sardine_b200", "tiles.json"))


def apply(ctx: Context, choice: Dict) -> None:
    tx, ty = choice["speckle"]
    rc = lib().sd_ctx_set_tile_shape(ctx.handle, int(tx), int(ty), int(choice["main_cps"]))
    if rc != 0:
        raise ValueError(ctx.last_error())


def batch_key(device_name: str, requests: Sequence[TileRequest]) -> str:
    px = sum(r.rows * r.cols for r in requests)
    kinds = sorted({-1 if r.speckle is None else int(r.speckle.kind) for r in requests})
    prec = sorted({int(r.config.precision) for r in requests})
    return f"{device_name}|n{len(requests)}|px2^{int(math.log2(max(px, 1)))}|sp{kinds}|p{prec}"


def _stage_ms(ctx: Context, requests, prefixes) -> float:
    lib().sd_ctx_set_timing(ctx.handle, 0)
    lib().sd_ctx_set_timing(ctx.handle, 1)
    tc_tiles(requests, ctx)
    kt = ctx.kernel_times()
    lib().sd_ctx_set_timing(ctx.handle, 0)
    return sum(v[0] for k, v in kt.items() if k.startswith(prefixes))


def tune(ctx: Context, requests: Sequence[TileRequest], repeats: int = 2,
         path: Optional[str] = None, device_name: Optional[str] = None) -> Dict:
    """Picks the speckle block shape, then the geocoding CTAs per SM, by
    timing each candidate `repeats` times on `requests` (after one warm run);
    applies the choice to `ctx` and caches it."""
    if device_name is None:
        import torch
        device_name = torch.cuda.get_device_name(ctx.device)
    path = path or cache_path()
    key = batch_key(device_name, requests)
    cache = {}
    try:
        with open(path) as f:
            cache = json.load(f)
    except (OSError, ValueError):
        cache = {}
    if key in cache:
        apply(ctx, cache[key])
        return cache[key]
    has_speckle = any(r.speckle is not None for r in requests)
    best = dict(DEFAULT)
    scores: Dict[str, float] = {}
    if has_speckle:
        best_ms = None
        for tx, ty in SPECKLE_SHAPES:
            apply(ctx, {"speckle": [tx, ty], "main_cps": 0})
            tc_tiles(requests, ctx)
            ms = min(_stage_ms(ctx, requests, ("k_speckle_tiles",)) for _ in range(repeats))
            scores[f"speckle {tx}x{ty}"] = ms
            if best_ms is None or ms < best_ms:
                best_ms, best["speckle"] = ms, [tx, ty]
    best_ms = None
    for cps in MAIN_CTAS_PER_SM:
        apply(ctx, {"speckle": best["speckle"], "main_cps": cps})
        tc_tiles(requests, ctx)
        ms = min(_stage_ms(ctx, requests, ("k_main", "k_scan")) for _ in range(repeats))
        scores[f"main_cps {cps}"] = ms
        if best_ms is None or ms < best_ms:
            best_ms, best["main_cps"] = ms, cps
    best["scores_ms"] = scores
    apply(ctx, best)
    cache[key] = best
    try:
        os.makedirs(os.path.dirname(path), exist_ok=True)
        with open(path, "w") as f:
            json.dump(cache, f, indent=1)
    except OSError:
        pass
    return best
