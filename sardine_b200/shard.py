"""Multi-GPU decomposition (host side), one process per GPU.

* One scene over N GPUs: the output grid is cut into contiguous row bands
  (`row_bands`); each rank geocodes its band with
  `terrain_correction(..., row_range=band)`.  Every output row's solve chain
  starts from its own LUT seed, so the bands are independent and equal the
  same rows of the whole grid: no data-path collective.
* A speckle filter over the whole geocoded raster needs `half` rows of each
  neighbouring band: `exchange_halo` swaps them (point-to-point
  torch.distributed; NCCL over NVLink on GPUs, gloo on CPU); the filtered
  band, cropped, equals the same rows of the filter over the whole raster.
* Tiles and served requests: independent jobs, placed by `assign_tiles`
  (longest processing time first, by pixel count).
"""
from __future__ import annotations

import heapq
from typing import List, Sequence, Tuple


def row_bands(rows: int, world: int) -> List[Tuple[int, int]]:
    """Contiguous [r0, r1) bands, sizes differing by at most one row."""
    base, extra = divmod(rows, world)
    out, r = [], 0
    for k in range(world):
        n = base + (1 if k < extra else 0)
        out.append((r, r + n))
        r += n
    return out


def assign_tiles(px: Sequence[int], world: int) -> List[List[int]]:
    """Indices of the tiles each rank processes: largest first onto the
    least-loaded rank."""
    heap = [(0, k) for k in range(world)]
    out: List[List[int]] = [[] for _ in range(world)]
    for i in sorted(range(len(px)), key=lambda i: -px[i]):
        load, k = heapq.heappop(heap)
        out[k].append(i)
        heapq.heappush(heap, (load + px[i], k))
    return out


def exchange_halo(band, half: int, rank: int, world: int, group=None):
    """`band` (rows x cols tensor) widened by `half` rows from each neighbour
    band (NaN beyond the first and last band).  Every rank calls it."""
    import torch
    import torch.distributed as dist
    rows, cols = band.shape
    top = torch.full((half, cols), float("nan"), dtype=band.dtype, device=band.device)
    bot = torch.full((half, cols), float("nan"), dtype=band.dtype, device=band.device)
    if half == 0 or world == 1:
        return torch.cat([top, band, bot], 0)
    if rows < half:
        raise ValueError("band thinner than the halo")
    ops = []
    if rank > 0:
        ops.append(dist.P2POp(dist.isend, band[:half].contiguous(), rank - 1, group))
        ops.append(dist.P2POp(dist.irecv, top, rank - 1, group))
    if rank < world - 1:
        ops.append(dist.P2POp(dist.isend, band[rows - half:].contiguous(), rank + 1, group))
        ops.append(dist.P2POp(dist.irecv, bot, rank + 1, group))
    for w in dist.batch_isend_irecv(ops):
        w.wait()
    return torch.cat([top, band, bot], 0)


def gather_rows(band, bands: Sequence[Tuple[int, int]], rank: int, world: int, group=None):
    """Whole raster on rank 0 (None elsewhere) from every rank's band."""
    import torch
    import torch.distributed as dist
    if world == 1:
        return band
    cols = band.shape[1]
    hmax = max(b - a for a, b in bands)
    pad = torch.full((hmax, cols), float("nan"), dtype=band.dtype, device=band.device)
    pad[: band.shape[0]] = band
    parts = [torch.empty_like(pad) for _ in range(world)] if rank == 0 else None
    dist.gather(pad, parts, dst=0, group=group)
    if rank != 0:
        return None
    return torch.cat([parts[k][: b - a] for k, (a, b) in enumerate(bands)], 0)
