"""Multi-rank decomposition on CPU (gloo, world size 2): row bands of one
scene plus a speckle halo exchange reproduce the whole-grid result; tile
placement balances pixels.  The geocoding itself runs in the oracle here
(the GPU path's row bands are checked against whole-grid calls in
test_gpu_tc.py)."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

from sardine_b200.shard import assign_tiles, row_bands


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, out_dir):
    import datetime

    import torch.distributed as dist

    import oracle
    import sardine_b200 as sd
    from sardine_b200 import synth
    from sardine_b200.shard import exchange_halo, gather_rows, row_bands

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        oracle.set_threads(2)
        sc = synth.config1_scene(seed=71, n_lines=256, n_samples=512, dem_n=64, flatten=True)
        _, g = oracle.tc_output_grid(sc.scene, sc.config)
        bands = row_bands(int(g.rows), world)
        r0, r1 = bands[rank]
        band = oracle.terrain_correction(sc.merged, sc.scene, sc.dem, sc.grids, sc.config, row_begin=r0,
                                         row_end=r1)
        filt = sd.SpeckleFilter.RefinedLee(4.4)
        half = 3
        wide = exchange_halo(torch.from_numpy(band.data), half, rank, world).numpy()
        f = oracle.apply_speckle_filter(wide, wide.shape[1], wide.shape[0], filt).reshape(wide.shape)
        mine = torch.from_numpy(np.ascontiguousarray(f[half:half + (r1 - r0)]))
        raw = gather_rows(torch.from_numpy(band.data), bands, rank, world)
        full = gather_rows(mine, bands, rank, world)
        cnt = torch.tensor([band.valid_pixel_count], dtype=torch.int64)
        dist.all_reduce(cnt)
        if rank == 0:
            np.save(os.path.join(out_dir, "raw.npy"), raw.numpy())
            np.save(os.path.join(out_dir, "filtered.npy"), full.numpy())
            np.save(os.path.join(out_dir, "valid.npy"), cnt.numpy())
    finally:
        dist.destroy_process_group()


def test_row_bands_and_halo_exchange_match_whole_grid(tmp_path):
    import oracle
    import sardine_b200 as sd
    from sardine_b200 import synth
    world = 2
    mp.spawn(_worker, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True)
    sc = synth.config1_scene(seed=71, n_lines=256, n_samples=512, dem_n=64, flatten=True)
    whole = oracle.terrain_correction(sc.merged, sc.scene, sc.dem, sc.grids, sc.config)
    filt = oracle.apply_speckle_filter(whole.data, whole.cols, whole.rows,
                                       sd.SpeckleFilter.RefinedLee(4.4)).reshape(whole.data.shape)
    assert np.array_equal(np.load(tmp_path / "raw.npy"), whole.data, equal_nan=True)
    assert np.array_equal(np.load(tmp_path / "filtered.npy"), filt, equal_nan=True)
    assert int(np.load(tmp_path / "valid.npy")[0]) == whole.valid_pixel_count


def test_row_bands_cover_grid():
    for rows, world in [(10, 3), (7, 8), (25000, 8), (1, 1)]:
        b = row_bands(rows, world)
        assert b[0][0] == 0 and b[-1][1] == rows
        assert all(x[1] == y[0] for x, y in zip(b, b[1:]))
        assert max(e - s for s, e in b) - min(e - s for s, e in b) <= 1


def test_assign_tiles_balances_pixels():
    rng = np.random.default_rng(3)
    px = [int(256 * 16 ** rng.uniform()) ** 2 for _ in range(64)]
    parts = assign_tiles(px, 4)
    assert sorted(i for p in parts for i in p) == list(range(64))
    loads = [sum(px[i] for i in p) for p in parts]
    assert max(loads) - min(loads) <= max(px)
