"""The debug bounds-checked build (-DSD_BOUNDS_CHECK=1): every radar-image
and DEM gather of the terrain-correction kernels tests its index and records
the first one outside the buffer in a device error word.  On a geographic and
a UTM scene, whole-scene and as tiles, the checked build must record nothing
and produce the same bits as the default build (the checks only skip
accesses that are out of bounds, and there are none).

The checked library is compiled into a temporary directory (nvcc, about a
minute) and driven from a child process through SARDINE_B200_LIB."""
import ctypes as C
import json
import os
import subprocess
import sys

import numpy as np
import pytest

import sardine_b200 as sd
from sardine_b200 import _lib, build

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))

# Runs in the child (and in this process with the default build): writes the
# rasters to out_dir and prints the bounds word.
RUN = r'''
import ctypes as C, copy, json, os, sys
import numpy as np
sys.path.insert(0, sys.argv[2])
import oracle
import sardine_b200 as sd
from sardine_b200 import _lib, synth, tiles

def run(out_dir, ctx):
    res = {}
    sc = synth.config1_scene(seed=41, n_lines=512, n_samples=1024, dem_n=160, flatten=True,
                             resampling=sd.ResamplingKernel.Lanczos3)
    res["geo"] = np.asarray(sd.terrain_correction(sc.merged, sc.scene, sc.dem, sc.grids, sc.config,
                                                  ctx=ctx).data)
    u = synth.config2_scene(seed=21, n_bursts=3, lines_per_burst=400, tiff_width=1500, burst_step=300,
                            swath_overlap=150, out_rows=None, out_cols=None, lut_lines_step=150)
    m = sd.calibrate_deburst_merge(u.swaths, ctx=ctx)
    res["utm"] = np.asarray(sd.terrain_correction(m, u.scene, u.dem, u.grids, u.config, ctx=ctx).data)
    rs = tiles.ResidentScene(m, u.scene, u.dem, u.grids, u.config.geoid, ctx)
    _, g = oracle.tc_output_grid(u.scene, u.config)
    sp = u.config.pixel_spacing_deg
    reqs = []
    for (r0, c0, rows, cols, k, f) in ((5, 7, 90, 120, sd.ResamplingKernel.Bicubic, sd.SpeckleFilter.RefinedLee(4.4)),
                                      (40, 60, 64, 200, sd.ResamplingKernel.Lanczos3, None),
                                      (0, 0, 33, 47, sd.ResamplingKernel.Bilinear, sd.SpeckleFilter.GammaMap(5, 4.4))):
        cfg = copy.copy(u.config)
        cfg.resampling = k
        reqs.append(tiles.TileRequest(rs, cfg, g.origin_lon_deg + c0 * sp, g.origin_lat_deg - r0 * sp,
                                      rows, cols, f))
    for i, t in enumerate(tiles.tc_tiles(reqs, ctx)):
        res[f"tile{i}"] = t.data.cpu().numpy()
    rs.close()
    for k, v in res.items():
        np.save(os.path.join(out_dir, k + ".npy"), v)
    word = (C.c_uint64 * 4)()
    assert _lib.lib().sd_debug_bounds(ctx.handle, word) == 0
    return [int(x) for x in word]

if __name__ == "__main__":
    print(json.dumps(run(sys.argv[1], sd.Context(0))))
'''


def test_bounds_checked_build_records_nothing_and_matches(tmp_path):
    lib_path = build.build(extra_flags=["-DSD_BOUNDS_CHECK=1"], out=str(tmp_path / "libsardine_b200.so"))
    script = tmp_path / "run_bounds.py"
    script.write_text(RUN)
    repo = os.path.dirname(HERE)
    checked_dir = tmp_path / "checked"
    checked_dir.mkdir()
    env = dict(os.environ, SARDINE_B200_LIB=lib_path)
    out = subprocess.run([sys.executable, str(script), str(checked_dir), repo], env=env, capture_output=True,
                         text=True, timeout=900, cwd=repo)
    assert out.returncode == 0, out.stderr[-3000:]
    word = json.loads(out.stdout.strip().splitlines()[-1])
    assert word[3] == 1, "the child did not load the checked build"
    assert word[0] == 0, f"out-of-bounds gather recorded: site {word[0]}, index {word[1]}, extent {word[2]}"
    # the default build, in a child of its own (same script)
    plain_dir = tmp_path / "plain"
    plain_dir.mkdir()
    env.pop("SARDINE_B200_LIB")
    out = subprocess.run([sys.executable, str(script), str(plain_dir), repo], env=env, capture_output=True,
                         text=True, timeout=900, cwd=repo)
    assert out.returncode == 0, out.stderr[-3000:]
    assert json.loads(out.stdout.strip().splitlines()[-1])[3] == 0
    names = sorted(os.listdir(plain_dir))
    assert names == sorted(os.listdir(checked_dir)) and len(names) == 5
    for n in names:
        a, b = np.load(plain_dir / n), np.load(checked_dir / n)
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32)), n
