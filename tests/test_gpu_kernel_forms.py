"""The parameter forms of k_row_anchors, k_heights and k_cand (the job
record as a kernel parameter) against their persistent work-table forms:
the same device functions on the same inputs, so the outputs must be equal
bit for bit.  A geographic and a UTM scene, whole-scene and as a tile batch
in the per-tile launch mode, run in two child processes, one with
SARDINE_B200_{ANCHORS,HEIGHTS,CAND}_PARAM=0 (each switch is read once per
process)."""
import os
import subprocess
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))

RUN = r'''
import copy, os, sys
import numpy as np
sys.path.insert(0, sys.argv[2])
import oracle
import sardine_b200 as sd
from sardine_b200 import autotune, synth, tiles

ctx = sd.Context(0)
autotune.apply(ctx, {"speckle": [32, 8], "main_cps": -1})  # tiles: per-tile launches
res = {}
sc = synth.config1_scene(seed=43, n_lines=512, n_samples=1024, dem_n=160, flatten=True,
                         resampling=sd.ResamplingKernel.Bicubic)
g1 = sd.terrain_correction(sc.merged, sc.scene, sc.dem, sc.grids, sc.config, ctx=ctx, return_times=True)
res["geo"] = np.asarray(g1.data)
res["geo_t"] = np.asarray(g1.azimuth_time_us)
u = synth.config2_scene(seed=23, n_bursts=3, lines_per_burst=400, tiff_width=1500, burst_step=300,
                        swath_overlap=150, out_rows=None, out_cols=None, lut_lines_step=150)
m = sd.calibrate_deburst_merge(u.swaths, ctx=ctx)
cfg = copy.copy(u.config)
cfg.precision = sd.Precision.SPLIT
cfg.resampling = sd.ResamplingKernel.Lanczos3
g2 = sd.terrain_correction(m, u.scene, u.dem, u.grids, cfg, ctx=ctx)
res["utm"] = np.asarray(g2.data)
res["utm_cos"] = np.asarray(g2.cos_lia) if g2.cos_lia is not None else np.zeros(1)
rs = tiles.ResidentScene(m, u.scene, u.dem, u.grids, u.config.geoid, ctx)
_, g = oracle.tc_output_grid(u.scene, u.config)
sp = u.config.pixel_spacing_deg
reqs = []
for (r0, c0, rows, cols, k, prec, f) in (
        (5, 7, 90, 120, sd.ResamplingKernel.Bicubic, sd.Precision.SPLIT, sd.SpeckleFilter.RefinedLee(4.4)),
        (40, 60, 64, 200, sd.ResamplingKernel.Lanczos3, sd.Precision.FP64, None),
        (0, 0, 33, 47, sd.ResamplingKernel.Bilinear, sd.Precision.SPLIT, sd.SpeckleFilter.GammaMap(5, 4.4)),
        (20, 30, 128, 96, sd.ResamplingKernel.Bilinear, sd.Precision.FP64, None)):
    c = copy.copy(u.config)
    c.resampling = k
    c.precision = prec
    reqs.append(tiles.TileRequest(rs, c, g.origin_lon_deg + c0 * sp, g.origin_lat_deg - r0 * sp, rows, cols, f))
for i, t in enumerate(tiles.tc_tiles(reqs, ctx)):
    res[f"tile{i}"] = t.data.cpu().numpy()
    res[f"tile{i}_mask"] = t.mask.cpu().numpy() if t.mask is not None else np.zeros(1)
rs.close()
for k, v in res.items():
    np.save(os.path.join(sys.argv[1], k + ".npy"), v)
print("ok")
'''


def _run(script, out_dir, repo, env):
    out = subprocess.run([sys.executable, str(script), str(out_dir), repo], env=env, capture_output=True,
                         text=True, timeout=900, cwd=repo)
    assert out.returncode == 0, out.stdout[-2000:] + out.stderr[-4000:]


def test_parameter_forms_equal_work_table_forms(tmp_path):
    repo = os.path.dirname(HERE)
    script = tmp_path / "run_forms.py"
    script.write_text(RUN)
    a, b = tmp_path / "param", tmp_path / "table"
    a.mkdir()
    b.mkdir()
    _run(script, a, repo, dict(os.environ))
    off = dict(os.environ, SARDINE_B200_ANCHORS_PARAM="0", SARDINE_B200_HEIGHTS_PARAM="0",
               SARDINE_B200_CAND_PARAM="0")
    _run(script, b, repo, off)
    names = sorted(f for f in os.listdir(a) if f.endswith(".npy"))
    assert names and names == sorted(os.listdir(b))
    for f in names:
        x, y = np.load(a / f), np.load(b / f)
        assert x.shape == y.shape, f
        assert x.tobytes() == y.tobytes(), f"{f}: parameter and work-table forms differ"
    valid = np.load(a / "geo.npy")
    assert np.isfinite(valid).sum() > 0
