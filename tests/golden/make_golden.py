"""Regenerates tests/golden/oracle_small_scenes.json: oracle outputs for
small seeded scenes (counters, Newton histogram, SHA-256 of the rasters).

    python tests/golden/make_golden.py

The file pins the oracle against drift; test_golden.py recomputes and
compares.  Run it only after a reviewed change to the oracle.
"""
import hashlib
import json
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402
import sardine_b200 as sd  # noqa: E402
from sardine_b200 import synth  # noqa: E402

HERE = os.path.dirname(os.path.abspath(__file__))


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def cases():
    yield "c1_bilinear_lia", lambda: synth.config1_scene(seed=101, n_lines=512, n_samples=1024, dem_n=96)
    yield "c1_bicubic_flatten", lambda: synth.config1_scene(
        seed=102, n_lines=512, n_samples=1024, dem_n=96, flatten=True,
        resampling=sd.ResamplingKernel.Bicubic)
    yield "c1_lanczos_flatten", lambda: synth.config1_scene(
        seed=103, n_lines=512, n_samples=1024, dem_n=96, flatten=True,
        resampling=sd.ResamplingKernel.Lanczos3)


def iw_case():
    sc = synth.config2_scene(seed=104, n_bursts=2, lines_per_burst=300, tiff_width=700,
                             burst_step=200, swath_overlap=60, out_rows=None, out_cols=None,
                             lut_lines_step=100)
    inputs = []
    for s in sc.swaths:
        deb = oracle.deburst_subswath(s.slc, s.sw, s.bursts)
        sig = oracle.apply_calibration(deb, s.cal, s.noise, s.bursts[0].first_line)
        inputs.append(sd.SwathInput(sig, s.sw, s.bursts[0].azimuth_time_us))
    m, _ = oracle.merge_subswaths(inputs)
    return sc, m


def compute():
    out = {}
    for name, mk in cases():
        sc = mk()
        r = oracle.terrain_correction(sc.merged, sc.scene, sc.dem, sc.grids, sc.config)
        out[name] = {
                     "rows": r.rows, "cols": r.cols,
                     "counters": {k: getattr(r, k) for k in (
                         "valid_pixel_count", "dem_missing_count", "outside_footprint_count",
                         "non_converged_count", "degenerate_geometry_count", "flat_masked_count",
                         "noise_masked_count")},
                     "hist": r.newton_iter_histogram, "data_sha256": sha(r.data),
                     "mask_sha256": sha(r.mask), "cos_lia_sha256": sha(r.cos_lia)}
    sc, m = iw_case()
    r = oracle.terrain_correction(m, sc.scene, sc.dem, sc.grids, sc.config)
    out["iw_utm_bicubic_flatten"] = {
        "merged_shape": [m.lines, m.samples], "merged_sha256": sha(m.data), "nesz_sha256": sha(m.nesz),
        "rows": r.rows, "cols": r.cols,
        "counters": {k: getattr(r, k) for k in (
            "valid_pixel_count", "dem_missing_count", "outside_footprint_count",
            "non_converged_count", "degenerate_geometry_count", "flat_masked_count",
            "noise_masked_count")},
        "hist": r.newton_iter_histogram, "data_sha256": sha(r.data), "mask_sha256": sha(r.mask)}
    return out


if __name__ == "__main__":
    res = compute()
    with open(os.path.join(HERE, "oracle_small_scenes.json"), "w") as f:
        json.dump(res, f, indent=1, sort_keys=True)
    print(json.dumps({k: v["counters"] for k, v in res.items()}, indent=1))
