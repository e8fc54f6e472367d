#!/usr/bin/env python
"""Benchmark: geocoded pixels per second of the full Sentinel-1 IW pipeline.

Workload (one step): 3 sub-swaths x 9 bursts x 1500 lines x 21000 samples of
CInt16 SLC -> sigma0 calibration with NESZ, TOPS midpoint deburst and IW
merge (one fused pass) -> backward Range-Doppler terrain correction onto a
25000 x 20000 UTM 10 m grid with a 10 m projected DEM (fBm 0-3000 m),
bicubic resampling, gamma0 flattening, LIA and shadow/layover mask, FP64
geometry.  Inputs are seeded synthetic data of that shape (no real S1 data
exists here).  All inputs exceed the 126 MB L2 (SLC 3.4 GB, DEM 2 GB).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--config c2|c1]

Prints one JSON line (rank 0).  `value` = output-grid pixels of all ranks /
max-over-ranks device time of the K timed steps, inputs resident in HBM.
`e2e` = the same metric through the public API with pinned host buffers,
host<->device copies inside the timed region.  Under torchrun (N > 1) every
rank processes its own scene (weak scaling, no data-path collective).
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "geocoded px/s"
UNIT = "px/s"

# Algorithmic work per unit, fixed before measuring:
#  * fused calibrate+deburst+merge: 4 B CInt16 read + 4 B sigma0 + 4 B NESZ
#    written per merged pixel (overlap lines / invalid samples never read).
#  * terrain correction: FP64 operations per output pixel of the reference
#    algorithm, F = N_it * 430 (8-point Lagrange pos/vel/acc + Newton update)
#    + 90 (target ECEF, slant range, image coordinates) + 150 (4 neighbour
#    ECEF + facet normal + flattening/LIA), N_it = mean Newton iterations.
PREP_BYTES_PER_PX = 12.0
TC_FLOPS = lambda n_it: n_it * 430.0 + 90.0 + 150.0


def _rank_env():
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def __enter__(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={q}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for ln in self.proc.stdout:
            self.lines.append(ln.strip())

    def __exit__(self, *a):
        if self.proc is not None:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def make_workload(cfg: str, device: str, seed: int):
    from sardine_b200 import synth
    import sardine_b200 as sd
    if cfg == "c1":
        return synth.config1_scene(seed=seed, device=device)
    if cfg == "c3":
        sc = synth.config2_scene(seed=seed, device=device, resampling=sd.ResamplingKernel.Lanczos3)
        sc.config.precision = sd.Precision.SPLIT
        return sc
    return synth.config2_scene(seed=seed, device=device)


def n_iter_mean(hist):
    h = np.asarray(hist, dtype=np.float64)
    return float((h * np.arange(len(h))).sum() / max(h.sum(), 1.0))


def run_ours(args):
    import torch
    import sardine_b200 as sd
    rank, world, local = _rank_env()
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    ctx = sd.Context(local)
    stream = torch.cuda.ExternalStream(ctx.stream_ptr, device=torch.device("cuda", local))
    sc = make_workload(args.config, f"cuda:{local}", seed=2 + 1000 * rank)

    if args.config == "c1":
        def step():
            return None, sd.terrain_correction(sc.merged, sc.scene, sc.dem, sc.grids, sc.config, ctx=ctx)
        merged_px = 0
        workload = "config1: plain TC, 4096x8192 sigma0 -> 1024x1024 EPSG:4326, bilinear, LIA"
    else:
        m0 = sd.calibrate_deburst_merge(sc.swaths, ctx=ctx)
        mbuf = (m0.data, m0.nesz)
        merged_px = m0.lines * m0.samples
        info = sd.tc_output_grid(sc.scene, sc.config, ctx=ctx)
        dev = torch.device("cuda", local)
        obuf = (torch.empty((info.rows, info.cols), dtype=torch.float32, device=dev),
                torch.empty((info.rows, info.cols), dtype=torch.float32, device=dev),
                torch.empty((info.rows, info.cols), dtype=torch.uint8, device=dev))

        def step():
            m = sd.calibrate_deburst_merge(sc.swaths, ctx=ctx, out=mbuf)
            r = sd.terrain_correction(m, sc.scene, sc.dem, sc.grids, sc.config, ctx=ctx, out=obuf)
            return m, r
        workload = ("config2: full IW scene 3x9x1500x21000 CInt16 -> cal+deburst+merge -> TC "
                    "25000x20000 UTM 10 m, bicubic, gamma0 flatten, LIA+mask, FP64")
        if args.config == "c3":
            workload = ("config3: config2 inputs, lanczos3, split precision (FP64 orbit/Newton/slant "
                        "range, FP32 resampling/facet/flattening), gamma0 flatten, LIA+mask")

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    for _ in range(args.warmup):
        _, res = step()
    barrier()
    launches0 = ctx.launches
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        barrier()
        e0.record(stream)
        for _ in range(args.steps):
            _, res = step()
        e1.record(stream)
        barrier()
    ms = e0.elapsed_time(e1)
    gpu_launches = ctx.launches - launches0
    if dist is not None:
        t = torch.tensor([ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    px_step = res.total_pixel_count
    value = world * px_step * args.steps / (ms / 1e3)
    n_it = n_iter_mean(res.newton_iter_histogram)

    # per-kernel breakdown: one more step with CUDA events around every launch
    ctx.set_timing(True)
    step()
    kt = ctx.kernel_times()
    ctx.set_timing(False)
    total_k = sum(v[0] for v in kt.values()) or 1.0
    tc_names = [k for k in kt if k.startswith(("k_main", "k_scan", "k_select", "k_row", "k_orbit"))]
    tc_ms = sum(kt[k][0] for k in tc_names)
    prep_ms = sum(kt[k][0] for k in kt if k.startswith(("k_fused", "k_lut_table")))
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        pass
    fp64 = ctypes_fp64_peak(ctx)
    dominant = max(kt.items(), key=lambda kv: kv[1][0])[0] if kt else None
    # Roofline of the dominant stage: the terrain-correction operator (its
    # kernels run back to back on one stream) against the measured FP64 peak.
    tc_flops = TC_FLOPS(n_it) * px_step
    tc_tflops = tc_flops / (tc_ms / 1e3) / 1e12 if tc_ms > 0 else None
    roofline = {
        "bound": "fp64", "kernel": "terrain_correction (" + "+".join(sorted(tc_names)) + ")",
        "achieved": tc_tflops, "peak": fp64, "unit": "TFLOP/s",
        "frac": (tc_tflops / fp64) if (tc_tflops and fp64) else None,
        "peak_source": "measured FP64 FMA-chain on this GPU (sd_measure_fp64_peak)",
        "flops_per_px": TC_FLOPS(n_it), "newton_iters_mean": n_it,
        "traffic": None,
        "stage_ms": tc_ms, "share": tc_ms / total_k,
    }
    if merged_px:
        hbm = float(peaks.get("hbm_gbs", 6650.0))
        ach = PREP_BYTES_PER_PX * merged_px / (kt.get("k_fused", (0, 1))[0] / 1e3) / 1e9 if "k_fused" in kt else None
        roofline["prep_kernel"] = {"kernel": "k_fused", "bound": "hbm", "achieved": ach, "peak": hbm,
                                   "unit": "GB/s", "frac": ach / hbm if ach else None,
                                   "bytes_per_px": PREP_BYTES_PER_PX, "ms": kt.get("k_fused", (0,))[0]}
    kernels = {k: {"ms": round(v[0], 3), "launches": v[1], "share": round(v[0] / total_k, 4)}
               for k, v in sorted(kt.items(), key=lambda kv: -kv[1][0])}

    e2e = run_e2e(args, sd, sc, ctx, stream, barrier, dist) if (args.config in ("c2", "c3") and args.e2e) else None
    accuracy = split_accuracy(sd, sc, ctx, stream) if args.config == "c3" else None

    if rank == 0:
        out = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded Sentinel-1 IW shapes; no real S1 data available)",
            "config": {"workload": workload, "output_px": px_step, "merged_px": merged_px,
                       "l2": "inputs larger than L2 (SLC 3.4 GB, DEM 2 GB)",
                       "parallelism": f"replicas x{world} (independent scenes)"},
            "roofline": roofline, "kernels": kernels, "dominant_kernel": dominant,
            "gpu_launches": gpu_launches, "clocks": clk.summary(),
            "e2e": e2e,
        }
        if accuracy is not None:
            out["accuracy_vs_fp64"] = accuracy
        if args.cpu_baseline and world == 1:
            out["cpu_baseline"] = cpu_baseline(args, sc, res, merged_px)
        print(json.dumps(out), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    ctx.close()


def split_accuracy(sd, sc, ctx, stream):
    """Split-precision result against the FP64 GPU path on the full scene
    (the FP64 path is checked against the oracle by the test suite), plus
    the FP64 path's own step time on the same inputs."""
    import copy
    import torch
    m = sd.calibrate_deburst_merge(sc.swaths, ctx=ctx)
    split = sd.terrain_correction(m, sc.scene, sc.dem, sc.grids, sc.config, ctx=ctx, return_times=True)
    cfg64 = copy.copy(sc.config)
    cfg64.precision = sd.Precision.FP64
    sd.terrain_correction(m, sc.scene, sc.dem, sc.grids, cfg64, ctx=ctx)  # warm
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    ref = sd.terrain_correction(m, sc.scene, sc.dem, sc.grids, cfg64, ctx=ctx, return_times=True)
    e1.record(stream)
    torch.cuda.synchronize()
    from sardine_b200.accuracy import compare_geocoded
    rep = compare_geocoded(split, ref, split.azimuth_time_us, ref.azimuth_time_us,
                           sc.scene.sub_swaths[0].azimuth_time_interval_s)
    rep["fp64_tc_ms"] = e0.elapsed_time(e1)
    rep["fp64_tc_px_per_s"] = ref.total_pixel_count / (rep["fp64_tc_ms"] / 1e3)
    rep["counters_equal"] = (split.newton_iter_histogram == ref.newton_iter_histogram and
                             split.valid_pixel_count == ref.valid_pixel_count and
                             split.flat_masked_count == ref.flat_masked_count)
    return rep


def ctypes_fp64_peak(ctx):
    import ctypes as C
    from sardine_b200 import _lib
    best = None
    for _ in range(3):
        v = C.c_double()
        if _lib.lib().sd_measure_fp64_peak(ctx.handle, 20000, C.byref(v)) == 0:
            best = v.value if best is None else max(best, v.value)
    return best


def run_e2e(args, sd, sc, ctx, stream, barrier, dist):
    """Same metric through the public API with pinned host buffers: H2D of the
    SLC rasters and the DEM, D2H of sigma0, cos(LIA) and the mask, per step."""
    import torch
    host_swaths = []
    h2d = 0
    for s in sc.swaths:
        hs = torch.empty(tuple(s.slc.shape), dtype=torch.int16, pin_memory=True)
        hs.copy_(s.slc)
        h2d += hs.numel() * 2
        host_swaths.append(type(s)(s.id, hs, s.sw, s.bursts, s.cal, s.noise))
    for s in sc.swaths:
        for v in s.cal.vectors:
            h2d += v.pixels.nbytes + v.sigma_nought.nbytes
        for v in s.noise.range_vectors:
            h2d += v.pixels.nbytes + v.noise_range_lut.nbytes
    hdem = torch.empty(tuple(sc.dem.data.shape), dtype=torch.float32, pin_memory=True)
    hdem.copy_(sc.dem.data)
    h2d += hdem.numel() * 4
    dem_h = sd.DemGrid(hdem, sc.dem.origin_y, sc.dem.origin_x, sc.dem.pixel_size, sc.dem.kind,
                       sc.dem.utm_zone, sc.dem.utm_south)
    info = sd.tc_output_grid(sc.scene, sc.config, ctx=ctx)
    R, Cc = int(info.rows), int(info.cols)
    hout = (torch.empty((R, Cc), dtype=torch.float32, pin_memory=True),
            torch.empty((R, Cc), dtype=torch.float32, pin_memory=True),
            torch.empty((R, Cc), dtype=torch.uint8, pin_memory=True))
    d2h = R * Cc * 9
    m0 = sd.calibrate_deburst_merge(sc.swaths, ctx=ctx)
    mbuf = (m0.data, m0.nesz)

    def step():
        m = sd.calibrate_deburst_merge(host_swaths, ctx=ctx, out=mbuf)
        return sd.terrain_correction(m, sc.scene, dem_h, sc.grids, sc.config, ctx=ctx, out=hout)

    for _ in range(max(1, min(args.warmup, 2))):
        step()
    barrier()
    t0 = time.perf_counter()
    n = max(1, min(args.steps, 3))
    for _ in range(n):
        r = step()
    barrier()
    dt = time.perf_counter() - t0
    if dist is not None:
        t = torch.tensor([dt], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        dt = float(t.item())
    world = dist.get_world_size() if dist is not None else 1
    return {"value": world * r.total_pixel_count * n / dt, "unit": UNIT, "h2d_bytes_per_step": int(h2d),
            "d2h_bytes_per_step": int(d2h), "steps": n,
            "api": "sardine_b200.calibrate_deburst_merge + terrain_correction, pinned host buffers"}


def cpu_baseline(args, sc, res_gpu, merged_px, threads=None, budget_s=12.0):
    """The oracle (C++ restatement of the reference) on the host cores over a
    bounded sample of the same workload: the full fused prep is timed at full
    size; the terrain correction on a band of output rows."""
    import torch
    import oracle
    import sardine_b200 as sd
    from sardine_b200 import types as T
    threads = threads or os.cpu_count()
    oracle.set_threads(threads)
    out = {"unit": UNIT, "cores": threads, "kind": "port"}
    if merged_px:
        swaths_h = [type(s)(s.id, s.slc.cpu().numpy(), s.sw, s.bursts, s.cal, s.noise) for s in sc.swaths]
        t0 = time.perf_counter()
        inputs = []
        for s in swaths_h:
            deb = oracle.deburst_subswath(s.slc, s.sw, s.bursts)
            sig = oracle.apply_calibration(deb, s.cal, s.noise, s.bursts[0].first_line)
            inputs.append(sd.SwathInput(sig, s.sw, s.bursts[0].azimuth_time_us))
        merged, _ = oracle.merge_subswaths(inputs)
        t_prep = time.perf_counter() - t0
        del inputs
    else:
        merged = sc.merged
        merged = T.MergedSigma0(np.asarray(merged.data.cpu()), merged.lines, merged.samples,
                                merged.near_slant_range_time_s, merged.range_pixel_spacing_s,
                                merged.range_pixel_spacing_m, 0, 0, None, merged.azimuth_start_time_us)
        t_prep = 0.0
    dem_h = sd.DemGrid(sc.dem.data.cpu().numpy() if hasattr(sc.dem.data, "cpu") else sc.dem.data,
                       sc.dem.origin_y, sc.dem.origin_x, sc.dem.pixel_size, sc.dem.kind,
                       sc.dem.utm_zone, sc.dem.utm_south)
    rows = res_gpu.rows
    # calibrate the band size with a short probe, then run ~budget_s
    r0 = rows // 2
    t0 = time.perf_counter()
    oracle.terrain_correction(merged, sc.scene, dem_h, sc.grids, sc.config, row_begin=r0, row_end=r0 + 4)
    t_probe = (time.perf_counter() - t0) / 4
    band = int(max(4, min(rows - r0, budget_s / max(t_probe, 1e-4))))
    t0 = time.perf_counter()
    oracle.terrain_correction(merged, sc.scene, dem_h, sc.grids, sc.config, row_begin=r0, row_end=r0 + band)
    t_band = time.perf_counter() - t0
    t_tc_full = t_band / band * rows
    value = res_gpu.total_pixel_count / (t_prep + t_tc_full)
    out.update({"value": value, "prep_s_full": t_prep, "tc_s_per_row": t_band / band,
                "sample": (f"full-size fused prep ({merged_px} merged px) + terrain correction on "
                           f"{band} of {rows} output rows (rows {r0}..{r0 + band}); value = output px / "
                           f"(prep time + per-row TC time x rows)")})
    return out


def run_reference(args):
    """Reference arm: the reference is Rust and cannot be built here, so the
    oracle port (its C++ restatement) is timed on the host cores, each step a
    bounded sample of the same workload."""
    rank, world, _ = _rank_env()
    if rank != 0:
        return
    import oracle
    import sardine_b200 as sd
    from sardine_b200 import synth
    threads = os.cpu_count()
    oracle.set_threads(threads)
    dev = None
    try:
        import torch
        if torch.cuda.is_available():
            dev = "cuda"
    except Exception:
        pass
    sc = make_workload(args.config, dev, seed=2)
    if args.config == "c1":
        merged = sd.MergedSigma0(np.asarray(sc.merged.data.cpu() if dev else sc.merged.data), *[
            getattr(sc.merged, k) for k in ("lines", "samples", "near_slant_range_time_s",
                                            "range_pixel_spacing_s", "range_pixel_spacing_m",
                                            "cal_lut_extrapolation_gap_px",
                                            "noise_lut_extrapolation_gap_px")], None,
            sc.merged.azimuth_start_time_us)
        prep = lambda: merged
    else:
        swaths_h = [type(s)(s.id, s.slc.cpu().numpy() if dev else s.slc, s.sw, s.bursts, s.cal, s.noise)
                    for s in sc.swaths]

        def prep():
            inputs = []
            for s in swaths_h:
                deb = oracle.deburst_subswath(s.slc, s.sw, s.bursts)
                sig = oracle.apply_calibration(deb, s.cal, s.noise, s.bursts[0].first_line)
                inputs.append(sd.SwathInput(sig, s.sw, s.bursts[0].azimuth_time_us))
            return oracle.merge_subswaths(inputs)[0]
    dem_h = sd.DemGrid(sc.dem.data.cpu().numpy() if dev else sc.dem.data, sc.dem.origin_y,
                       sc.dem.origin_x, sc.dem.pixel_size, sc.dem.kind, sc.dem.utm_zone,
                       sc.dem.utm_south)
    t0 = time.perf_counter()
    merged = prep()
    t_prep = time.perf_counter() - t0
    rc, info = oracle.tc_output_grid(sc.scene, sc.config)
    rows, total = int(info.rows), int(info.total_pixel_count)
    band = args.ref_rows
    r0 = rows // 2 - band // 2
    per_row = []
    for i in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        oracle.terrain_correction(merged, sc.scene, dem_h, sc.grids, sc.config, row_begin=r0,
                                  row_end=r0 + band)
        if i >= args.warmup:
            per_row.append((time.perf_counter() - t0) / band)
    t_row = float(np.mean(per_row))
    value = total / (t_prep + t_row * rows)
    sample = (f"oracle port, {threads} threads: full-size prep ({t_prep:.1f} s) + TC on a {band}-row band "
              f"per step, extrapolated to {rows} rows")
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
        "ms_per_step": 1e3 * (t_prep + t_row * rows), "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded Sentinel-1 IW shapes)",
        "config": {"workload": args.config},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                         "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "note": "reference (Rust) unbuildable here: no cargo/rustc and crates not vendored; "
                "the C++ oracle port stands in",
    }), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="c2", choices=["c2", "c1", "c3"])
    ap.add_argument("--no-cpu-baseline", dest="cpu_baseline", action="store_false")
    ap.add_argument("--no-e2e", dest="e2e", action="store_false")
    ap.add_argument("--ref-rows", type=int, default=16)
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
