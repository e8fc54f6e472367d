#!/usr/bin/env python
"""Benchmark: geocoded pixels per second of SARdine's hot path on one B200.

Default workload (config 5, served geocoding): 8 Sentinel-1 IW scenes of
config-2 shape (3 sub-swaths x 9 bursts x 1500 x 21000 CInt16, calibrated,
debursted and merged on the device, then resident in HBM with their 10 m UTM
DEM and orbit) receive Poisson streams of tile requests (sides 256-2048
log-uniform, random scene, bounding box, resampler and speckle filter, split
precision) at 100, 500 and 2000 req/s, then all queued at once ('max').  A
continuous-batching loop admits them by HBM budget into two overlapping
slots.  `value` = geocoded output pixels per second of device time with every
request queued at once (the saturated throughput); p50/p99 request latency
per Poisson rate; the plain per-request FP64 path on the same GPU beside it.

Other workloads: --config c2 (one full IW scene per step: fused
calibration+deburst+merge then terrain correction onto 25000 x 20000 UTM
10 m, bicubic, flatten, LIA, FP64), c3 (c2 with lanczos3 in split
precision), c4 (64 uneven tiles over 8 config-1-shape scenes per step,
one persistent launch per stage replayed from a CUDA graph), c1 (plain
terrain correction of the config-1 scene).  Inputs are seeded synthetic
data of those shapes (no real S1 data exists here) and exceed the 126 MB L2.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--config c5|c2|c3|c4|c1]

Prints one JSON line (rank 0).  Under torchrun (N > 1) every rank serves
its own scenes / processes its own scene (weak scaling, no data-path
collective); times are the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import math
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
# every kernel of the terrain-correction stage (the FP64 roofline's time)
TC_STAGE = ("k_main", "k_heights", "k_resample", "k_redo", "k_scan", "k_cand", "k_row")
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


# reduced IW shape for profiler captures (a few GB on the device, inputs
# still larger than L2): 3 sub-swaths x 3 bursts x 1500 x 10000 -> 2000 x 12000
SMALL_IW = dict(n_bursts=3, lines_per_burst=1500, tiff_width=10000, swath_overlap=1000,
                out_rows=2000, out_cols=12000)


def make_workload(cfg: str, device: str, seed: int, small: bool = False):
    from sardine_b200 import synth
    import sardine_b200 as sd
    kw = SMALL_IW if small else {}
    if cfg == "c1":
        return synth.config1_scene(seed=seed, device=device)
    if cfg == "c3":
        sc = synth.config2_scene(seed=seed, device=device, resampling=sd.ResamplingKernel.Lanczos3, **kw)
        sc.config.precision = sd.Precision.SPLIT
        return sc
    return synth.config2_scene(seed=seed, device=device, **kw)


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
    sc = make_workload(args.config, f"cuda:{local}", seed=2 + 1000 * rank, small=args.small)

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

    if args.small:
        workload = "REDUCED SHAPE (profiler capture, not a bench number): " + workload + f" {SMALL_IW}"

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
    tc_names = [k for k in kt if k.startswith(TC_STAGE + ("k_orbit",))]
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
            def gpu_band(b0, b1):
                m = sd.calibrate_deburst_merge(sc.swaths, ctx=ctx) if merged_px else sc.merged
                g = sd.terrain_correction(m, sc.scene, sc.dem, sc.grids, sc.config, ctx=ctx,
                                          row_range=(b0, b1), return_times=True)
                for k in ("data", "cos_lia", "mask", "azimuth_time_us"):
                    v = getattr(g, k)
                    if v is not None and hasattr(v, "cpu"):
                        setattr(g, k, v.cpu().numpy())
                return g
            out["cpu_baseline"] = cpu_baseline(args, sc, res, merged_px, gpu_band=gpu_band)
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
    # the whole FP64 call (host work and the azimuth-time copy included)
    rep["fp64_tc_ms"] = e0.elapsed_time(e1)
    rep["fp64_tc_px_per_s"] = ref.total_pixel_count / (rep["fp64_tc_ms"] / 1e3)
    # like for like with roofline.stage_ms: the FP64 call's TC-stage kernels
    ctx.set_timing(True)
    sd.terrain_correction(m, sc.scene, sc.dem, sc.grids, cfg64, ctx=ctx)
    kt = ctx.kernel_times()
    ctx.set_timing(False)
    rep["fp64_tc_stage_ms"] = sum(v[0] for k, v in kt.items() if k.startswith(TC_STAGE + ("k_orbit",)))
    # split candidates whose FP32 resampling sum failed its error bound (re-sampled in FP64)
    rep["split_fp64_resampled_px"] = int(split.diag_fp64_resampled)
    rep["fp64_kernels_ms"] = {k: round(v[0], 3) for k, v in sorted(kt.items(), key=lambda kv: -kv[1][0])}
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
    # the scene upload alone (the same pinned SLC and DEM bytes to the device)
    dev_bufs = [torch.empty_like(hs, device="cuda") for hs in (*[s.slc for s in host_swaths], hdem)]
    torch.cuda.synchronize()
    u0 = time.perf_counter()
    for d, hs in zip(dev_bufs, (*[s.slc for s in host_swaths], hdem)):
        d.copy_(hs, non_blocking=True)
    torch.cuda.synchronize()
    up_s = time.perf_counter() - u0
    up_bytes = sum(d.numel() * d.element_size() for d in dev_bufs)
    del dev_bufs
    return {"value": world * r.total_pixel_count * n / dt, "unit": UNIT, "h2d_bytes_per_step": int(h2d),
            "d2h_bytes_per_step": int(d2h), "steps": n,
            "scene_upload_ms": round(up_s * 1e3, 2), "scene_upload_gbs": round(up_bytes / up_s / 1e9, 2),
            "api": "sardine_b200.calibrate_deburst_merge + terrain_correction, pinned host buffers"}


def cpu_baseline(args, sc, res_gpu, merged_px, threads=None, budget_s=12.0, gpu_band=None):
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
    ref, ref_t, _ = oracle.terrain_correction(merged, sc.scene, dem_h, sc.grids, sc.config, row_begin=r0,
                                              row_end=r0 + band, return_times=True)
    t_band = time.perf_counter() - t0
    t_tc_full = t_band / band * rows
    value = res_gpu.total_pixel_count / (t_prep + t_tc_full)
    # one thread: the prep of the first sub-swath (scaled by merged pixels)
    # and four output rows
    oracle.set_threads(1)
    t1_prep = 0.0
    if merged_px:
        s = swaths_h[0]
        t0 = time.perf_counter()
        deb = oracle.deburst_subswath(s.slc, s.sw, s.bursts)
        sig = oracle.apply_calibration(deb, s.cal, s.noise, s.bursts[0].first_line)
        t1_prep = (time.perf_counter() - t0) * merged_px / max(1, deb.lines * deb.samples)
        del deb, sig
    t0 = time.perf_counter()
    oracle.terrain_correction(merged, sc.scene, dem_h, sc.grids, sc.config, row_begin=r0, row_end=r0 + 4)
    t1_row = (time.perf_counter() - t0) / 4
    oracle.set_threads(threads)
    out["value_1thread"] = res_gpu.total_pixel_count / (t1_prep + t1_row * rows)
    out["sample_1thread"] = ("one thread: calibrate+deburst of the first sub-swath scaled to all merged px, "
                             "terrain correction of 4 rows scaled to all rows")
    out.update({"value": value, "prep_s_full": t_prep, "tc_s_per_row": t_band / band,
                "sample": (f"full-size fused prep ({merged_px} merged px) + terrain correction on "
                           f"{band} of {rows} output rows (rows {r0}..{r0 + band}); value = output px / "
                           f"(prep time + per-row TC time x rows)")})
    if gpu_band is not None:
        # the GPU product path on the same rows of the full-size scene, against
        # the oracle with glibc's sines and cosines (as timed) and with
        # correctly rounded ones (untimed)
        with oracle.libm("cr"):
            ref_cr, ref_cr_t, _ = oracle.terrain_correction(merged, sc.scene, dem_h, sc.grids, sc.config,
                                                            row_begin=r0, row_end=r0 + band, return_times=True)
        g = gpu_band(r0, r0 + band)
        out["parity_vs_oracle"] = parity_both(g, ref, ref_t, ref_cr, ref_cr_t,
                                              sc.scene.sub_swaths[0].azimuth_time_interval_s)
        out["parity_vs_oracle"]["rows"] = [r0, r0 + band]
    return out


def _neq(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return ~((a == b) | (np.isnan(a) & np.isnan(b)))


def parity_both(g, gl, gl_t, cr, cr_t, ati_s):
    """GPU result against the oracle run with glibc's sines and cosines and
    with correctly rounded ones: the full report against the latter, the
    count of pixels where the two oracle runs differ (glibc not correctly
    rounded) and, outside those, time flips and pixels beyond 1e-4 against
    the former."""
    from sardine_b200.accuracy import compare_geocoded
    rep_cr = compare_geocoded(g, cr, g.azimuth_time_us, cr_t, ati_s)
    rep_cr["counters_equal"] = (g.valid_pixel_count == cr.valid_pixel_count and
                                g.newton_iter_histogram == cr.newton_iter_histogram and
                                g.flat_masked_count == cr.flat_masked_count and
                                g.noise_masked_count == cr.noise_masked_count)
    libm = _neq(gl.data, cr.data) | (np.asarray(gl_t) != np.asarray(cr_t))
    if gl.mask is not None:
        libm |= (np.asarray(gl.mask) != np.asarray(cr.mask)) | _neq(gl.cos_lia, cr.cos_lia)
    keep = ~libm
    a = np.asarray(g.data, np.float64)[keep]
    b = np.asarray(gl.data, np.float64)[keep]
    both = np.isfinite(a) & np.isfinite(b)
    rel = np.abs(a[both] - b[both]) / np.maximum(np.abs(b[both]), 1e-30)
    outside = {
        "px": int(keep.sum()),
        "time_mismatch_px": int((np.asarray(g.azimuth_time_us)[keep] != np.asarray(gl_t)[keep]).sum()),
        "nan_pattern_equal": bool(np.array_equal(np.isfinite(a), np.isfinite(b))),
        "sigma_rel_over_1e-4_px": int((rel > 1e-4).sum()),
        "mask_equal": bool(gl.mask is None or np.array_equal(np.asarray(g.mask)[keep], np.asarray(gl.mask)[keep])),
    }
    keys = ("compared_px", "time_mismatch_px", "geoloc_err_px_max", "nan_pattern_equal", "mask_equal",
            "sigma_rel_over_1e-4_px", "sigma_rel_err_max", "sigma_rel_err_mean", "cos_lia_abs_err_max",
            "counters_equal")
    return {"vs_correctly_rounded_oracle": {k: rep_cr.get(k) for k in keys},
            "oracle_glibc_vs_correctly_rounded_px": int(libm.sum()),
            "oracle_glibc_vs_correctly_rounded_time_px": int((np.asarray(gl_t) != np.asarray(cr_t)).sum()),
            "vs_glibc_oracle_outside_those_px": outside}


# ── config 4: batched multi-scene tiles ─────────────────────────────────────
def _c4_setup(sd, ctx, dev, rank, n_scenes=8, n_tiles=64, precision=None):
    import copy
    import torch
    from sardine_b200 import synth, tiles
    precision = sd.Precision.SPLIT if precision is None else precision
    scenes = []
    for k in range(n_scenes):
        sc, slc, cal, noise = synth.config4_scene(100 + k + 1000 * rank, device=dev)
        L, S = slc.shape[0], slc.shape[1]
        deb = sd.DeburstArray(slc, L, S, 0)
        sig = torch.empty((L, S), dtype=torch.float32, device=dev)
        nesz = torch.empty((L, S), dtype=torch.float32, device=dev)
        sd.apply_calibration(deb, cal, noise, 0, ctx=ctx, out=(sig, nesz))
        m = sc.merged
        merged = sd.MergedSigma0(sig, L, S, m.near_slant_range_time_s, m.range_pixel_spacing_s,
                                 m.range_pixel_spacing_m, 0, 0, nesz, m.azimuth_start_time_us)
        rs = tiles.ResidentScene(merged, sc.scene, sc.dem, sc.grids, sc.config.geoid, ctx)
        cfg = copy.copy(sc.config)
        cfg.pixel_spacing_deg = sc.config.pixel_spacing_deg / 4.0   # output spacing = posting / 4
        info = sd.tc_output_grid(sc.scene, cfg, ctx=ctx)
        scenes.append(dict(sc=sc, deb=deb, cal=cal, noise=noise, sig=sig, nesz=nesz, rs=rs, cfg=cfg,
                           info=info))
    rng = np.random.default_rng(4 + rank)
    specs = synth.random_tiles(rng, [(int(s["info"].rows), int(s["info"].cols)) for s in scenes],
                               n_tiles, 256, 4096)
    reqs = []
    for t in specs:
        s = scenes[t["scene"]]
        cfg = copy.copy(s["cfg"])
        cfg.resampling = t["kernel"]
        cfg.precision = precision
        sp = cfg.pixel_spacing_deg
        reqs.append(tiles.TileRequest(s["rs"], cfg, s["info"].origin_lon_deg + t["c0"] * sp,
                                      s["info"].origin_lat_deg - t["r0"] * sp, t["rows"], t["cols"],
                                      t["speckle"]))
    return scenes, reqs


def run_c4(args):
    import torch
    import sardine_b200 as sd
    from sardine_b200 import autotune, tiles
    rank, world, local = _rank_env()
    torch.cuda.set_device(local)
    dist = _init_dist(world)
    ctx = sd.Context(local)
    stream = torch.cuda.ExternalStream(ctx.stream_ptr, device=torch.device("cuda", local))
    dev = f"cuda:{local}"
    scenes, reqs = _c4_setup(sd, ctx, dev, rank)
    outputs = [tiles._alloc_outputs(r, dev) for r in reqs]
    tune = autotune.tune(ctx, reqs)
    tiles.set_graphs(ctx, True)
    px_step = sum(r.rows * r.cols for r in reqs)

    def step():
        for s in scenes:  # calibrate every scene's SLC into its resident sigma0
            sd.apply_calibration(s["deb"], s["cal"], s["noise"], 0, ctx=ctx, out=(s["sig"], s["nesz"]))
        return tiles.TileBatch(ctx, reqs, outputs).launch().finish()

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    for _ in range(args.warmup):
        res = step()
    barrier()
    l0 = ctx.launches
    evs = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps + 1)]
    with ClockSampler(local) as clk:
        barrier()
        evs[0].record(stream)
        for i in range(args.steps):
            res = step()
            evs[i + 1].record(stream)
        barrier()
    step_ms = [evs[i].elapsed_time(evs[i + 1]) for i in range(args.steps)]
    ms = sum(step_ms)
    gpu_launches = ctx.launches - l0
    ms = _max_over_ranks(dist, ms)
    value = world * px_step * args.steps / (ms / 1e3)
    ctx.set_timing(True)
    step()
    kt = ctx.kernel_times()
    ctx.set_timing(False)
    total_k = sum(v[0] for v in kt.values()) or 1.0
    hist = np.sum([r.newton_iter_histogram for r in res], axis=0)
    n_it = n_iter_mean(hist)
    tc_ms = sum(v[0] for k, v in kt.items() if k.startswith(TC_STAGE))
    fp64 = ctypes_fp64_peak(ctx)
    tc_tf = TC_FLOPS(n_it) * px_step / (tc_ms / 1e3) / 1e12 if tc_ms else None
    sp_ms = kt.get("k_speckle_tiles", (0.0, 0))[0]
    hbm = _hbm_peak()
    sp_gbs = 9.0 * px_step / (sp_ms / 1e3) / 1e9 if sp_ms else None
    roofline = {"bound": "fp64", "kernel": "tile geocoding (" + "+".join(sorted(k for k in kt if k.startswith(TC_STAGE))) + ")",
                "achieved": tc_tf, "peak": fp64, "unit": "TFLOP/s",
                "frac": tc_tf / fp64 if (tc_tf and fp64) else None, "traffic": None,
                "flops_per_px": TC_FLOPS(n_it), "newton_iters_mean": n_it, "stage_ms": tc_ms,
                "speckle_stage": {"kernel": "k_speckle_tiles", "bound": "hbm", "achieved": sp_gbs,
                                  "peak": hbm, "peak_source": _hbm_peak_source(), "unit": "GB/s",
                                  "frac": sp_gbs / hbm if sp_gbs else None,
                                  "bytes_per_px": 9.0, "ms": sp_ms}}
    kernels = {k: {"ms": round(v[0], 3), "launches": v[1], "share": round(v[0] / total_k, 4)}
               for k, v in sorted(kt.items(), key=lambda kv: -kv[1][0])}
    if rank == 0:
        sizes = [r.rows for r in reqs]
        out = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64+f32 (split)",
            "data": "synthetic (seeded config-1-shape scenes, CInt16 SLC + LUTs)",
            "config": {"workload": ("config4: 8 scenes (4096x8192 CInt16, distinct orbits) calibrated on "
                                    "the device each step, 64 tiles 256^2-4096^2 log-uniform at posting/4, "
                                    "mixed bilinear/bicubic/lanczos3, split precision, Refined Lee 7x7 or "
                                    "Gamma-MAP 5x5 (ENL 4.4) after a halo, one persistent launch per stage "
                                    "replayed from a CUDA graph"),
                       "tiles": len(reqs), "tile_px": px_step, "tile_side_min": min(sizes),
                       "tile_side_max": max(sizes), "autotune": tune,
                       "l2": "inputs larger than L2 (SLC 8 x 128 MB, sigma0 8 x 128 MB)",
                       "parallelism": f"replicas x{world}"},
            "latency_ms": {"p50": float(np.percentile(step_ms, 50)), "p99": float(np.percentile(step_ms, 99)),
                           "what": "batch latency (all 64 tiles complete together)"},
            "roofline": roofline, "kernels": kernels, "gpu_launches": gpu_launches, "clocks": clk.summary(),
            "e2e": None,
        }
        if args.cpu_baseline and world == 1:
            def gpu_tiles(rs):  # the same requests through the GPU path, results on the host
                got = []
                for i in range(0, len(rs), 16):
                    for x in tiles.tc_tiles(rs[i:i + 16], ctx):
                        x.data = x.data.cpu().numpy()
                        x.mask = x.mask.cpu().numpy() if x.mask is not None else None
                        x.cos_lia = None
                        got.append(x)
                return got
            out["cpu_baseline"] = _tiles_cpu_baseline(scenes, reqs, gpu_tiles=gpu_tiles)
        print(json.dumps(out), flush=True)
    _finish_dist(dist)
    ctx.close()


def _rl_taps():
    """Taps of the eight Refined Lee directional masks of a 7 x 7 window."""
    def inside(d, dy, dx):
        if dy == 0 and dx == 0:
            return False
        return [1 <= dy <= 3, -3 <= dy <= -1, 1 <= dx <= 3, -3 <= dx <= -1,
                abs(dy - dx) <= 1 and dy + dx >= 1, abs(dy - dx) <= 1 and dy + dx <= -1,
                abs(dy + dx) <= 1 and dx - dy >= 1, abs(dy + dx) <= 1 and dx - dy <= -1][d]
    return [sum(inside(d, dy, dx) for dy in range(-3, 4) for dx in range(-3, 4)) for d in range(8)]


def _speckle_adds(sd, filt):
    """FP64 additions per output pixel of a filter's window statistics, as
    the reference sums them (sum and sum of squares per window, in order)."""
    if filt is None:
        return 0
    if filt.kind == sd._abi.SPECKLE_REFINED_LEE:
        return 2 * sum(_rl_taps())
    w = filt.window
    return 4 * w * w if filt.kind == sd._abi.SPECKLE_FROST else 2 * w * w


# DRAM bytes per output pixel of the TC stage and of the speckle/crop stage on
# the config-5 tile batch in the per-tile kernel forms the served arm runs,
# from one ncu capture (dram__bytes_read.sum + dram__bytes_write.sum of every
# stage launch, profiles/tc_c5_traffic.md).  Reads are complete; writes are a
# lower bound (a small tile's output still in L2 when its launch ends is
# written back outside any launch's count).
C5_TC_TRAFFIC_B_PER_PX = 270.9
C5_SP_TRAFFIC_B_PER_PX = 10.2


def _tile_roofline(sd, tiles, ctx, reqs):
    """Per-stage CUDA-event times of one batch of `reqs` on `ctx` (timing
    replaces graph replay for that batch): the geocoding stage against the
    measured FP64 peak, the speckle/crop stage against measured HBM."""
    ctx.set_timing(True)
    res = tiles.tc_tiles(reqs, ctx)
    kt = ctx.kernel_times()
    ctx.set_timing(False)
    px = sum(r.rows * r.cols for r in reqs)
    hist = np.sum([r.newton_iter_histogram for r in res], axis=0)
    n_it = n_iter_mean(hist)
    tc_ms = sum(v[0] for k, v in kt.items() if k.startswith(TC_STAGE))
    sp_ms = kt.get("k_speckle_tiles", (0.0, 0))[0]
    fp64 = ctypes_fp64_peak(ctx)
    hbm = _hbm_peak()
    tf = TC_FLOPS(n_it) * px / (tc_ms / 1e3) / 1e12 if tc_ms else None
    gbs = 9.0 * px / (sp_ms / 1e3) / 1e9 if sp_ms else None
    adds = sum(_speckle_adds(sd, r.speckle) * r.rows * r.cols for r in reqs)
    add_rate = adds / (sp_ms / 1e3) / 1e12 if sp_ms else None  # T adds/s
    add_peak = fp64 / 2 if fp64 else None  # an add issues at the FMA rate: half the FMA-chain flops
    total = sum(v[0] for v in kt.values()) or 1.0
    roof = {"bound": "fp64", "kernel": "tile geocoding (" + "+".join(sorted(k for k in kt if k.startswith(TC_STAGE))) + ")",
            "achieved": tf, "peak": fp64, "unit": "TFLOP/s", "frac": tf / fp64 if (tf and fp64) else None,
            "traffic": C5_TC_TRAFFIC_B_PER_PX * px,
            "traffic_source": ("ncu dram__bytes_read.sum + dram__bytes_write.sum of every TC-stage launch (per-tile "
                               "forms) on this batch's tile sizes, %.1f B/px x the batch's px "
                               "(profiles/tc_c5_traffic.md); writes a lower bound" % C5_TC_TRAFFIC_B_PER_PX),
            "flops_per_px": TC_FLOPS(n_it), "newton_iters_mean": n_it, "stage_ms": tc_ms,
            "batch": f"{len(reqs)} tiles, {px} px",
            "speckle_stage": {"kernel": "k_speckle_tiles", "bound": "fp64_add", "achieved": add_rate,
                              "peak": add_peak, "unit": "T adds/s",
                              "frac": add_rate / add_peak if (add_rate and add_peak) else None,
                              "adds": adds, "peak_source": "measured FP64 FMA-chain rate / 2 (adds per s)",
                              "hbm_gbs": gbs, "hbm_frac": gbs / hbm if gbs else None,
                              "hbm_peak_source": _hbm_peak_source(), "bytes_per_px": 9.0, "ms": sp_ms,
                              "traffic": C5_SP_TRAFFIC_B_PER_PX * px}}
    kernels = {k: {"ms": round(v[0], 3), "launches": v[1], "share": round(v[0] / total, 4)}
               for k, v in sorted(kt.items(), key=lambda kv: -kv[1][0])}
    return roof, kernels


def _host_scene(s):
    import sardine_b200 as sd
    sc = s["sc"]
    m = s.get("merged") or sc.merged
    sig = s["sig"] if "sig" in s else m.data
    nz = s["nesz"] if "nesz" in s else m.nesz
    merged = sd.MergedSigma0(sig.cpu().numpy() if hasattr(sig, "cpu") else sig, m.lines, m.samples,
                             m.near_slant_range_time_s, m.range_pixel_spacing_s, m.range_pixel_spacing_m, 0, 0,
                             (nz.cpu().numpy() if hasattr(nz, "cpu") else nz) if nz is not None else None,
                             m.azimuth_start_time_us)
    dem = sd.DemGrid(sc.dem.data.cpu().numpy() if hasattr(sc.dem.data, "cpu") else sc.dem.data,
                     sc.dem.origin_y, sc.dem.origin_x, sc.dem.pixel_size, sc.dem.kind,
                     sc.dem.utm_zone, sc.dem.utm_south)
    return merged, dem, sc


def _oracle_tile(merged, dem, sc, r):
    """The oracle on the tile's (halo'd) grid, filtered and cropped as the
    GPU tile is: (geocoded result, cropped geocoded data, cropped filtered
    data or None, cropped mask)."""
    import oracle
    h = r.halo()
    spd = r.config.pixel_spacing_deg
    g = oracle.terrain_correction_grid(merged, sc.scene, dem, sc.grids, r.config, r.origin_x - h * spd,
                                       r.origin_y + h * spd, r.rows + 2 * h, r.cols + 2 * h)
    crop = lambda a: np.asarray(a).reshape(r.rows + 2 * h, r.cols + 2 * h)[h:h + r.rows, h:h + r.cols]
    filt = None
    if r.speckle is not None:
        filt = crop(oracle.apply_speckle_filter(g.data, r.cols + 2 * h, r.rows + 2 * h, r.speckle))
    mask = None if g.mask is None else crop(g.mask)
    return g, crop(g.data), filt, mask


def _tiles_cpu_baseline(scenes, reqs, budget_s=12.0, gpu_tiles=None):
    """The oracle (C++ restatement) on the host cores: geocode + speckle of
    one scene's tiles, smallest first, until ~budget_s of work.  With
    gpu_tiles (a function returning the GPU's results for a list of
    requests) the GPU tiles of the timed sample are compared with the
    oracle's: against the glibc run that was timed and, untimed, against the
    run with correctly rounded sines and cosines."""
    import oracle
    threads = os.cpu_count()
    oracle.set_threads(threads)
    by_req = sorted(range(len(reqs)), key=lambda i: reqs[i].rows * reqs[i].cols)
    # tiles of one scene only (a host copy of a config-2-shape scene is 6 GB)
    first = reqs[by_req[0]].scene
    by_req = [i for i in by_req if reqs[i].scene is first]
    s = next(x for x in scenes if x["rs"] is first)
    merged, dem, sc = _host_scene(s)
    px, t = 0, 0.0
    done = []
    for i in by_req:
        r = reqs[i]
        t0 = time.perf_counter()
        _oracle_tile(merged, dem, sc, r)
        t += time.perf_counter() - t0
        px += r.rows * r.cols
        done.append(r)
        if t > budget_s:
            break
    out = {"value": px / t, "unit": UNIT, "cores": threads, "kind": "port",
           "sample": (f"oracle geocode+speckle of the {len(done)} smallest tiles of one scene among {len(reqs)} "
                      f"requests ({px} px, {t:.1f} s)")}
    # the same tiles on one thread, until ~3 s
    oracle.set_threads(1)
    px1, t1 = 0, 0.0
    for r in done:
        t0 = time.perf_counter()
        _oracle_tile(merged, dem, sc, r)
        t1 += time.perf_counter() - t0
        px1 += r.rows * r.cols
        if t1 > 3.0:
            break
    oracle.set_threads(threads)
    out["value_1thread"] = px1 / t1
    out["sample_1thread"] = f"the smallest of those tiles on 1 thread ({px1} px, {t1:.1f} s)"
    if gpu_tiles is not None:
        # the GPU's geocoded tiles (filters off) and its filtered tiles
        import copy
        bare = []
        for r in done:
            q = copy.copy(r)
            q.speckle = None
            bare.append(q)
        res, filt_res = gpu_tiles(bare), gpu_tiles([r for r in done if r.speckle is not None])
        par = {"tiles": len(done), "px": 0, "filtered_tiles": len(filt_res)}

        def nbad(a, b):
            a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
            both = np.isfinite(a) & np.isfinite(b)
            rel = np.abs(a[both] - b[both]) / np.maximum(np.abs(b[both]), 1e-30)
            return int((rel > 1e-4).sum()), bool(np.array_equal(np.isfinite(a), np.isfinite(b))), int(both.sum())
        for kind in ("glibc", "cr"):
            bad = fbad = 0
            mask_eq = cnt_eq = nan_eq = True
            fi = iter(filt_res)
            with oracle.libm(kind):
                for r, gr in zip(done, res):
                    g, data, fdata, mask = _oracle_tile(merged, dem, sc, r)
                    h = r.halo()
                    b_, eq, n = nbad(gr.data, data if h == 0 else
                                     np.asarray(oracle.terrain_correction_grid(
                                         merged, sc.scene, dem, sc.grids, r.config, r.origin_x, r.origin_y,
                                         r.rows, r.cols).data))
                    bad += b_
                    nan_eq &= eq
                    if kind == "glibc":
                        par["px"] += n
                    if fdata is not None:
                        fbad += nbad(next(fi).data, fdata)[0]
                    if mask is not None and gr.mask is not None and h == 0:
                        mask_eq &= bool(np.array_equal(np.asarray(gr.mask), mask))
                    if h == 0:
                        cnt_eq &= (gr.valid_pixel_count == g.valid_pixel_count and
                                   gr.newton_iter_histogram == g.newton_iter_histogram)
            par[f"vs_{kind}_oracle"] = {"geocoded_px_over_1e-4": bad, "nan_pattern_equal": nan_eq,
                                         "mask_equal": mask_eq, "counters_equal": cnt_eq,
                                         "filtered_px_over_1e-4": fbad}
        par["what"] = ("geocoded tiles (filters off) on each tile's grid, and the filtered tiles; a filter's "
                       "direction and regime choices turn 1e-7 input differences (gamma0 through the f32 "
                       "flattening weight) into larger ones")
        out["parity_vs_oracle"] = par
    return out


# ── config 5: served geocoding ──────────────────────────────────────────────
def _c5_config(args, world):
    """The config-5 workload description; the reference arm prints the same."""
    return {"workload": (f"config5: {args.scenes} config-2-shape scenes resident (merged sigma0+NESZ, "
                         "DEM, orbit table); Poisson tile requests, sides 256-2048 log-uniform, "
                         "random scene/bbox/resampler/speckle, split precision, continuous batching "
                         f"over {args.slots} slots, HBM-budget admission; value at the last rate ('max': "
                         "every request queued at once = saturated throughput)"),
            "rates_req_s": args.rates.split(","), "burst_per_step": args.burst,
            "hbm_budget_gb": args.budget_gb, "max_batch": args.max_batch, "slots": args.slots,
            "parallelism": f"replicas x{world}"}



def _c5_setup(sd, ctx, dev, rank, n_scenes):
    import torch
    from sardine_b200 import synth, tiles
    scenes = []
    for k in range(n_scenes):
        sc = synth.config2_scene(seed=200 + k + 1000 * rank, device=dev)
        m = sd.calibrate_deburst_merge(sc.swaths, ctx=ctx)
        sc.swaths = None  # the SLC leaves HBM; the merged sigma0 + NESZ stay resident
        rs = tiles.ResidentScene(m, sc.scene, sc.dem, sc.grids, sc.config.geoid, ctx)
        info = sd.tc_output_grid(sc.scene, sc.config, ctx=ctx)
        scenes.append(dict(sc=sc, merged=m, rs=rs, cfg=sc.config, info=info))
        torch.cuda.synchronize()
        torch.cuda.empty_cache()
    return scenes


def _c5_requests(sd, scenes, rng, n, precision):
    import copy
    from sardine_b200 import synth, tiles
    specs = synth.random_tiles(rng, [(int(s["info"].rows), int(s["info"].cols)) for s in scenes], n, 256, 2048,
                               speckles=(None, "refined_lee", "gamma_map"))
    reqs = []
    for t in specs:
        s = scenes[t["scene"]]
        cfg = copy.copy(s["cfg"])
        cfg.resampling = t["kernel"]
        cfg.precision = precision
        sp = cfg.pixel_spacing_deg
        reqs.append(tiles.TileRequest(s["rs"], cfg, s["info"].origin_lon_deg + t["c0"] * sp,
                                      s["info"].origin_lat_deg - t["r0"] * sp, t["rows"], t["cols"],
                                      t["speckle"]))
    return reqs


def _arrivals(rng, rate, n):
    """Poisson arrival offsets (s) at `rate` req/s; rate inf ('max') queues
    every request at once, which measures the saturated throughput."""
    if math.isinf(rate):
        return np.zeros(n)
    return np.cumsum(rng.exponential(1.0 / rate, n))


def _rate_key(rate):
    return "max" if math.isinf(rate) else str(int(rate))


_SCHED = {"work_s": 0.0, "batches": 0}


def _serve(server, reqs, arrivals, clock=time.perf_counter):
    """Feeds requests at their arrival offsets (s) and runs the loop dry.
    _SCHED accumulates the host time of the scheduler passes that collected
    or launched a batch (the rest only poll)."""
    t0 = clock()
    tickets = []
    i = 0
    while i < len(reqs) or server.busy():
        now = clock() - t0
        while i < len(reqs) and arrivals[i] <= now:
            tickets.append(server.submit(reqs[i]))
            i += 1
        in_flight = sum(s.batch is not None for s in server.slots)
        s0 = clock()
        done = server.step()
        launched = sum(s.batch is not None for s in server.slots) - in_flight + (1 if done else 0)
        if done or launched > 0:
            _SCHED["work_s"] += clock() - s0
            _SCHED["batches"] += max(launched, 1)
    return tickets


def run_c5(args):
    import torch
    import sardine_b200 as sd
    from sardine_b200 import autotune, tiles
    from sardine_b200.serve import GeocodingServer, latency_summary
    rank, world, local = _rank_env()
    torch.cuda.set_device(local)
    dist = _init_dist(world)
    ctx = sd.Context(local)
    dev = f"cuda:{local}"
    t_prep = time.perf_counter()
    scenes = _c5_setup(sd, ctx, dev, rank, args.scenes)
    t_prep = time.perf_counter() - t_prep
    rng = np.random.default_rng(5 + rank)
    rates = [math.inf if r.strip() == "max" else float(r) for r in args.rates.split(",")]
    budget = args.budget_gb << 30
    server = GeocodingServer(local, hbm_budget=budget, slots=args.slots, max_batch=args.max_batch, graphs=True)
    sample = _c5_requests(sd, scenes, rng, 64, sd.Precision.SPLIT)
    tune = None
    for s in server.slots:
        tune = autotune.tune(s.ctx, sample[:32])
    for _ in range(args.warmup):  # graph capture, allocator, autotuned shapes in place
        reqs = _c5_requests(sd, scenes, rng, args.burst // 4, sd.Precision.SPLIT)
        _serve(server, reqs, _arrivals(rng, rates[-1], len(reqs)))
    # a serving process keeps its long-lived objects out of the collector's
    # generations, so a collection does not stall the scheduler mid-stream
    import gc
    gc.collect()
    gc.freeze()
    by_rate = {}
    lat = None
    value = ms = None
    gpu_launches = 0
    clk_summary = None
    for rate in rates:
        n = (args.burst * args.steps if rate == rates[-1] or math.isinf(rate)
             else int(max(64, min(args.burst * args.steps, rate * 3))))
        reqs = _c5_requests(sd, scenes, rng, n, sd.Precision.SPLIT)
        arrivals = _arrivals(rng, rate, n)
        _SCHED["work_s"], _SCHED["batches"] = 0.0, 0
        l0 = sum(s.ctx.launches for s in server.slots)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with ClockSampler(local) as clk:
            torch.cuda.synchronize()
            e0.record()
            tickets = _serve(server, reqs, arrivals)
            torch.cuda.synchronize()
            e1.record()
            torch.cuda.synchronize()
        summ = latency_summary(tickets)
        summ["host_sched_ms_per_batch"] = 1e3 * _SCHED["work_s"] / max(_SCHED["batches"], 1)
        summ["rate_req_s"] = _rate_key(rate)
        summ["requests"] = n
        by_rate[_rate_key(rate)] = summ
        if not math.isinf(rate):
            lat = (rate, summ)
        if rate == rates[-1]:
            ms = _max_over_ranks(dist, e0.elapsed_time(e1))
            value = _sum_over_ranks(dist, summ["px"]) / (ms / 1e3)
            gpu_launches = sum(s.ctx.launches for s in server.slots) - l0
            clk_summary = clk.summary()
    # end to end: the headline stream again, each result copied to host memory
    # as it completes (the D2H is inside the latency)
    d2h = [0]

    def on_host(t):  # the result planes are in pinned host memory when the request completes
        for plane in (t.result.data, t.result.cos_lia, t.result.mask):
            if plane is not None:
                assert not plane.is_cuda
                d2h[0] += plane.numel() * plane.element_size()
    e2e_server = GeocodingServer(local, hbm_budget=budget, slots=args.slots, max_batch=args.max_batch, graphs=True,
                                 on_done=on_host, host_results=True)
    for s in e2e_server.slots:
        autotune.apply(s.ctx, tune)
    n = args.burst * args.steps
    reqs = _c5_requests(sd, scenes, rng, n, sd.Precision.SPLIT)
    arrivals = _arrivals(rng, rates[-1], n)
    _serve(e2e_server, reqs[:16], arrivals[:16])
    d2h[0] = 0
    t0 = time.perf_counter()
    et = _serve(e2e_server, reqs, arrivals)
    torch.cuda.synchronize()
    e2e_s = time.perf_counter() - t0
    esum = latency_summary(et)
    e2e_s = _max_over_ranks(dist, e2e_s)
    e2e_px = _sum_over_ranks(dist, esum["px"])
    e2e_server.close()
    # the same batched loop with every request in FP64: what split precision
    # itself contributes (same tiles; the arms alternate, best of two each)
    arm_px_s = {"fp64": 0.0, "split": 0.0}
    for _ in range(2):
        for arm, prec in (("split", sd.Precision.SPLIT), ("fp64", sd.Precision.FP64)):
            rq = _c5_requests(sd, scenes, np.random.default_rng(58 + rank), args.burst, prec)
            torch.cuda.synchronize()
            a0 = time.perf_counter()
            asum = latency_summary(_serve(server, rq, np.zeros(len(rq))))
            torch.cuda.synchronize()
            arm_px_s[arm] = max(arm_px_s[arm], asum["px"] / (time.perf_counter() - a0))
    batched_fp64 = {"what": (f"the same {args.burst} requests queued at once through the same 2-slot batched loop "
                             "in FP64 and in split precision (arms alternated, best of two, wall clock)"),
                    "fp64_px_per_s": arm_px_s["fp64"], "split_px_per_s": arm_px_s["split"],
                    "split_over_fp64": arm_px_s["split"] / arm_px_s["fp64"]}
    # plain per-request FP64 path on the same GPU: one tile per launch, no graphs
    base = GeocodingServer(local, hbm_budget=4 << 30, slots=1, max_batch=1, graphs=False)
    nb = max(64, args.burst * args.steps // 2)
    breqs = _c5_requests(sd, scenes, np.random.default_rng(55 + rank), nb, sd.Precision.FP64)
    barr = _arrivals(np.random.default_rng(56), rates[-1], nb)
    _serve(base, breqs[:8], barr[:8])
    bsum = latency_summary(_serve(base, breqs, barr))
    acc = _split_vs_fp64(sd, tiles, server.slots[0].ctx, scenes, rng)
    base.close()
    roofline, kernels = _tile_roofline(sd, tiles, server.slots[0].ctx, sample)
    cpu = None
    if args.cpu_baseline and world == 1:  # tiles of one scene (one 6 GB host copy)
        def gpu_tiles(rs):
            got = []
            for i in range(0, len(rs), 16):
                for x in tiles.tc_tiles(rs[i:i + 16], server.slots[0].ctx):
                    x.data = x.data.cpu().numpy()
                    x.mask = x.mask.cpu().numpy() if x.mask is not None else None
                    x.cos_lia = None
                    got.append(x)
            return got
        cpu = _tiles_cpu_baseline(scenes, _c5_requests(sd, scenes[:1], np.random.default_rng(57), 96,
                                                       sd.Precision.FP64), gpu_tiles=gpu_tiles)
    if rank == 0:
        out = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64+f32 (split)",
            "data": "synthetic (seeded config-2-shape IW scenes resident in HBM)",
            "config": _c5_config(args, world),
            # per Poisson rate (req/s): [p50, p99] request latency in ms, submit -> results on the device
            "latency_p50_p99_ms": {k: [round(v["p50_ms"], 3), round(v["p99_ms"], 3)]
                                   for k, v in by_rate.items() if "p50_ms" in v},
            "clocks": clk_summary, "gpu_launches": gpu_launches,
            "e2e": {"value": e2e_px / e2e_s, "unit": UNIT, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": int(d2h[0] / max(1, args.steps)),
                    "p50_ms": esum["p50_ms"], "p99_ms": esum["p99_ms"],
                    "api": "GeocodingServer(host_results=True): each batch's result planes copied to pinned "
                           "host memory on the slot's stream behind its kernels; a request completes when its "
                           "results are on the host (scenes resident; request inputs are descriptors only)",
                    "scene_prepare_s": round(t_prep, 3),
                    "scene_prepare": (f"{args.scenes} scenes synthesised on the device, calibrated + debursted + "
                                      "merged and made resident before the timed region")},
            "roofline": roofline, "cpu_baseline": cpu,
            "accuracy_split_vs_fp64": acc,
            "per_request_fp64": bsum,
            "batched_fp64_vs_split": batched_fp64,
            "run_details": {"autotune": tune,
                            "scene_device_gb": round(sum(s["rs"].device_bytes for s in scenes) / 2**30, 2)},
            "served_by_rate": by_rate,
            "kernels": kernels,
        }
        print(json.dumps(out), flush=True)
    server.close()
    _finish_dist(dist)


def _split_vs_fp64(sd, tiles, ctx, scenes, rng, n=64):
    """Split-precision tiles against the same tiles through the FP64 path:
    geocoded values (before any speckle filter: the filters' regime and
    direction choices amplify 1e-7 input differences into flips, counted
    separately), mask, Newton histogram.  Pixel counts are summed over the
    tiles, errors are the worst tile's."""
    import copy
    from sardine_b200.accuracy import compare_geocoded
    reqs = _c5_requests(sd, scenes, rng, n, sd.Precision.SPLIT)
    filtered = [r for r in reqs if r.speckle is not None]
    r64, raw = [], []
    for r in reqs:
        q = copy.copy(r)
        q.speckle = None
        raw.append(q)
        q64 = copy.copy(q)
        q64.config = copy.copy(r.config)
        q64.config.precision = sd.Precision.FP64
        r64.append(q64)
    out = {"tiles": n, "px": 0, "sigma_rel_over_1e-4_px": 0, "sigma_rel_err_max": 0.0,
           "cos_lia_abs_err_max": 0.0, "sigma_db_err_max": 0.0, "nan_pattern_equal": True,
           "mask_equal": True, "hist_equal": True,
           "resamplers": sorted({int(r.config.resampling) for r in reqs})}
    for i in range(0, n, 16):  # batches of 16 tiles bound the device memory
        a = tiles.tc_tiles(raw[i:i + 16], ctx)
        b = tiles.tc_tiles(r64[i:i + 16], ctx)
        for x, y in zip(a, b):
            rep = compare_geocoded(x, y)
            out["px"] += rep["compared_px"]
            out["sigma_rel_over_1e-4_px"] += rep["sigma_rel_over_1e-4_px"]
            for k in ("sigma_rel_err_max", "cos_lia_abs_err_max", "sigma_db_err_max"):
                out[k] = max(out[k], rep.get(k, 0.0))
            out["nan_pattern_equal"] &= rep["nan_pattern_equal"]
            out["mask_equal"] &= rep.get("mask_equal", True)
            out["hist_equal"] &= x.newton_iter_histogram == y.newton_iter_histogram
        del a, b
    if filtered:
        flips, fpx = 0, 0
        for i in range(0, len(filtered), 16):
            part = filtered[i:i + 16]
            f64 = []
            for r in part:
                q = copy.copy(r)
                q.config = copy.copy(r.config)
                q.config.precision = sd.Precision.FP64
                f64.append(q)
            fa, fb = tiles.tc_tiles(part, ctx), tiles.tc_tiles(f64, ctx)
            flips += sum(compare_geocoded(x, y)["sigma_rel_over_1e-4_px"] for x, y in zip(fa, fb))
            fpx += sum(r.rows * r.cols for r in part)
        out["speckled_px_over_1e-4"] = int(flips)
        out["speckled_px"] = int(fpx)
    out["what"] = "geocoded sigma0/gamma0 before speckle; times equal by construction (histogram, mask)"
    return out


def _write_slc_tiff(path, iq):
    """A Sentinel-1-style measurement TIFF of iq ((lines, samples, 2) int16):
    one IFD, LONG strip offsets, one contiguous row per strip."""
    import struct
    h, w = iq.shape[:2]
    tags = [(256, 4, w), (257, 4, h), (258, 3, 32), (259, 3, 1), (273, 4, None), (277, 3, 1), (278, 4, 1),
            (339, 3, 5)]
    table_at = 8 + 2 + 12 * len(tags) + 4
    data_at = table_at + 4 * h
    head = bytearray(b"II" + struct.pack("<HIH", 42, 8, len(tags)))
    for tag, typ, val in tags:
        if tag == 273:
            head += struct.pack("<HHII", 273, 4, h, table_at)
        elif typ == 3:
            head += struct.pack("<HHIHH", tag, typ, 1, val, 0)
        else:
            head += struct.pack("<HHII", tag, typ, 1, val)
    head += struct.pack("<I", 0)
    head += (data_at + np.arange(h, dtype=np.uint64) * (w * 4)).astype("<u4").tobytes()
    with open(path, "wb") as f:
        f.write(bytes(head))
        np.ascontiguousarray(iq, dtype="<i2").tofile(f)


def run_ingest(args):
    """SLC ingest feeding the fused calibrate+deburst+merge: the three
    sub-swath measurement TIFFs of a config-2 scene (3 x 13,500 x 21,000
    CInt16, 3.4 GB, on the machine's local disk, in its page cache after the
    warm-up) are read through SlcReader straight into device buffers, then
    calibrated, debursted and merged.  value = merged pixels per second of
    the whole step; the read alone is reported in GB/s."""
    import torch
    import sardine_b200 as sd
    rank, world, local = _rank_env()
    torch.cuda.set_device(local)
    dist = _init_dist(world)
    ctx = sd.Context(local)
    dev = f"cuda:{local}"
    sc = make_workload("c2", dev, seed=2 + 1000 * rank, small=args.small)
    paths, bufs = [], []
    for k, s in enumerate(sc.swaths):
        p = f"/tmp/sardine_b200_slc_r{rank}_{k}.tiff"
        _write_slc_tiff(p, s.slc.cpu().numpy())
        paths.append(p)
        bufs.append(torch.empty_like(s.slc))
    swaths = [type(s)(s.id, b, s.sw, s.bursts, s.cal, s.noise) for s, b in zip(sc.swaths, bufs)]
    m0 = sd.calibrate_deburst_merge(sc.swaths, ctx=ctx)
    mbuf = (m0.data, m0.nesz)
    slc_bytes = sum(b.numel() * 2 for b in bufs)

    readers = [sd.SlcReader.open(p, ctx=ctx) for p in paths]  # open once, as a pipeline run does

    def read_all():
        for r, b in zip(readers, bufs):
            r.read_burst_raw(0, r.height, out=b)

    for _ in range(args.warmup):
        read_all()
        sd.calibrate_deburst_merge(swaths, ctx=ctx, out=mbuf)
    t_read = t_step = 0.0
    l0 = ctx.launches
    with ClockSampler(local) as clk:
        for _ in range(args.steps):
            torch.cuda.synchronize()
            if dist is not None:
                dist.barrier()
            t0 = time.perf_counter()
            read_all()
            t1 = time.perf_counter()
            m = sd.calibrate_deburst_merge(swaths, ctx=ctx, out=mbuf)
            torch.cuda.synchronize()
            t2 = time.perf_counter()
            t_read += t1 - t0
            t_step += t2 - t0
    t_read = _max_over_ranks(dist, t_read) / args.steps
    t_step = _max_over_ranks(dist, t_step) / args.steps
    ok = bool(torch.equal(m.data, m0.data))
    merged_px = int(m.lines) * int(m.samples)
    # pre-TC multilook of the merged image (4 range looks), HBM-bound
    ml = None
    if rank == 0:
        for _ in range(2):
            sd.apply_multilook(m, 4, 1, 2.055556e-3, ctx=ctx)
        ctx.set_timing(True)
        for _ in range(3):
            mo = sd.apply_multilook(m, 4, 1, 2.055556e-3, ctx=ctx)
        kt = ctx.kernel_times()
        ctx.set_timing(False)
        ml_ms = kt["k_multilook"][0] / 3
        ml_bytes = 8 * merged_px + 8 * int(mo.lines) * int(mo.samples)
        ml = {"looks": "4x1", "ms": ml_ms, "gbs": ml_bytes / (ml_ms / 1e3) / 1e9,
              "frac_of_hbm": ml_bytes / (ml_ms / 1e3) / 1e9 / _hbm_peak(), "bytes": ml_bytes}
        # ground range at 10 m (synthetic incidence grids of three overlapping sub-swaths, 30-46 deg)
        from sardine_b200.types import GeolocationGridPoint as GP
        S = int(m.samples)
        grids = []
        for k, (c0, c1) in enumerate([(0, 0.40 * S), (0.33 * S, 0.72 * S), (0.66 * S, S - 1)]):
            pts = [GP(0, 0.0, 0.0, m.near_slant_range_time_s + (c0 + (c1 - c0) * i / 20) * m.range_pixel_spacing_s,
                      line, 30.0 + 16.0 * (c0 + (c1 - c0) * i / 20) / S) for line in (0, 5000, 10000) for i in range(21)]
            grids.append((f"IW{k + 1}", pts))
        for _ in range(2):
            sd.to_ground_range(m, grids, 10.0, 13.9, ctx=ctx)
        ctx.set_timing(True)
        for _ in range(3):
            g = sd.to_ground_range(m, grids, 10.0, 13.9, ctx=ctx)
        kt = ctx.kernel_times()
        ctx.set_timing(False)
        g_ms = kt["k_grd"][0] / 3
        g_bytes = 4 * merged_px + 4 * g.lines * g.samples  # input read once (neighbouring columns share taps)
        ml["grd"] = {"target_m": 10.0, "out": [g.lines, g.samples], "ms": g_ms,
                     "gbs": g_bytes / (g_ms / 1e3) / 1e9, "frac_of_hbm": g_bytes / (g_ms / 1e3) / 1e9 / _hbm_peak()}
        # TOPS deramping of the first sub-swath as read (CInt16 -> complex f32), nine DC estimates
        # 2.758 s apart with quadratic range terms, line 0 0.8 s before the first
        from sardine_b200.types import DcEstimate, DeburstArray
        sw0 = sc.swaths[0].sw
        est = [DcEstimate(800_000 + int(2.758e6 * k), sw0.slant_range_time_s + 1e-6 * (k % 3),
                          [-40.0 + 10.0 * k, 3.0e4 - 7.0e3 * k, -5.0e6 + 1.3e6 * k]) for k in range(9)]
        sw_dc = type(sw0)(**{**sw0.__dict__, "dc_estimates": est})
        db = DeburstArray(bufs[0], int(bufs[0].shape[0]), int(bufs[0].shape[1]), 0)
        for _ in range(2):
            sd.deramp_subswath(db, sw_dc, 0, ctx=ctx)
        ctx.set_timing(True)
        for _ in range(3):
            dr = sd.deramp_subswath(db, sw_dc, 0, ctx=ctx)
        kt = ctx.kernel_times()
        ctx.set_timing(False)
        d_ms = kt["k_deramp"][0] / 3
        d_px = db.lines * db.samples
        d_bytes = 12 * d_px  # 4 B CInt16 in, 8 B complex f32 out
        del dr
        ml["deramp"] = {"in": [db.lines, db.samples], "ms": d_ms, "gpx_s": d_px / (d_ms / 1e3) / 1e9,
                        "gbs": d_bytes / (d_ms / 1e3) / 1e9,
                        "frac_of_hbm": d_bytes / (d_ms / 1e3) / 1e9 / _hbm_peak()}
        # the oracle's sequential deramp on the first 64 lines, one host thread
        import oracle
        n_cpu = min(64, db.lines)
        db_cpu = DeburstArray(bufs[0][:n_cpu].cpu().numpy(), n_cpu, db.samples, 0)
        t_c = time.perf_counter()
        oracle.deramp_subswath(db_cpu, sw_dc, 0)
        t_c = time.perf_counter() - t_c
        ml["deramp"]["cpu_baseline"] = {"value": n_cpu * db.samples / t_c, "unit": "px/s", "cores": 1,
                                        "kind": "port", "sample": f"{n_cpu} lines x {db.samples} samples"}
    for r in readers:
        r.close()
    for p in paths:
        os.remove(p)
    if rank == 0:
        out = {
            "metric": "merged px/s from measurement TIFFs", "value": world * merged_px / t_step, "unit": "px/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": t_step * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int16 -> f32",
            "data": "synthetic config-2 SLC written as measurement TIFFs",
            "config": {"workload": "ingest: 3 sub-swath TIFFs -> SlcReader into device buffers -> fused "
                                   "calibrate+deburst+merge" + (" (REDUCED SHAPE)" if args.small else ""),
                       "slc_bytes": slc_bytes, "merged_px": merged_px, "parallelism": f"replicas x{world}"},
            "read_gbs": slc_bytes / t_read / 1e9, "read_ms": t_read * 1e3,
            "merged_equal_to_device_input": ok, "multilook": ml, "clocks": clk.summary(),
            "gpu_launches": (ctx.launches - l0) // args.steps,
            "e2e": {"value": world * merged_px / t_step, "unit": "px/s", "h2d_bytes_per_step": slc_bytes,
                    "d2h_bytes_per_step": 0,
                    "api": "sardine_b200.SlcReader.read_burst_raw (device out) + calibrate_deburst_merge"},
            "cpu_baseline": None,
        }
        print(json.dumps(out), flush=True)
    _finish_dist(dist)


def _insar_orbit(baseline=(0.0, 0.0, 0.0), t0_us=0):
    """A circular, 98-degree inclined orbit 700 km up, 15 state vectors 10 s
    apart from t0 - 20 s; `baseline` shifts every position (a secondary pass)."""
    import math
    from sardine_b200.types import OrbitData
    r = 6_378_137.0 + 700_000.0
    w = math.sqrt(3.986004418e14 / r ** 3)
    e1, e2 = np.array([1.0, 0.0, 0.0]), np.array([0.0, math.cos(math.radians(98.0)), math.sin(math.radians(98.0))])
    t = [-20.0 + 10.0 * i for i in range(15)]
    ps = [r * (math.cos(0.7 + w * x) * e1 + math.sin(0.7 + w * x) * e2) + np.array(baseline) for x in t]
    vs = [r * w * (-math.sin(0.7 + w * x) * e1 + math.cos(0.7 + w * x) * e2) for x in t]
    return OrbitData(np.array([t0_us + int(x * 1e6) for x in t], np.int64), np.array(ps), np.array(vs))


def run_insar(args):
    """The InSAR chain of one IW sub-swath pair after deburst (insar/deramp.rs,
    coreg.rs, interferogram.rs): deramp both CInt16 sub-swaths, resample the
    secondary through the degree-2 offset polynomials, then the flat-earth
    phase, cross-product and 10 x 40 coherence (the reference's defaults).
    13,500 x 21,000 pixels (one config-2 sub-swath).  value = reference-grid
    pixels per second of device time of the chain's kernels, inputs resident;
    e2e = the same four public calls from pinned host CInt16 buffers with the
    coherence read back to host memory."""
    import torch
    import sardine_b200 as sd
    from sardine_b200.types import (CoregPoly, Coregistered, DcEstimate, DeburstArray, InterferogramConfig,
                                    SubSwathMetadata)
    rank, world, local = _rank_env()
    torch.cuda.set_device(local)
    dist = _init_dist(world)
    ctx = sd.Context(local)
    dev = f"cuda:{local}"
    lines, samples = (1500, 21000) if args.small else (13500, 21000)
    g = torch.Generator(device=dev).manual_seed(11 + rank)
    ref_iq = torch.randint(-120, 121, (lines, samples, 2), device=dev, dtype=torch.int16, generator=g)
    noise = torch.randint(-40, 41, (lines, samples, 2), device=dev, dtype=torch.int16, generator=g)
    sec_iq = torch.roll(ref_iq, shifts=(1, 2), dims=(0, 1)) + noise  # offset by ~(1, 2) px
    ati, rps, srt, wl = 2.055556e-3, 2.329562, 5.35e-3, 0.05546576
    est = [DcEstimate(800_000 + int(2.758e6 * k), srt + 1e-6 * (k % 3),
                      [-40.0 + 10.0 * k, 3.0e4 - 7.0e3 * k, -5.0e6 + 1.3e6 * k]) for k in range(6)]
    sw = SubSwathMetadata("IW1", 9, 1500, samples, ati, rps, srt, est)
    ro, so = _insar_orbit(), _insar_orbit((110.0, -60.0, 150.0))
    poly = CoregPoly([1.03, 1e-6, -2e-7, 0.0, 0.0, 0.0], [1.98, 0.0, 3e-6, 0.0, 0.0, 1e-10])
    cfg = InterferogramConfig()

    def chain(r_iq, s_iq, host_out=False):
        rd = sd.deramp_subswath(DeburstArray(r_iq, lines, samples, 0), sw, 0, ctx=ctx)
        sdr = sd.deramp_subswath(DeburstArray(s_iq, lines, samples, 0), sw, 0, ctx=ctx)
        rs = sd.resample_secondary(lines, samples, poly, sdr, ctx=ctx)
        return sd.form_interferogram(Coregistered(rd, rs), sw, ro, 0, so, wl, cfg, ctx=ctx)

    for _ in range(args.warmup):
        chain(ref_iq, sec_iq)
    names = ("k_deramp", "k_coreg_resample", "k_igram", "k_coherence")
    ctx.set_timing(True)
    l0 = ctx.launches
    with ClockSampler(local) as clk:
        for _ in range(args.steps):
            torch.cuda.synchronize()
            if dist is not None:
                dist.barrier()
            ig = chain(ref_iq, sec_iq)
    launches = (ctx.launches - l0) // args.steps
    kt = ctx.kernel_times()
    ctx.set_timing(False)
    n = lines * samples
    dev_ms = _max_over_ranks(dist, sum(kt[k][0] for k in names if k in kt) / args.steps)
    # algorithmic bytes per launch: CInt16 in + complex f32 out; 4 corners in + out; ref + sec in + float4
    # out; the float4 plane in once + coherence out
    alg = {"k_deramp": 12 * n, "k_coreg_resample": 16 * n, "k_igram": 32 * n, "k_coherence": 20 * n}
    per_k = {k: {"ms": round(kt[k][0] / args.steps, 3), "launches": kt[k][1] // args.steps,
                 "gbs": round(alg[k] * (kt[k][1] // args.steps) / (kt[k][0] / args.steps / 1e3) / 1e9, 1)}
             for k in names if k in kt}
    # coherence: 4 sums of (2 az/2 + 1)(2 rg/2 + 1) f64 adds per pixel, the reference's order
    win = (2 * (cfg.az_looks // 2) + 1) * (2 * (cfg.rg_looks // 2) + 1)
    coh_ms = kt["k_coherence"][0] / args.steps
    fp64 = ctypes_fp64_peak(ctx)
    coh_tflops = 4 * win * n / (coh_ms / 1e3) / 1e12
    add_peak = fp64 / 2 if fp64 else None  # an f64 add takes the issue slot of an FMA (2 FLOPs)
    roof = {"bound": "fp64", "kernel": "k_coherence", "achieved": coh_tflops, "peak": add_peak,
            "unit": "T f64 adds/s", "frac": coh_tflops / add_peak if add_peak else None, "traffic": None,
            "adds_per_step": 4 * win * n,
            "peak_source": "measured FP64 FMA chain (sd_measure_fp64_peak) / 2: the f64 add issue rate"}
    mean_coh = float(ig.coherence.float().mean())
    # e2e: pinned host CInt16 in, coherence out to pinned host memory
    e2e = None
    if args.e2e:
        hr = ref_iq.cpu().pin_memory()
        hs = sec_iq.cpu().pin_memory()
        hc = torch.empty((lines, samples), dtype=torch.float32).pin_memory()
        t_e = 0.0
        for i in range(args.steps + 1):
            torch.cuda.synchronize()
            if dist is not None:
                dist.barrier()
            t0 = time.perf_counter()
            r_d = hr.to(dev)  # blocking: the library's calls run on their own stream
            s_d = hs.to(dev)
            out = chain(r_d, s_d)
            hc.copy_(out.coherence, non_blocking=True)
            torch.cuda.synchronize()
            if i:
                t_e += time.perf_counter() - t0
        t_e = _max_over_ranks(dist, t_e / args.steps)
        e2e = {"value": world * n / t_e, "unit": "px/s", "ms_per_step": t_e * 1e3,
               "h2d_bytes_per_step": 8 * n, "d2h_bytes_per_step": 4 * n,
               "api": "sardine_b200.deramp_subswath x2 + resample_secondary + form_interferogram"}
    cpu = None
    if args.cpu_baseline and world == 1 and rank == 0:
        import oracle
        band = 24
        r_np, s_np = ref_iq[:band].cpu().numpy(), sec_iq[:band].cpu().numpy()
        t0 = time.perf_counter()
        _, rd = oracle.deramp_subswath(DeburstArray(r_np, band, samples, 0), sw, 0)
        _, sdr = oracle.deramp_subswath(DeburstArray(s_np, band, samples, 0), sw, 0)
        rs = oracle.resample_secondary(band, samples, poly, sdr)
        oracle.form_interferogram(Coregistered(rd, rs), sw, ro, 0, so, wl, cfg)
        cpu_s = time.perf_counter() - t0
        cpu = {"value": band * samples / cpu_s, "unit": "px/s", "cores": 1, "kind": "port",
               "sample": f"oracle chain on the first {band} lines (coherence at the band's edge rows included)"}
    if rank == 0:
        out = {
            "metric": "interferogram px/s", "value": world * n / (dev_ms / 1e3), "unit": "px/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": dev_ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64 (f32 storage)",
            "data": "synthetic (seeded CInt16 pair, secondary offset by ~(1, 2) px plus noise; inclined "
                    "circular orbits 700 km up with a 200 m baseline)",
            "config": {"workload": f"insar: deramp x2 + resample_secondary + form_interferogram "
                                   f"({cfg.az_looks}x{cfg.rg_looks} coherence) of {lines}x{samples}"
                                   + (" (REDUCED SHAPE)" if args.small else ""),
                       "l2": "inputs larger than L2", "parallelism": f"replicas x{world}"},
            "kernels": per_k, "roofline": roof, "mean_coherence": mean_coh, "cpu_baseline": cpu,
            "gpu_launches": launches, "e2e": e2e, "clocks": clk.summary(),
        }
        print(json.dumps(out), flush=True)
    _finish_dist(dist)


def _hbm_peak():
    """Measured HBM copy bandwidth (GB/s), else the fallback figure (6650 GB/s,
    an earlier STREAM-style copy on this kind of B200)."""
    try:
        return float(json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json"))).get("hbm_gbs", 6650.0))
    except Exception:
        return 6650.0


def _hbm_peak_source():
    return ("measured (MEASURED_PEAKS.json hbm_gbs)" if os.path.exists(os.path.join(ROOT, "MEASURED_PEAKS.json"))
            else "fallback 6650 GB/s (no measured peaks file)")


def run_export(args):
    """The output stage of the reference pipeline (run.rs:394-450):
    to_db_inplace + compute_db_stats, then write_cog_with_crs (512-px tiles)
    of a geocoded raster on the config-2 output grid (25000 x 20000 UTM 10 m),
    resident on the device.  value = output pixels per second of device time
    of the stage's kernels; e2e = the two public calls end to end, file
    written to local disk included."""
    import torch
    import sardine_b200 as sd
    rank, world, local = _rank_env()
    torch.cuda.set_device(local)
    dist = _init_dist(world)
    ctx = sd.Context(local)
    dev = f"cuda:{local}"
    rows, cols = (2000, 12000) if args.small else (20000, 25000)
    n = rows * cols
    g = torch.Generator(device=dev).manual_seed(7 + rank)
    src = torch.empty(n, device=dev).exponential_(20.0, generator=g)  # mean 0.05, as calibrated sigma0
    src[torch.rand(n, device=dev, generator=g) < 0.1] = float("nan")
    src[torch.rand(n, device=dev, generator=g) < 0.05] = 0.0
    work = torch.empty_like(src)
    gt = [500000.0, 10.0, 0.0, 5_200_000.0, 0.0, -10.0]
    crs = sd.OutputCrs.utm_north(32)
    path = f"/tmp/sardine_b200_export_r{rank}.tif"
    ts = 512

    def step():
        c, st = sd.to_db_inplace(work, 0.0, ctx=ctx, stats=True)
        sd.write_cog_with_crs(path, work, cols, rows, gt, crs, ts, ctx=ctx)
        return c, st

    for _ in range(args.warmup):
        work.copy_(src)
        step()
    ctx.set_timing(True)
    wall = 0.0
    with ClockSampler(local) as clk:
        for _ in range(args.steps):
            work.copy_(src)
            torch.cuda.synchronize()
            if dist is not None:
                dist.barrier()
            t0 = time.perf_counter()
            counts, stats = step()
            wall += time.perf_counter() - t0
    kt = ctx.kernel_times()
    ctx.set_timing(False)
    names = ("k_to_db", "k_db_sample", "k_downsample_2x", "k_tile_pack")
    dev_ms = sum(kt[k][0] for k in names if k in kt) / args.steps
    dev_ms = _max_over_ranks(dist, dev_ms)
    wall = _max_over_ranks(dist, wall)
    # algorithmic bytes per step and kernel
    lv, c, r = [], (cols + 1) // 2, (rows + 1) // 2
    while True:
        lv.append((c, r))
        if not (c > ts or r > ts):
            break
        c, r = (c + 1) // 2, (r + 1) // 2
    ds_bytes = 4 * (cols * rows + sum(a * b for a, b in lv[:-1])) + 4 * sum(a * b for a, b in lv)
    tiles = lambda a, b: -(-a // ts) * -(-b // ts)
    pack_bytes = sum(4 * a * b + 4 * tiles(a, b) * ts * ts for a, b in lv + [(cols, rows)])
    alg = {"k_to_db": 8 * n, "k_db_sample": 4 * n, "k_downsample_2x": ds_bytes, "k_tile_pack": pack_bytes}
    per_k = {k: {"ms": round(kt[k][0] / args.steps, 3), "launches": kt[k][1] // args.steps,
                 "gbs": round(alg[k] / (kt[k][0] / args.steps / 1e3) / 1e9, 1)} for k in names if k in kt}
    dom = max(per_k, key=lambda k: per_k[k]["ms"])
    peak = _hbm_peak()
    roof = {"bound": "hbm", "kernel": dom, "achieved": per_k[dom]["gbs"], "peak": peak, "unit": "GB/s",
            "frac": per_k[dom]["gbs"] / peak, "traffic": None,
            "bytes_per_step": alg[dom], "stage_gbs": round(sum(alg.values()) / (dev_ms / 1e3) / 1e9, 1)}
    file_bytes = os.path.getsize(path)
    # the dB conversion fused into the stage that produces the raster (here
    # a Gamma-MAP 5 x 5 filter, as run.rs applies speckle before to_db): the
    # filter then to_db_inplace, against the filter writing dB itself
    flt = sd.SpeckleFilter.GammaMap(5, 4.4)

    def dev_ms_of(fn):
        fn()  # warm
        ctx.set_timing(True)
        fn()
        t = ctx.kernel_times()
        ctx.set_timing(False)
        return {k: round(v[0], 3) for k, v in t.items()}

    def separate():
        filtered = sd.apply_speckle_filter(src, cols, rows, flt, ctx=ctx)
        return sd.to_db_inplace(filtered, 0.0, ctx=ctx, stats=True)

    def fused():
        sd.set_db_output(ctx, True, 0.0)
        try:
            sd.apply_speckle_filter(src, cols, rows, flt, ctx=ctx)
            return sd.db_result(ctx)
        finally:
            sd.set_db_output(ctx, False)
    sep_k = dev_ms_of(separate)
    sep_res = separate()
    fus_k = dev_ms_of(fused)
    fus_res = fused()
    db_fusion = {"what": (f"Gamma-MAP 5x5 of the {rows}x{cols} raster, then to_db_inplace + stats, against the "
                          "filter writing dB itself (statistics from a read-only pass)"),
                 "separate_kernels_ms": sep_k, "fused_kernels_ms": fus_k,
                 "separate_ms": round(sum(sep_k.values()), 3), "fused_ms": round(sum(fus_k.values()), 3),
                 "same_counts_and_stats": bool(sep_res[0] == fus_res[0] and
                                               np.array_equal(np.array(sep_res[1], np.float32).view(np.uint32),
                                                              np.array(fus_res[1], np.float32).view(np.uint32)))}
    cpu = None
    if args.cpu_baseline and world == 1 and rank == 0:
        import oracle
        band = min(rows, 1000)
        sample = src[: band * cols].cpu().numpy().copy()
        t0 = time.perf_counter()
        oracle.to_db_inplace(sample, 0.0)
        oracle.db_stats(sample)
        oracle.write_cog(path + ".cpu", sample, cols, band, gt, crs, ts)
        cpu_s = (time.perf_counter() - t0) * rows / band
        os.remove(path + ".cpu")
        cpu = {"value": n / cpu_s, "unit": "px/s", "cores": 1, "kind": "port",
               "sample": f"oracle to_db + stats + COG writer on {band} of {rows} rows, scaled to all rows"}
    os.remove(path)
    if rank == 0:
        out = {
            "metric": "output px/s", "value": world * n / (dev_ms / 1e3), "unit": "px/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": dev_ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32 (f64 sums)",
            "data": "synthetic (seeded exponential sigma0 with NaN and zero pixels)",
            "config": {"workload": f"export: to_db + dB stats + COG (tile {ts}) of a {rows}x{cols} geocoded raster"
                                   + (" (REDUCED SHAPE)" if args.small else ""),
                       "l2": "inputs larger than L2", "parallelism": f"replicas x{world}"},
            "kernels": per_k, "roofline": roof, "counts": list(counts), "db_stats": list(stats),
            "db_fused_into_speckle": db_fusion,
            "cpu_baseline": cpu, "gpu_launches": sum(v["launches"] for v in per_k.values()),
            "clocks": clk.summary(),
            "e2e": {"value": world * n / (wall / args.steps), "unit": "px/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": file_bytes, "file_bytes": file_bytes,
                    "api": "sardine_b200.to_db_inplace + write_cog_with_crs, file on local disk"},
        }
        print(json.dumps(out), flush=True)
    _finish_dist(dist)


def _init_dist(world):
    if world <= 1:
        return None
    import datetime
    import torch.distributed as dist
    dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    return dist


def _max_over_ranks(dist, ms):
    if dist is None:
        return ms
    import torch
    t = torch.tensor([ms], device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def _sum_over_ranks(dist, x):
    if dist is None:
        return x
    import torch
    t = torch.tensor([float(x)], device="cuda", dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def _finish_dist(dist):
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


def run_reference_tiles(args):
    """Reference arm for config 5: the oracle port geocodes (and filters) a
    bounded sample of the same request stream per step, on the host cores,
    from one config-2-shape scene it prepared itself (deburst, calibration,
    merge on the CPU)."""
    import oracle
    import sardine_b200 as sd
    from sardine_b200 import synth, tiles
    threads = os.cpu_count()
    oracle.set_threads(threads)
    dev = None
    try:
        import torch
        if torch.cuda.is_available():
            dev = "cuda"
    except Exception:
        pass
    sc = synth.config2_scene(seed=200, device=dev)   # synthetic inputs only
    swaths_h = [type(s)(s.id, s.slc.cpu().numpy() if dev else s.slc, s.sw, s.bursts, s.cal, s.noise)
                for s in sc.swaths]
    sc.swaths = None
    inputs = []
    for s in swaths_h:
        deb = oracle.deburst_subswath(s.slc, s.sw, s.bursts)
        sig = oracle.apply_calibration(deb, s.cal, s.noise, s.bursts[0].first_line)
        inputs.append(sd.SwathInput(sig, s.sw, s.bursts[0].azimuth_time_us))
    merged = oracle.merge_subswaths(inputs)[0]
    del inputs, swaths_h
    dem = sd.DemGrid(sc.dem.data.cpu().numpy() if dev else sc.dem.data, sc.dem.origin_y, sc.dem.origin_x,
                     sc.dem.pixel_size, sc.dem.kind, sc.dem.utm_zone, sc.dem.utm_south)
    rc, g = oracle.tc_output_grid(sc.scene, sc.config)
    fake = type("S", (), {})()  # request geometry only; the oracle reads the host scene
    scenes = [{"rs": fake, "cfg": sc.config, "info": g}]
    rng = np.random.default_rng(57)
    # the main arm's CPU-baseline spec: FP64 requests of one scene, smallest
    # first, until the step's share of ~12 s of timed work
    budget = 12.0 / max(1, args.steps)
    per_step, px_all, t_all, n_all = [], 0, 0.0, 0
    for i in range(args.warmup + args.steps):
        reqs = sorted(_c5_requests(sd, scenes, rng, 96, sd.Precision.FP64), key=lambda r: r.rows * r.cols)
        px, t = 0, 0.0
        for r in reqs:
            h = r.halo()
            t0 = time.perf_counter()
            out = oracle.terrain_correction_grid(merged, sc.scene, dem, sc.grids, r.config,
                                                 r.origin_x - h * r.config.pixel_spacing_deg,
                                                 r.origin_y + h * r.config.pixel_spacing_deg,
                                                 r.rows + 2 * h, r.cols + 2 * h)
            if r.speckle is not None:
                oracle.apply_speckle_filter(out.data, r.cols + 2 * h, r.rows + 2 * h, r.speckle)
            t += time.perf_counter() - t0
            px += r.rows * r.cols
            if i >= args.warmup:
                n_all += 1
            if t > budget:
                break
        if i >= args.warmup:
            per_step.append(t)
            px_all += px
            t_all += t
    value = px_all / t_all
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * float(np.mean(per_step)),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded config-2-shape IW scene)", "config": _c5_config(args, 1),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                         "sample": (f"oracle port, {threads} threads: geocode + speckle of one scene's random "
                                    f"tile requests, smallest first, {budget:.2f} s per step ({n_all} requests, "
                                    f"{px_all} px, {t_all:.1f} s timed)")},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "note": "reference (Rust) unbuildable here: no cargo/rustc and crates not vendored; "
                "the C++ oracle port stands in",
    }), flush=True)


def run_reference(args):
    """Reference arm: the reference is Rust and cannot be built here, so the
    oracle port (its C++ restatement) is timed on the host cores, each step a
    bounded sample of the same workload."""
    rank, world, _ = _rank_env()
    if rank != 0:
        return
    if args.config in ("c4", "c5"):
        return run_reference_tiles(args)
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


def run_tile_batch(args):
    """A profiling aid, not a bench number: the config-5 scenes and 64 seeded
    requests of the served arm geocoded as one `tc_tiles` batch (after a
    warm-up batch of 8) in the kernel form `--tile-form` names, twice per group: all tiles, the narrow ones
    (<= 512 columns) and the wide ones (>= 1024).  Prints the per-kernel
    device time of the second pass of each group, in ms and ps per output
    pixel, as one JSON line."""
    import numpy as np
    import torch
    import sardine_b200 as sd
    from sardine_b200 import tiles
    torch.cuda.set_device(0)
    ctx = sd.Context(0)
    if args.tile_form == "tile":  # the per-tile parameter forms the served arm's autotuner picks
        from sardine_b200 import autotune
        autotune.apply(ctx, {"speckle": [32, 8], "main_cps": -1})
    scenes = _c5_setup(sd, ctx, "cuda:0", 0, args.tile_batch)
    reqs = _c5_requests(sd, scenes, np.random.default_rng(5), 64, sd.Precision.SPLIT)
    groups = {"all": reqs, "narrow<=512": [r for r in reqs if r.cols <= 512],
              "wide>=1024": [r for r in reqs if r.cols >= 1024]}
    tiles.tc_tiles(reqs[:8], ctx)
    out = {"tile_batch": {"scenes": args.tile_batch, "requests": len(reqs), "form": args.tile_form}}
    for name, g in groups.items():
        if not g:
            continue
        for _ in range(2):
            ctx.set_timing(True)
            tiles.tc_tiles(g, ctx)
            kt = ctx.kernel_times()
            ctx.set_timing(False)
        px = sum(r.rows * r.cols for r in g)
        out[name] = {"tiles": len(g), "px": px,
                     "ps_per_px": {k: round(v[0] * 1e9 / px, 1)
                                   for k, v in sorted(kt.items(), key=lambda kv: -kv[1][0])},
                     "ms": {k: round(v[0], 3) for k, v in kt.items()}}
    print(json.dumps(out))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="c5", choices=["c5", "c2", "c1", "c3", "c4", "export", "ingest", "insar"])
    ap.add_argument("--rates", default="100,500,2000,max",
                    help="config5 request rates (req/s; 'max' queues every request at once); value at the last")
    ap.add_argument("--burst", type=int, default=512, help="config5 requests per step")
    ap.add_argument("--scenes", type=int, default=8, help="config5 resident scenes")
    ap.add_argument("--budget-gb", dest="budget_gb", type=int, default=16, help="config5 HBM budget")
    ap.add_argument("--max-batch", dest="max_batch", type=int, default=64, help="config5 requests per batch at most")
    ap.add_argument("--slots", type=int, default=2, help="config5 concurrent batches (server slots)")
    ap.add_argument("--no-cpu-baseline", dest="cpu_baseline", action="store_false")
    ap.add_argument("--no-e2e", dest="e2e", action="store_false")
    ap.add_argument("--ref-rows", type=int, default=16)
    ap.add_argument("--small", action="store_true",
                    help="reduced IW shape (profiler captures); not a bench number")
    ap.add_argument("--tile-batch", dest="tile_batch", type=int, default=0, metavar="N_SCENES",
                    help="time one config-5 tile batch over N_SCENES scenes per kernel (profiler captures); "
                         "not a bench number")
    ap.add_argument("--tile-form", dest="tile_form", default="batch", choices=["batch", "tile"],
                    help="--tile-batch: persistent work-table kernels (batch) or the per-tile parameter forms (tile)")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.tile_batch:
        run_tile_batch(args)
    elif args.impl == "reference":
        run_reference(args)
    elif args.config == "c4":
        run_c4(args)
    elif args.config == "c5":
        run_c5(args)
    elif args.config == "export":
        run_export(args)
    elif args.config == "ingest":
        run_ingest(args)
    elif args.config == "insar":
        run_insar(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
