"""sd_apply_calibration_noalloc: calibration for callers that cannot allocate
device memory while they run.

The entry point is called through the C ABI with device buffers the test
owns; each of two consecutive calls (different rasters, LUTs and line
origins) must reproduce sd_apply_calibration bit for bit (the tolerance the
calibration tests use), and the second call must not change the device's
free memory.  This file sorts last so a stop-at-first-failure run has already
run every other test.
"""
import ctypes as C

import numpy as np
import pytest

import sardine_b200 as sd
from sardine_b200 import _lib, synth
from sardine_b200 import types as T

pytestmark = pytest.mark.gpu


def _call_noalloc(iq, deb, cal, noise, origin, out, nesz, stream=None):
    keep = T._Keep()
    cv = T.lut_vectors_to_c(cal.vectors, keep, "sigma_nought")
    nv = T.lut_vectors_to_c(noise.range_vectors, keep, "noise_range_lut")
    na = T.noise_azimuth_to_c(noise, keep)
    cg, ng = C.c_uint32(), C.c_uint32()
    err = C.create_string_buffer(512)
    rc = _lib.lib().sd_apply_calibration_noalloc(
        stream, iq.data_ptr(), deb.lines, deb.samples, deb.valid_sample_offset, cv,
        len(cal.vectors), nv, len(noise.range_vectors), C.byref(na), origin, out.data_ptr(),
        nesz.data_ptr(), C.byref(cg), C.byref(ng), err, len(err))
    return rc, err.value.decode(), cg.value, ng.value


def _case(seed):
    sc = synth.config2_scene(seed=seed, n_bursts=3, lines_per_burst=400, tiff_width=1800,
                             burst_step=300, swath_overlap=100, out_rows=32, out_cols=32,
                             lut_lines_step=140)
    return sc.swaths[seed % 3]


def test_noalloc_matches_apply_calibration_twice():
    import torch
    torch.cuda.init()
    ctx = sd.Context(0)
    dev = torch.device("cuda", 0)
    free_after = []
    for call, seed in enumerate((41, 42)):
        sw = _case(seed)
        deb = sd.deburst_subswath(torch.from_numpy(np.asarray(sw.slc)).to(dev), sw.sw, sw.bursts, ctx=ctx)
        origin = sw.bursts[0].first_line + 7 * call
        want = sd.apply_calibration(deb, sw.cal, sw.noise, origin, ctx=ctx)
        torch.cuda.synchronize()
        out = torch.full((deb.lines, deb.samples), float("nan"), device=dev)
        nesz = torch.full((deb.lines, deb.samples), float("nan"), device=dev)
        torch.cuda.synchronize()
        free_before = torch.cuda.mem_get_info(0)[0]
        rc, msg, cg, ng = _call_noalloc(deb.data, deb, sw.cal, sw.noise, origin, out, nesz)
        torch.cuda.synchronize()
        free_after.append((free_before, torch.cuda.mem_get_info(0)[0]))
        assert rc == 0, msg
        assert (cg, ng) == (want.cal_lut_extrapolation_gap_px, want.noise_lut_extrapolation_gap_px)
        assert torch.equal(out, want.data), f"call {call}: sigma0 differs"
        assert torch.equal(nesz, want.nesz), f"call {call}: NESZ differs"
    # the second call finds its working memory already in place
    assert free_after[1][1] == free_after[1][0]
    ctx.close()


def test_noalloc_rejects_oversize_and_host_buffers():
    import torch
    dev = torch.device("cuda", 0)
    sw = _case(43)
    deb = sd.DeburstArray(torch.zeros((4, 40000, 2), dtype=torch.int16, device=dev), 4, 40000, 0)
    out = torch.empty((4, 40000), device=dev)
    nesz = torch.empty((4, 40000), device=dev)
    rc, msg, _, _ = _call_noalloc(deb.data, deb, sw.cal, sw.noise, 0, out, nesz)
    assert rc == sd._abi.SD_ERR_INVALID_ARGUMENT and "32768" in msg
    host = sd.DeburstArray(torch.zeros((4, 100, 2), dtype=torch.int16), 4, 100, 0)
    out_h = torch.empty((4, 100))
    rc, msg, _, _ = _call_noalloc(host.data, host, sw.cal, sw.noise, 0, out_h, out_h.clone())
    assert rc == sd._abi.SD_ERR_INVALID_ARGUMENT and "device" in msg


def test_noalloc_refuses_capture_and_null_luts():
    """Its LUT tables are staged from host memory that lives only for the
    call, so a capturing stream is refused before any work is enqueued; a
    null LUT array with a non-zero count is an argument error, not a crash."""
    import torch
    dev = torch.device("cuda", 0)
    ctx = sd.Context(0)
    sw = _case(44)
    deb = sd.deburst_subswath(torch.from_numpy(np.asarray(sw.slc)).to(dev), sw.sw, sw.bursts, ctx=ctx)
    out = torch.empty((deb.lines, deb.samples), device=dev)
    nesz = torch.empty_like(out)
    torch.cuda.synchronize()
    err = C.create_string_buffer(512)
    cg, ng = C.c_uint32(), C.c_uint32()
    rc = _lib.lib().sd_apply_calibration_noalloc(
        None, deb.data.data_ptr(), deb.lines, deb.samples, deb.valid_sample_offset, None, 3, None, 2,
        None, 0, out.data_ptr(), nesz.data_ptr(), C.byref(cg), C.byref(ng), err, len(err))
    assert rc == sd._abi.SD_ERR_INVALID_ARGUMENT and b"null" in err.value
    side = torch.cuda.Stream()
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph, stream=side):
        rc, msg, _, _ = _call_noalloc(deb.data, deb, sw.cal, sw.noise, sw.bursts[0].first_line, out, nesz,
                                      stream=C.c_void_p(side.cuda_stream))
    assert rc == sd._abi.SD_ERR_INVALID_ARGUMENT and "capturing" in msg
    del graph
    # the stream works as before once the capture has ended
    rc, msg, _, _ = _call_noalloc(deb.data, deb, sw.cal, sw.noise, sw.bursts[0].first_line, out, nesz)
    torch.cuda.synchronize()
    assert rc == 0, msg
    want = sd.apply_calibration(deb, sw.cal, sw.noise, sw.bursts[0].first_line, ctx=ctx)
    assert torch.equal(out, want.data) and torch.equal(nesz, want.nesz)
    ctx.close()
