"""TOPS deramping (deramp_subswath, insar/deramp.rs:114-276): the oracle
against the reference's own tests (deramp.rs:336-468) and a numpy
restatement, then the GPU kernel against the oracle."""
import numpy as np
import pytest

import oracle
import sardine_b200 as sd
from sardine_b200 import _abi
from sardine_b200.types import DcEstimate, DeburstArray, SubSwathMetadata

EPOCH_US = 1_548_221_628_000_000  # 2019-01-23T05:33:48Z
ATI = 2.055_556e-3


def _est(t_s, a0, a1=0.0, a2=0.0, t0=5.354e-3):
    """make_dc_estimate (deramp.rs:286-296): microseconds truncated as i64."""
    return DcEstimate(EPOCH_US + int(t_s * 1e6), t0, [a0, a1, a2])


def _swath(est, ati=ATI, rps=2.329_562, srt=5.354e-3):
    """make_subswath (deramp.rs:298-319)."""
    return SubSwathMetadata("IW1", 1, 10, 5, ati, rps, srt, est)


def _deburst(lines, samples, iq=None, off=0):
    if iq is None:
        iq = np.tile(np.array([100, 0], np.int16), (lines, samples, 1))  # make_deburst (321-330)
    return DeburstArray(iq, lines, samples, off)


def _numpy_deramp(db, sw, start_us):
    """A numpy restatement (vectorised over columns)."""
    est = sw.dc_estimates
    et = np.array([(e.azimuth_time_us - start_us) / 1e6 for e in est])
    tau = sw.slant_range_time_s + (np.arange(db.samples) + db.valid_sample_offset) * (
        2.0 * sw.range_pixel_spacing_m / 299_792_458.0)
    iq = np.asarray(db.data, np.float64).reshape(db.lines, db.samples, 2)
    out = np.empty((db.lines, db.samples, 2), np.float32)
    for ln in range(db.lines):
        t = ln * sw.azimuth_time_interval_s
        if t < et[0] or t >= et[-1]:
            e = est[0] if t < et[0] else est[-1]
            q = [*e.data_dc_poly, e.t0_s]
        else:
            k = next(j for j in range(len(et) - 1) if et[j] <= t < et[j + 1])
            a = (t - et[k]) / (et[k + 1] - et[k])
            e0, e1 = est[k], est[k + 1]
            q = [e0.data_dc_poly[j] + (e1.data_dc_poly[j] - e0.data_dc_poly[j]) * a for j in range(3)]
            q.append(e0.t0_s + (e1.t0_s - e0.t0_s) * a)
        dt = tau - q[3]
        phi = 6.283185307179586 * (q[0] + q[1] * dt + q[2] * dt * dt) * t
        s, c = np.sin(phi), np.cos(phi)
        out[ln, :, 0] = (iq[ln, :, 0] * c + iq[ln, :, 1] * s).astype(np.float32)
        out[ln, :, 1] = (iq[ln, :, 1] * c - iq[ln, :, 0] * s).astype(np.float32)
    return out


def _scene(lines, samples, seed, off=37):
    """An IW-like sub-swath: 9 bursts' worth of estimates 2.758 s apart,
    quadratic range dependence, line 0 0.8 s before the first estimate."""
    rng = np.random.default_rng(seed)
    iq = np.clip(np.round(rng.normal(0, 80, (lines, samples, 2))), -32768, 32767).astype(np.int16)
    est = [_est(-0.8 + 2.758 * k + 0.8, rng.uniform(-60, 60), rng.uniform(-4e4, 4e4), rng.uniform(-1e7, 1e7),
                5.354e-3 + rng.uniform(-1e-6, 1e-6)) for k in range(9)]
    return _deburst(lines, samples, iq, off), _swath(est), EPOCH_US - 800_000


# ── oracle vs the reference's deramp tests ──────────────────────────────────
def test_oracle_zero_dc_is_identity():
    # deramp.rs:333-361
    rc, r = oracle.deramp_subswath(_deburst(4, 3), _swath([_est(0.0, 0.0), _est(3.0, 0.0)]), EPOCH_US)
    assert rc == 0 and (r.lines, r.samples) == (4, 3)
    assert np.all(np.abs(r.data[..., 0] - 100.0) < 1e-3) and np.all(np.abs(r.data[..., 1]) < 1e-3)


def test_oracle_empty_estimates():
    # deramp.rs:363-373
    assert oracle.deramp_subswath(_deburst(2, 2), _swath([]), EPOCH_US)[0] == _abi.SD_ERR_INSAR_NO_DC_ESTIMATES


def test_oracle_power_is_conserved():
    # deramp.rs:375-400
    rc, r = oracle.deramp_subswath(_deburst(5, 4), _swath([_est(0.0, 100.0), _est(3.0, 100.0)]), EPOCH_US)
    assert rc == 0
    p = r.data[..., 0] * r.data[..., 0] + r.data[..., 1] * r.data[..., 1]
    assert np.all(np.abs(p - 10000.0) < 0.1)


def test_oracle_temporal_interpolation():
    # deramp.rs:402-422: a0 = 0 Hz at 0 s, 200 Hz at 2 s; observed at t = 1 s as
    # the phase of a line whose azimuth time is 1 s (ATI = 1 s, line 1)
    sw = _swath([_est(0.0, 0.0), _est(2.0, 200.0)], ati=1.0)
    sw.dc_estimates[0].t0_s = sw.dc_estimates[1].t0_s = sw.slant_range_time_s
    rc, r = oracle.deramp_subswath(_deburst(2, 1), sw, EPOCH_US)
    assert rc == 0
    phi = 2 * np.pi * 100.0 * 1.0
    assert np.allclose(r.data[1, 0], [100 * np.cos(phi), -100 * np.sin(phi)], atol=1e-6)


def test_oracle_quarter_cycle_rotation():
    # deramp.rs:424-468
    f = 0.25 / ATI
    rc, r = oracle.deramp_subswath(_deburst(2, 1), _swath([_est(0.0, f), _est(3.0, f)]), EPOCH_US)
    assert rc == 0
    assert abs(r.data[0, 0, 0] - 100) < 0.1 and abs(r.data[0, 0, 1]) < 0.1
    assert abs(r.data[1, 0, 0]) < 0.5 and abs(r.data[1, 0, 1] + 100) < 0.5


def test_oracle_before_first_estimate():
    # interp_dc_poly (deramp.rs:233-246): up to 2 s before the first estimate uses it, beyond is an error
    db = _deburst(3, 2)
    rc, r = oracle.deramp_subswath(db, _swath([_est(1.9, 50.0), _est(4.0, 50.0)]), EPOCH_US)
    assert rc == 0
    rc, t = oracle.deramp_subswath(db, _swath([_est(2.5, 50.0), _est(4.0, 50.0)]), EPOCH_US)
    assert rc == _abi.SD_ERR_INSAR_AZIMUTH_TIME_BEFORE_DC and t == 0.0


def test_oracle_equals_numpy_restatement():
    db, sw, t0 = _scene(60, 70, 3)
    sw.azimuth_time_interval_s = 0.4  # 60 lines span all nine estimates and beyond
    rc, r = oracle.deramp_subswath(db, sw, t0)
    assert rc == 0
    want = _numpy_deramp(db, sw, t0)
    d = np.abs(r.data.astype(np.float64) - want)
    # numpy's and the C library's sin/cos may differ in the last bit of f64
    assert np.mean(r.data == want) > 0.99
    assert np.all(d <= 2 * np.spacing(np.abs(want).astype(np.float32)) + 1e-30)


# ── GPU vs oracle ────────────────────────────────────────────────────────────
def _close(got, want):
    """Bit-equal except where CUDA's and the C library's FP64 sincos differ in
    the last bit and that difference survives the f32 rounding: then within 2
    f32 spacings of |I| + |Q| (the complex product's magnitude bound)."""
    got = np.asarray(got, np.float32)
    mag = (np.abs(want[..., 0]) + np.abs(want[..., 1]))[..., None]
    tol = 2 * np.spacing(mag.astype(np.float32))
    assert np.all(np.abs(got.astype(np.float64) - want) <= tol)
    assert np.mean(got == want) >= 0.99


@pytest.mark.gpu
@pytest.mark.parametrize("lines,samples,ati", [(4, 3, ATI), (1498, 2400, ATI), (3001, 777, 0.01)])
def test_gpu_deramp_matches_oracle(ctx, lines, samples, ati):
    import torch
    db, sw, t0 = _scene(lines, samples, lines)
    sw.azimuth_time_interval_s = ati
    rc, want = oracle.deramp_subswath(db, sw, t0)
    assert rc == 0
    for kind in ("host", "device"):
        src = db if kind == "host" else DeburstArray(torch.from_numpy(db.data).cuda(), lines, samples,
                                                     db.valid_sample_offset)
        got = sd.deramp_subswath(src, sw, t0, ctx=ctx)
        assert (got.lines, got.samples, got.valid_sample_offset) == (lines, samples, db.valid_sample_offset)
        gd = got.data if kind == "host" else got.data.cpu().numpy()
        _close(gd, want.data)


@pytest.mark.gpu
def test_gpu_deramp_reference_cases(ctx):
    f = 0.25 / ATI
    r = sd.deramp_subswath(_deburst(2, 1), _swath([_est(0.0, f), _est(3.0, f)]), EPOCH_US, ctx=ctx)
    assert abs(r.data[1, 0, 0]) < 0.5 and abs(r.data[1, 0, 1] + 100) < 0.5
    r = sd.deramp_subswath(_deburst(4, 3), _swath([_est(0.0, 0.0), _est(3.0, 0.0)]), EPOCH_US, ctx=ctx)
    assert np.all(r.data[..., 0] == 100.0) and np.all(r.data[..., 1] == 0.0)


@pytest.mark.gpu
def test_gpu_deramp_errors(ctx):
    with pytest.raises(sd.InsarError) as e:
        sd.deramp_subswath(_deburst(2, 2), _swath([]), EPOCH_US, ctx=ctx)
    assert e.value.kind == "NoDcEstimates"
    with pytest.raises(sd.InsarError) as e:
        sd.deramp_subswath(_deburst(3, 2), _swath([_est(2.5, 50.0), _est(4.0, 50.0)]), EPOCH_US, ctx=ctx)
    assert e.value.kind == "AzimuthTimeBeforeDcEstimates"
