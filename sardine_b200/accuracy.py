"""Per-output error of one geocoded result against another (host-side).

Used to state the split-precision path's error against the FP64 path or the
oracle: geolocation in azimuth pixels (from the converged zero-Doppler times;
both sides share the target ECEF, so equal times mean equal slant range),
sigma0/gamma0 as relative and dB error, cos(LIA) as absolute error, and mask
equality.
"""
from __future__ import annotations

import numpy as np

NO_TIME = np.iinfo(np.int64).min


def _np(a):
    if a is None:
        return None
    if hasattr(a, "detach"):
        return a.detach().cpu().numpy()
    return np.asarray(a)


def compare_geocoded(test, ref, t_test=None, t_ref=None, ati_s: float = 1.0) -> dict:
    """Error of `test` against `ref` (both GeocodedImage-like with data,
    cos_lia, mask).  `t_test`/`t_ref`: per-pixel converged times in us.
    CUDA tensors are compared on the device."""
    if hasattr(test.data, "is_cuda") and test.data.is_cuda:
        return _compare_torch(test, ref, t_test, t_ref, ati_s)
    a = _np(test.data).astype(np.float64)
    b = _np(ref.data).astype(np.float64)
    rep: dict = {}
    fa, fb = np.isfinite(a), np.isfinite(b)
    rep["nan_pattern_equal"] = bool(np.array_equal(fa, fb))
    both = fa & fb
    rep["compared_px"] = int(both.sum())
    if both.any():
        x, y = a[both], b[both]
        rel = np.abs(x - y) / np.maximum(np.abs(y), 1e-30)
        pos = (x > 0) & (y > 0)
        db = np.abs(10.0 * np.log10(x[pos] / y[pos])) if pos.any() else np.zeros(1)
        rep["sigma_rel_err_max"] = float(rel.max())
        rep["sigma_rel_over_1e-4_px"] = int((rel > 1e-4).sum())
        # relative to max(|ref|, floor): a value interpolated to nearly zero
        # between non-zero samples is ill-conditioned (any sub-ulp change of
        # the image coordinates moves it by more than 1e-4 of itself); the
        # floor, 1 % of the median |ref|, is a noise-floor-level magnitude
        pos_b = np.abs(y[y != 0])
        floor = 0.01 * float(np.median(pos_b)) if pos_b.size else 0.0
        rep["sigma_floor"] = floor
        rep["sigma_floor_over_1e-4_px"] = int((np.abs(x - y) > 1e-4 * np.maximum(np.abs(y), floor)).sum())
        rep["sigma_rel_err_p99"] = float(np.quantile(rel, 0.99))
        rep["sigma_rel_err_mean"] = float(rel.mean())
        rep["sigma_db_err_max"] = float(db.max())
        rep["sigma_db_err_p99"] = float(np.quantile(db, 0.99))
        rep["sigma_db_err_mean"] = float(db.mean())
    else:
        for k in ("sigma_rel_err_max", "sigma_rel_err_p99", "sigma_rel_err_mean",
                  "sigma_db_err_max", "sigma_db_err_p99", "sigma_db_err_mean"):
            rep[k] = 0.0
        rep["sigma_rel_over_1e-4_px"] = 0
        rep["sigma_floor_over_1e-4_px"] = 0
        rep["sigma_floor"] = 0.0
    if test.mask is not None and ref.mask is not None:
        rep["mask_equal"] = bool(np.array_equal(_np(test.mask), _np(ref.mask)))
        ca = _np(test.cos_lia).astype(np.float64)
        cb = _np(ref.cos_lia).astype(np.float64)
        cboth = np.isfinite(ca) & np.isfinite(cb)
        rep["cos_lia_nan_equal"] = bool(np.array_equal(np.isfinite(ca), np.isfinite(cb)))
        rep["cos_lia_abs_err_max"] = float(np.abs(ca[cboth] - cb[cboth]).max()) if cboth.any() else 0.0
    if t_test is not None and t_ref is not None:
        ta, tb = _np(t_test), _np(t_ref)
        ha, hb = ta != NO_TIME, tb != NO_TIME
        tboth = ha & hb
        d = np.abs(ta[tboth] - tb[tboth]).astype(np.float64) * 1e-6 / ati_s
        rep["time_mismatch_px"] = int((ha != hb).sum() + (ta[tboth] != tb[tboth]).sum())
        rep["geoloc_err_px_max"] = float(d.max()) if d.size else 0.0
        rep["geoloc_err_px_mean"] = float(d.mean()) if d.size else 0.0
    return rep


def _compare_torch(test, ref, t_test, t_ref, ati_s):
    import torch
    rep: dict = {}
    a = test.data.double()
    b = ref.data.double()
    fa, fb = torch.isfinite(a), torch.isfinite(b)
    rep["nan_pattern_equal"] = bool(torch.equal(fa, fb))
    both = fa & fb
    rep["compared_px"] = int(both.sum())
    x, y = a[both], b[both]
    del a, b
    rel = (x - y).abs() / y.abs().clamp_min(1e-30)
    rep["sigma_rel_err_max"] = float(rel.max()) if rel.numel() else 0.0
    rep["sigma_rel_over_1e-4_px"] = int((rel > 1e-4).sum())
    nz = y.abs()[y != 0]
    floor = 0.01 * float(nz[torch.randint(0, max(1, nz.numel()), (min(nz.numel(), 1 << 22),),
                                          device=nz.device)].median()) if nz.numel() else 0.0
    rep["sigma_floor"] = floor
    rep["sigma_floor_over_1e-4_px"] = int(((x - y).abs() > 1e-4 * y.abs().clamp_min(floor)).sum())
    rep["sigma_rel_err_mean"] = float(rel.mean()) if rel.numel() else 0.0
    g = torch.Generator(device=rel.device).manual_seed(0)
    sub = rel[torch.randint(0, max(1, rel.numel()), (min(rel.numel(), 1 << 22),), device=rel.device,
                            generator=g)] if rel.numel() else rel
    rep["sigma_rel_err_p99"] = float(torch.quantile(sub, 0.99)) if sub.numel() else 0.0
    pos = (x > 0) & (y > 0)
    db = (10.0 * torch.log10(x[pos] / y[pos])).abs()
    rep["sigma_db_err_max"] = float(db.max()) if db.numel() else 0.0
    rep["sigma_db_err_mean"] = float(db.mean()) if db.numel() else 0.0
    del x, y, rel, db
    if test.mask is not None and ref.mask is not None:
        rep["mask_equal"] = bool(torch.equal(test.mask, ref.mask))
        ca, cb = test.cos_lia.double(), ref.cos_lia.double()
        cboth = torch.isfinite(ca) & torch.isfinite(cb)
        rep["cos_lia_nan_equal"] = bool(torch.equal(torch.isfinite(ca), torch.isfinite(cb)))
        rep["cos_lia_abs_err_max"] = float((ca[cboth] - cb[cboth]).abs().max()) if bool(cboth.any()) else 0.0
        del ca, cb, cboth
    if t_test is not None and t_ref is not None:
        ha, hb = t_test != NO_TIME, t_ref != NO_TIME
        tboth = ha & hb
        d = (t_test[tboth] - t_ref[tboth]).abs().double() * 1e-6 / ati_s
        rep["time_mismatch_px"] = int((ha != hb).sum()) + int((d != 0).sum())
        rep["geoloc_err_px_max"] = float(d.max()) if d.numel() else 0.0
        rep["geoloc_err_px_mean"] = float(d.mean()) if d.numel() else 0.0
    return rep
