"""Seeded synthetic Sentinel-1 IW scenes.

No real Sentinel-1 data, orbit files or DEM tiles exist in this environment,
so every workload is synthesised from seeds with the shapes, sizes and value
distributions of the benchmark configurations:

* orbit: circular, a = 7 071 km, i = 98.18 deg, seeded ascending node, 17
  ECEF state vectors 10 s apart (integer-microsecond times);
* radar geometry: near slant range 800 km, range spacing 2.329562 m,
  azimuth time interval 2.055556e-3 s, right-looking;
* sigma0 images: i.i.d. exponential (mean 0.05); SLC bursts: circular complex
  Gaussian (sigma = 60 DN) rounded and clipped to int16;
* calibration LUTs: knots every 40 samples and ~1 s, values 700 +/- 30;
  noise LUTs 0-400 DN^2;
* DEM: fractional-Brownian surface (H = 0.8) by spectral synthesis;
  geoid: smooth seeded field in [-30, 30] m on the 73 x 144 2.5-degree grid;
* geolocation grid: 10 x 21 points from forward zero-Doppler geocoding at
  h = 0.

Array sizes are parameters so the same scenes exist at test size and at full
benchmark size.  Large arrays can be generated with torch on a CUDA device
(``device="cuda"``); the generator is not on any timed path.
"""
from __future__ import annotations

import math
from dataclasses import dataclass
from typing import Any, List, Optional, Tuple

import numpy as np

from . import _abi
from . import types as T

MU = 3.986004418e14
OMEGA_E = 7.2921150e-5
C_LIGHT = 299792458.0
WGS84_A = 6378137.0
WGS84_F = 1.0 / 298.257223563
WGS84_E2 = 2.0 * WGS84_F - WGS84_F * WGS84_F
WGS84_B = WGS84_A * (1.0 - WGS84_F)

ATI = 2.055556e-3
RPS = 2.329562
NEAR_RANGE = 800e3
WAVELENGTH = 0.05547
EPOCH_US = 1_548_221_628_000_000  # 2019-01-23T05:33:48Z, an arbitrary epoch


# ── orbit ──────────────────────────────────────────────────────────────────
@dataclass
class CircularOrbit:
    a: float
    inc: float
    raan: float
    u0: float        # argument of latitude at t_ref
    theta0: float    # Earth rotation angle at t_ref
    t_ref_us: int

    def state(self, t_us):
        """Analytic ECEF position/velocity (arrays broadcast over t)."""
        t = (np.asarray(t_us, dtype=np.float64) - self.t_ref_us) / 1e6
        n = math.sqrt(MU / self.a ** 3)
        u = self.u0 + n * t
        cO, sO, ci, si = math.cos(self.raan), math.sin(self.raan), math.cos(self.inc), math.sin(self.inc)
        cu, su = np.cos(u), np.sin(u)
        r = self.a * np.stack([cO * cu - sO * su * ci, sO * cu + cO * su * ci, su * si], -1)
        v = self.a * n * np.stack([-cO * su - sO * cu * ci, -sO * su + cO * cu * ci, cu * si], -1)
        th = self.theta0 + OMEGA_E * t
        c, s = np.cos(th), np.sin(th)
        re = np.stack([c * r[..., 0] + s * r[..., 1], -s * r[..., 0] + c * r[..., 1], r[..., 2]], -1)
        vr = np.stack([c * v[..., 0] + s * v[..., 1], -s * v[..., 0] + c * v[..., 1], v[..., 2]], -1)
        # V_ecef = R v_eci - omega x r_ecef
        ve = vr - np.stack([-OMEGA_E * re[..., 1], OMEGA_E * re[..., 0], np.zeros_like(re[..., 2])], -1)
        return re, ve


def make_orbit(rng: np.random.Generator, t_center_us: int, center_lat_deg: float = 46.0,
               n_sv: int = 17, spacing_s: float = 10.0) -> Tuple[T.OrbitData, CircularOrbit]:
    inc = math.radians(98.18)
    raan = rng.uniform(0.0, 2.0 * math.pi)
    # ascending pass through center_lat at t_center
    u_c = math.asin(math.sin(math.radians(center_lat_deg)) / math.sin(inc))
    orb = CircularOrbit(7_071_000.0, inc, raan, u_c, rng.uniform(0, 2 * math.pi), t_center_us)
    half = (n_sv - 1) // 2
    times = np.array([t_center_us + int(round((k - half) * spacing_s * 1e6)) for k in range(n_sv)],
                     dtype=np.int64)
    pos, vel = orb.state(times)
    return T.OrbitData(times, np.ascontiguousarray(pos), np.ascontiguousarray(vel)), orb


def ecef_to_geodetic(p):
    """Bowring's method (same scheme as geodesy.rs:63-94), vectorised."""
    x, y, z = p[..., 0], p[..., 1], p[..., 2]
    lon = np.arctan2(y, x)
    pp = np.hypot(x, y)
    ep2 = WGS84_E2 / (1.0 - WGS84_E2)
    th = np.arctan2(z * WGS84_A, pp * WGS84_B)
    lat = np.arctan2(z + ep2 * WGS84_B * np.sin(th) ** 3, pp - WGS84_E2 * WGS84_A * np.cos(th) ** 3)
    for _ in range(5):
        s = np.sin(lat)
        n = WGS84_A / np.sqrt(1.0 - WGS84_E2 * s * s)
        lat = np.arctan2(z + WGS84_E2 * n * s, pp)
    return np.degrees(lat), np.degrees(lon)


def forward_geocode(S, V, R, h=0.0):
    """Ground point at slant range R in the zero-Doppler plane of (S, V),
    right-looking, on the ellipsoid raised by h."""
    S = np.asarray(S, np.float64)
    V = np.asarray(V, np.float64)
    up = S / np.linalg.norm(S, axis=-1, keepdims=True)
    vh = V / np.linalg.norm(V, axis=-1, keepdims=True)
    down = -(up - np.sum(up * vh, -1, keepdims=True) * vh)
    down /= np.linalg.norm(down, axis=-1, keepdims=True)
    right = np.cross(vh, up)
    right -= np.sum(right * vh, -1, keepdims=True) * vh
    right /= np.linalg.norm(right, axis=-1, keepdims=True)
    a2, b2 = (WGS84_A + h) ** 2, (WGS84_B + h) ** 2

    def g(phi):
        d = np.cos(phi)[..., None] * down + np.sin(phi)[..., None] * right
        P = S + np.asarray(R)[..., None] * d
        return (P[..., 0] ** 2 + P[..., 1] ** 2) / a2 + P[..., 2] ** 2 / b2 - 1.0, P

    lo = np.zeros(np.broadcast(S[..., 0], np.asarray(R)).shape)
    hi = np.full_like(lo, 1.4)
    for _ in range(80):  # bisection: g(lo) < 0 (inside), g(hi) > 0
        mid = 0.5 * (lo + hi)
        gm, _ = g(mid)
        inside = gm < 0
        lo = np.where(inside, mid, lo)
        hi = np.where(inside, hi, mid)
    _, P = g(0.5 * (lo + hi))
    return P


# ── rasters ────────────────────────────────────────────────────────────────
def fbm_surface(rng: np.random.Generator, h: int, w: int, hurst: float = 0.8,
                hmax: float = 1500.0, device: Optional[str] = None):
    """Fractional-Brownian surface by spectral synthesis, scaled to [0, hmax]."""
    if device is not None and device != "cpu":
        import torch
        g = torch.Generator(device=device)
        g.manual_seed(int(rng.integers(0, 2**62)))
        fy = torch.fft.fftfreq(h, device=device).view(-1, 1)
        fx = torch.fft.rfftfreq(w, device=device).view(1, -1)
        f = torch.sqrt(fx * fx + fy * fy)
        f[0, 0] = 1.0
        amp = f ** (-(hurst + 1.0))
        amp[0, 0] = 0.0
        ph = torch.rand(f.shape, generator=g, device=device) * (2 * math.pi)
        spec = torch.polar(amp, ph)
        z = torch.fft.irfft2(spec, s=(h, w))
        z = (z - z.min()) / (z.max() - z.min()) * hmax
        return z.float().contiguous()
    fy = np.fft.fftfreq(h).reshape(-1, 1)
    fx = np.fft.rfftfreq(w).reshape(1, -1)
    f = np.sqrt(fx * fx + fy * fy)
    f[0, 0] = 1.0
    amp = f ** (-(hurst + 1.0))
    amp[0, 0] = 0.0
    ph = rng.uniform(0, 2 * math.pi, size=f.shape)
    z = np.fft.irfft2(amp * np.exp(1j * ph), s=(h, w))
    z = (z - z.min()) / (z.max() - z.min()) * hmax
    return np.ascontiguousarray(z, dtype=np.float32)


def geoid_grid(rng: np.random.Generator, amp: float = 30.0) -> np.ndarray:
    """Smooth seeded undulation field on the 73 x 144 EGM96 layout."""
    lat = np.radians(90.0 - 2.5 * np.arange(73)).reshape(-1, 1)
    lon = np.radians(2.5 * np.arange(144)).reshape(1, -1)
    z = np.zeros((73, 144))
    for l in range(1, 5):
        for m in range(0, l + 1):
            a, b = rng.normal(size=2)
            z += (np.cos(lat) ** m) * np.sin(lat) ** (l - m) * (a * np.cos(m * lon) + b * np.sin(m * lon))
    z = z / np.abs(z).max() * amp
    return np.ascontiguousarray(z, dtype=np.float32)


def exponential_image(rng: np.random.Generator, lines: int, samples: int, mean: float = 0.05,
                      device: Optional[str] = None):
    if device is not None and device != "cpu":
        import torch
        g = torch.Generator(device=device)
        g.manual_seed(int(rng.integers(0, 2**62)))
        u = torch.rand((lines, samples), generator=g, device=device, dtype=torch.float32)
        return (-mean * torch.log1p(-u)).contiguous()
    return np.ascontiguousarray(rng.exponential(mean, size=(lines, samples)).astype(np.float32))


def slc_raster(rng: np.random.Generator, lines: int, samples: int, sigma: float = 60.0,
               device: Optional[str] = None):
    if device is not None and device != "cpu":
        import torch
        g = torch.Generator(device=device)
        g.manual_seed(int(rng.integers(0, 2**62)))
        x = torch.randn((lines, samples, 2), generator=g, device=device) * sigma
        return torch.clamp(torch.round(x), -32768, 32767).to(torch.int16).contiguous()
    x = rng.normal(0.0, sigma, size=(lines, samples, 2))
    return np.ascontiguousarray(np.clip(np.round(x), -32768, 32767).astype(np.int16))


# ── numpy UTM (generator-side only: places grids and bounding boxes) ───────
def utm_forward_np(lon_deg, lat_deg, zone: int, south: bool = False):
    """Transverse Mercator, Krueger series to n^3 (sub-millimetre)."""
    n = WGS84_F / (2 - WGS84_F)
    A = WGS84_A / (1 + n) * (1 + n * n / 4 + n ** 4 / 64)
    al = [0, n / 2 - 2 * n * n / 3 + 5 * n ** 3 / 16, 13 * n * n / 48 - 3 * n ** 3 / 5, 61 * n ** 3 / 240]
    e = math.sqrt(WGS84_F * (2 - WGS84_F))
    lam = np.radians(np.asarray(lon_deg, np.float64)) - math.radians((zone - 1) * 6 - 180 + 3)
    phi = np.radians(np.asarray(lat_deg, np.float64))
    tau = np.tan(phi)
    sig = np.sinh(e * np.arctanh(e * tau / np.hypot(1, tau)))
    taup = tau * np.hypot(1, sig) - sig * np.hypot(1, tau)
    xip = np.arctan2(taup, np.cos(lam))
    etap = np.arcsinh(np.sin(lam) / np.hypot(taup, np.cos(lam)))
    xi, eta = xip.copy(), etap.copy()
    for j in (1, 2, 3):
        xi = xi + al[j] * np.sin(2 * j * xip) * np.cosh(2 * j * etap)
        eta = eta + al[j] * np.cos(2 * j * xip) * np.sinh(2 * j * etap)
    return 500000.0 + 0.9996 * A * eta, (1e7 if south else 0.0) + 0.9996 * A * xi


# ── scenes ─────────────────────────────────────────────────────────────────
@dataclass
class TcScene:
    """Inputs of one terrain_correction call."""
    merged: T.MergedSigma0
    scene: T.SceneMetadata
    dem: T.DemGrid
    grids: List[Tuple[str, List[T.GeolocationGridPoint]]]
    config: T.TerrainCorrectionConfig
    orbit_model: CircularOrbit


def _geo_grid(orb: CircularOrbit, az0_us: int, n_lines: int, near_range: float, n_samples: int,
              n_az: int = 10, n_rg: int = 21) -> List[T.GeolocationGridPoint]:
    pts = []
    for i in range(n_az):
        t = az0_us + int(round(i * (n_lines - 1) / (n_az - 1) * ATI * 1e6))
        S, V = orb.state(t)
        for j in range(n_rg):
            R = near_range + j * (n_samples - 1) / (n_rg - 1) * RPS
            P = forward_geocode(S, V, R)
            lat, lon = ecef_to_geodetic(P)
            pts.append(T.GeolocationGridPoint(t, float(lat), float(lon), 2 * R / C_LIGHT))
    return pts


def config1_scene(seed: int = 1, n_lines: int = 4096, n_samples: int = 8192, dem_n: int = 1024,
                  resampling=T.ResamplingKernel.Bilinear, flatten: bool = False,
                  compute_lia: bool = True, device: Optional[str] = None,
                  center_lat_deg: float = 46.0, geoid_zero: bool = False) -> TcScene:
    """Plain terrain correction: exponential sigma0 image in radar geometry,
    EPSG:4326 DEM at 1 arcsec, geoid +/-30 m, bilinear, compute_lia."""
    rng = np.random.default_rng(seed)
    t_center = EPOCH_US + int(rng.integers(0, 10**6)) * 1000
    orbit, orb = make_orbit(rng, t_center, center_lat_deg)
    az0 = t_center - int(round(n_lines / 2 * ATI * 1e6))
    S, V = orb.state(t_center)
    P = forward_geocode(S, V, NEAR_RANGE + n_samples / 2 * RPS)
    lat_c, lon_c = (float(x) for x in ecef_to_geodetic(P))
    sp = 1.0 / 3600.0
    k_n = math.floor(lat_c / sp) + dem_n // 2
    k_w = math.floor(lon_c / sp) - dem_n // 2
    bb = T.BoundingBox((k_n - dem_n + 0.25) * sp, (k_n - 0.25) * sp, (k_w + 0.25) * sp,
                       (k_w + dem_n - 0.25) * sp)
    lat_north = math.ceil(bb.max_lat_deg / sp) * sp
    lon_west = math.floor(bb.min_lon_deg / sp) * sp
    dem = T.DemGrid(fbm_surface(rng, dem_n, dem_n, 0.8, 1500.0, device), lat_north - 0.5 * sp,
                    lon_west + 0.5 * sp, sp, _abi.DEM_GEOGRAPHIC)
    geoid = T.GeoidModel.zero() if geoid_zero else T.GeoidModel(geoid_grid(rng))
    img = exponential_image(rng, n_lines, n_samples, 0.05, device)
    merged = T.MergedSigma0(img, n_lines, n_samples, 2 * NEAR_RANGE / C_LIGHT, 2 * RPS / C_LIGHT,
                            RPS, 0, 0, None, az0)
    sw = T.SubSwathMetadata("IW2", 1, n_lines, n_samples, ATI, RPS, 2 * NEAR_RANGE / C_LIGHT)
    scene = T.SceneMetadata([sw], [], orbit, bb)
    grids = [("IW2", _geo_grid(orb, az0, n_lines, NEAR_RANGE, n_samples))]
    cfg = T.TerrainCorrectionConfig(geoid=geoid, pixel_spacing_deg=sp, flatten=flatten,
                                    compute_lia=compute_lia, resampling=resampling)
    return TcScene(merged, scene, dem, grids, cfg, orb)


@dataclass
class IwSwath:
    id: str
    slc: Any                       # (tiff_height, tiff_width, 2) int16
    sw: T.SubSwathMetadata
    bursts: List[T.BurstEntry]
    cal: T.SwathCalibration
    noise: T.SwathNoise


@dataclass
class IwScene:
    """Inputs of the full IW pipeline: three swaths of bursts + TC inputs."""
    swaths: List[IwSwath]
    scene: T.SceneMetadata
    dem: T.DemGrid
    grids: List[Tuple[str, List[T.GeolocationGridPoint]]]
    config: T.TerrainCorrectionConfig
    orbit_model: CircularOrbit


def _luts(rng, sid: str, tiff_height: int, tiff_width: int, lines_step: int, px_step: int = 40):
    lines = list(range(0, tiff_height + lines_step, lines_step))
    pixels = np.arange(0, tiff_width + px_step - 1, px_step, dtype=np.uint32)
    pixels[-1] = min(pixels[-1], tiff_width - 1)
    ph = rng.uniform(0, 2 * math.pi, 3)
    cal, nr = [], []
    for li in lines:
        x = pixels / float(tiff_width)
        k = 700.0 + 30.0 * np.sin(2 * math.pi * x + ph[0] + li * 1e-4) * np.cos(ph[1] + li * 3e-4)
        cal.append(T.CalibrationVector(li, pixels.copy(), k.astype(np.float32)))
        nz = 200.0 + 200.0 * np.sin(3 * math.pi * x + ph[2] + li * 2e-4)
        nr.append(T.NoiseRangeVector(li, pixels.copy(), np.clip(nz, 0, 400).astype(np.float32)))
    az_lines = np.array([0, tiff_height // 2, tiff_height - 1], np.int32)
    az_vals = (1.0 + 0.02 * rng.uniform(-1, 1, 3)).astype(np.float32)
    return (T.SwathCalibration(sid, cal),
            T.SwathNoise(sid, nr, [T.NoiseAzimuthVector(az_lines, az_vals)]))


def config2_scene(seed: int = 2, n_bursts: int = 9, lines_per_burst: int = 1500,
                  tiff_width: int = 21000, burst_step: int = 1400, swath_overlap: int = 2000,
                  out_rows: Optional[int] = 20000, out_cols: Optional[int] = 25000,
                  resampling=T.ResamplingKernel.Bicubic, flatten: bool = True,
                  compute_lia: bool = True, device: Optional[str] = None,
                  center_lat_deg: float = 46.0, utm_zone: Optional[int] = None,
                  hmax: float = 3000.0, spacing_m: float = 10.0,
                  lut_lines_step: Optional[int] = None) -> IwScene:
    """Full IW scene: 3 swaths x n_bursts x lines_per_burst x tiff_width CInt16,
    bursts overlapping by lines_per_burst - burst_step lines, swaths overlapping
    by ~swath_overlap samples; UTM 10 m DEM/output with fBm heights."""
    rng = np.random.default_rng(seed)
    t_center = EPOCH_US + int(rng.integers(0, 10**6)) * 1000
    orbit, orb = make_orbit(rng, t_center, center_lat_deg)
    tiff_height = n_bursts * lines_per_burst
    deb_lines = n_bursts * lines_per_burst - (n_bursts - 1) * (lines_per_burst - burst_step)
    dt = 2 * RPS / C_LIGHT
    t0 = t_center - int(round(deb_lines / 2 * ATI * 1e6))
    swaths: List[IwSwath] = []
    tau0 = 2 * NEAR_RANGE / C_LIGHT
    lut_step = lut_lines_step or int(round(1.0 / ATI))
    for k in range(3):
        sid = f"IW{k + 1}"
        tau_k = tau0 + k * (tiff_width - swath_overlap) * dt
        tk = t0 + k * int(round(0.25 * burst_step * ATI * 1e6))
        bursts = []
        for j in range(n_bursts):
            fv = int(rng.integers(40, 90))
            lv = tiff_width - int(rng.integers(40, 90))
            bursts.append(T.BurstEntry(sid, j, tk + int(round(j * burst_step * ATI * 1e6)),
                                       j * lines_per_burst, (j + 1) * lines_per_burst, fv, lv))
        sw = T.SubSwathMetadata(sid, n_bursts, lines_per_burst, tiff_width, ATI, RPS, tau_k)
        cal, noise = _luts(rng, sid, tiff_height, tiff_width, lut_step)
        swaths.append(IwSwath(sid, slc_raster(rng, tiff_height, tiff_width, 60.0, device), sw,
                              bursts, cal, noise))
    # footprint-centred UTM output grid
    width_slant = 3 * tiff_width - 2 * swath_overlap
    S, V = orb.state(t_center)
    Pc = forward_geocode(S, V, NEAR_RANGE + width_slant / 2 * RPS)
    lat_c, lon_c = (float(x) for x in ecef_to_geodetic(Pc))
    zone = utm_zone or int((lon_c + 180.0) // 6.0) + 1
    if out_rows is None or out_cols is None:
        corners = []
        for t in (t0, t0 + int(deb_lines * ATI * 1e6)):
            St, Vt = orb.state(t)
            for R in (NEAR_RANGE, NEAR_RANGE + width_slant * RPS):
                corners.append(ecef_to_geodetic(forward_geocode(St, Vt, R)))
        xs, ys = utm_forward_np([c[1] for c in corners], [c[0] for c in corners], zone)
        out_cols = int((np.max(xs) - np.min(xs)) / spacing_m)
        out_rows = int((np.max(ys) - np.min(ys)) / spacing_m)
    xc, yc = utm_forward_np(lon_c, lat_c, zone)
    x_left = math.floor(float(xc) / spacing_m - out_cols / 2) * spacing_m
    y_top = math.floor(float(yc) / spacing_m + out_rows / 2) * spacing_m
    bb = _bbox_for_utm_rect(x_left, y_top, out_cols, out_rows, spacing_m, zone)
    dem = T.DemGrid(fbm_surface(rng, out_rows, out_cols, 0.8, hmax, device),
                    y_top - 0.5 * spacing_m, x_left + 0.5 * spacing_m, spacing_m,
                    _abi.DEM_PROJECTED_UTM, zone, False)
    geoid = T.GeoidModel(geoid_grid(rng))
    scene = T.SceneMetadata([s.sw for s in swaths], [b for s in swaths for b in s.bursts], orbit, bb)
    iw2 = swaths[1]
    grid_pts = _geo_grid(orb, iw2.bursts[0].azimuth_time_us, deb_lines,
                         iw2.sw.slant_range_time_s * C_LIGHT / 2, tiff_width)
    grids = [(s.id, grid_pts if s.id == "IW2" else []) for s in swaths]
    cfg = T.TerrainCorrectionConfig(geoid=geoid, pixel_spacing_deg=spacing_m,
                                    crs=T.OutputCrs.utm_north(zone), flatten=flatten,
                                    compute_lia=compute_lia, resampling=resampling)
    return IwScene(swaths, scene, dem, grids, cfg, orb)


def _bbox_for_utm_rect(x_left, y_top, cols, rows, sp, zone) -> T.BoundingBox:
    """Lat/lon box whose projected corner envelope, snapped outward
    (terrain_correction.rs:1174-1216), is exactly the given UTM rectangle."""
    # targets a quarter pixel inside the rectangle so ceil/floor snap to it
    tx0, tx1 = x_left + 0.25 * sp, x_left + (cols - 0.25) * sp
    ty0, ty1 = y_top - (rows - 0.25) * sp, y_top - 0.25 * sp
    lon0, lon1, lat0, lat1 = _inv_guess(tx0, ty0, zone), _inv_guess(tx1, ty0, zone), None, None
    lat0 = _inv_guess_lat(tx0, ty0, zone)
    lat1 = _inv_guess_lat(tx0, ty1, zone)
    for _ in range(60):
        corners = [(lon0, lat0), (lon0, lat1), (lon1, lat0), (lon1, lat1)]
        xs, ys = utm_forward_np([c[0] for c in corners], [c[1] for c in corners], zone)
        ex0, ex1 = np.min(xs) - tx0, np.max(xs) - tx1
        ey0, ey1 = np.min(ys) - ty0, np.max(ys) - ty1
        m_lat = 111_320.0
        m_lon = 111_320.0 * math.cos(math.radians(0.5 * (lat0 + lat1)))
        lon0 -= ex0 / m_lon
        lon1 -= ex1 / m_lon
        lat0 -= ey0 / m_lat
        lat1 -= ey1 / m_lat
        if max(abs(ex0), abs(ex1), abs(ey0), abs(ey1)) < 1e-4:
            break
    return T.BoundingBox(lat0, lat1, lon0, lon1)


def _inv_guess(x, y, zone):
    lon0 = (zone - 1) * 6 - 180 + 3
    lat = y / 111_320.0
    return lon0 + (x - 500000.0) / (111_320.0 * math.cos(math.radians(lat)))


def _inv_guess_lat(x, y, zone):
    return y / 111_320.0


# ── batched tiles (config 4) and served requests (config 5) ────────────────
def config4_scene(seed: int, n_lines: int = 4096, n_samples: int = 8192, dem_n: int = 1024,
                  device: Optional[str] = None):
    """A config-1-shape scene whose radar image starts as CInt16 SLC with
    sigma0/noise LUTs (calibrated on the device every step): returns the
    TcScene, the (lines, samples, 2) int16 raster and (cal, noise)."""
    sc = config1_scene(seed=seed, n_lines=n_lines, n_samples=n_samples, dem_n=dem_n, flatten=True,
                       device=device)
    rng = np.random.default_rng(seed + 7919)
    slc = slc_raster(rng, n_lines, n_samples, 60.0, device)
    cal, noise = _luts(rng, "IW1", n_lines, n_samples, int(round(1.0 / ATI)))
    return sc, slc, cal, noise


def random_tiles(rng: np.random.Generator, grids, n: int, side_min: int, side_max: int,
                 kernels=(0, 1, 2), speckles=("refined_lee", "gamma_map"), enl: float = 4.4):
    """n tile specs over `grids` (per scene: (rows, cols)): side log-uniform
    in [side_min, side_max] (clipped to the grid), uniform scene, origin,
    resampling kernel and speckle filter.  Returns dicts of
    scene, r0, c0, rows, cols, kernel, speckle."""
    out = []
    for _ in range(n):
        k = int(rng.integers(0, len(grids)))
        gr, gc = grids[k]
        side = int(round(side_min * (side_max / side_min) ** rng.uniform()))
        rows, cols = min(side, gr), min(side, gc)
        r0 = int(rng.integers(0, gr - rows + 1))
        c0 = int(rng.integers(0, gc - cols + 1))
        sp = speckles[int(rng.integers(0, len(speckles)))] if speckles else None
        filt = None
        if sp == "refined_lee":
            filt = T.SpeckleFilter.RefinedLee(enl)
        elif sp == "gamma_map":
            filt = T.SpeckleFilter.GammaMap(5, enl)
        out.append({"scene": k, "r0": r0, "c0": c0, "rows": rows, "cols": cols,
                    "kernel": int(kernels[int(rng.integers(0, len(kernels)))]), "speckle": filt})
    return out
