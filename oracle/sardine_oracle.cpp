// sardine_oracle.cpp — CPU ORACLE for the SARdine hot path.
//
// TEST INFRASTRUCTURE ONLY.  This file restates, in plain C++, the reference
// Rust functions of SARdine's data-parallel hot path so that the CUDA
// implementation can be checked against it and so that bench.py can time a
// CPU baseline.  Nothing in the product (the sardine_b200 package and its CUDA
// library) links, loads or calls this code.
//
// Pinning: the reference cannot be built here (no Rust toolchain, crates not
// vendored).  The restatement is pinned against the reference's own synthetic
// known-answer tests (tests/test_oracle_kat.py, each case citing its source
// line).  Two parts rest on third-party code that is absent from the
// reference checkout and are restated from the published method instead:
//   * UTM (proj4rs 0.1.10, Cargo.lock:716-719): transverse Mercator from
//     Krueger's n-series as given by Karney (2011), "Transverse Mercator with
//     an accuracy of a few nanometers", J. Geodesy 85, eqs. 7-11, 35-36.
//     Pinned only to the reference's own UTM tests (output_crs.rs:597-628).
//     Its inverse (the anchors of a projected output row) always takes its
//     elementary functions from sardine_b200/csrc/crmath.cuh, one arithmetic
//     for host and device: proj4rs's own arithmetic is not available here,
//     and with one libm on both sides the anchors are the same bits in the
//     oracle and on the device.  The forward projection of DEM lookups
//     follows the libm setting below.
//   * libm sin/cos/sqrt: the reference calls the platform libm (glibc on
//     Linux); this file calls the same functions by default.  orc_set_libm(1)
//     switches the sines and cosines of geodetic_to_ecef and the functions of
//     the forward UTM projection to crmath.cuh (correctly rounded sin/cos):
//     the reference as it would run on a platform whose libm rounds
//     correctly.  The two settings differ exactly where glibc's results are
//     not correctly rounded (~1.4e-3 of its sin/cos results).
//
// Arithmetic follows the reference operation by operation: f32 where the
// reference uses f32, f64 where it uses f64, left-to-right evaluation, no
// fused multiply-add (build with -ffp-contract=off), microsecond time steps
// truncated toward zero, column-sequential Newton seeding.
//
// Citations are file:line in the reference repository (sardine/src/...).

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <mutex>
#include <thread>
#include <vector>

#include "../include/sardine_b200.h"
#include "../sardine_b200/csrc/crmath.cuh"

namespace {

// 0: the platform libm (the reference's); 1: crmath.cuh (correctly rounded
// sin/cos) for geodetic_to_ecef and the forward UTM projection.
std::atomic<int> g_cr_libm{0};
inline bool cr_libm() { return g_cr_libm.load(std::memory_order_relaxed) != 0; }

// ── constants (geodesy.rs:13-25, types.rs:11) ─────────────────────────────
constexpr double kPi = 3.14159265358979323846;  // std::f64::consts::PI
constexpr double WGS84_A = 6378137.0;
constexpr double WGS84_F = 1.0 / 298.257223563;
constexpr double WGS84_E2 = 2.0 * WGS84_F - WGS84_F * WGS84_F;
constexpr double SPEED_OF_LIGHT = 299792458.0;

// ── host parallelism: std::thread over row blocks (the reference uses Rayon
// over 64-row chunks; results never depend on the schedule) ───────────────
std::atomic<int> g_threads{0};
int n_threads() {
  int t = g_threads.load();
  if (t > 0) return t;
  unsigned h = std::thread::hardware_concurrency();
  return h == 0 ? 1 : (int)h;
}
// fn(begin, end, worker_index) over [0, n) in chunks of `chunk`.
template <class F>
void parallel_for(int64_t n, int64_t chunk, F fn) {
  int nt = n_threads();
  if (nt <= 1 || n <= chunk) {
    for (int64_t b = 0; b < n; b += chunk) fn(b, std::min(n, b + chunk), 0);
    return;
  }
  std::atomic<int64_t> next{0};
  std::vector<std::thread> pool;
  for (int w = 0; w < nt; ++w)
    pool.emplace_back([&, w]() {
      for (;;) {
        int64_t b = next.fetch_add(chunk);
        if (b >= n) break;
        fn(b, std::min(n, b + chunk), w);
      }
    });
  for (auto &t : pool) t.join();
}

// Rust `f as i64`: saturating, NaN -> 0.
inline int64_t f64_as_i64(double x) {
  if (std::isnan(x)) return 0;
  if (x >= 9223372036854775807.0) return INT64_MAX;
  if (x <= -9223372036854775808.0) return INT64_MIN;
  return (int64_t)x;
}
// Rust `f as isize` (64-bit).
inline int64_t f64_as_isize(double x) { return f64_as_i64(x); }
// Rust `f as usize`: saturating at 0 and u64::MAX, NaN -> 0.
inline uint64_t f64_as_usize(double x) {
  if (std::isnan(x) || x <= 0.0) return 0;
  if (x >= 18446744073709551615.0) return UINT64_MAX;
  return (uint64_t)x;
}
inline double clamp_f64(double x, double lo, double hi) {  // f64::clamp
  if (x < lo) x = lo;
  if (x > hi) x = hi;
  return x;
}
inline float clamp_f32(float x, float lo, float hi) {
  if (x < lo) x = lo;
  if (x > hi) x = hi;
  return x;
}
inline int64_t clamp_i64(int64_t x, int64_t lo, int64_t hi) { return x < lo ? lo : (x > hi ? hi : x); }
// f32::max / f64::max: NaN-ignoring.
inline float max_f32(float a, float b) { return std::isnan(a) ? b : (std::isnan(b) ? a : (a > b ? a : b)); }
inline double max_f64(double a, double b) { return std::isnan(a) ? b : (std::isnan(b) ? a : (a > b ? a : b)); }

// ── vec3 (geodesy.rs:98-132) ──────────────────────────────────────────────
struct V3 { double x, y, z; };
inline double dot3(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline double norm3(V3 v) { return std::sqrt(dot3(v, v)); }
inline V3 sub3(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline V3 cross3(V3 a, V3 b) {
  return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
inline V3 normalize3(V3 v) {
  double n = norm3(v);
  if (n == 0.0) return {0.0, 0.0, 0.0};
  return {v.x / n, v.y / n, v.z / n};
}

// geodetic_to_ecef (geodesy.rs:38-55)
inline V3 geodetic_to_ecef(double lat_deg, double lon_deg, double h) {
  double lat = lat_deg * kPi / 180.0;
  double lon = lon_deg * kPi / 180.0;
  double sin_lat, cos_lat, sin_lon, cos_lon;
  if (cr_libm()) {
    sd::crm::sincos(lat, &sin_lat, &cos_lat);
    sd::crm::sincos(lon, &sin_lon, &cos_lon);
  } else {
    sin_lat = std::sin(lat), cos_lat = std::cos(lat);
    sin_lon = std::sin(lon), cos_lon = std::cos(lon);
  }
  double n = WGS84_A / std::sqrt(1.0 - WGS84_E2 * sin_lat * sin_lat);
  return {(n + h) * cos_lat * cos_lon, (n + h) * cos_lat * sin_lon,
          (n * (1.0 - WGS84_E2) + h) * sin_lat};
}

// ── transverse Mercator (UTM) — Karney (2011) Krueger series, 6th order ──
struct Utm {
  int zone = 0;
  bool south = false;
  double lon0 = 0.0;  // radians
  double k0A = 0.0;
  double e = 0.0, e2m = 0.0;
  double alp[7] = {0}, bet[7] = {0};
};

Utm make_utm(int zone, bool south) {
  Utm u;
  u.zone = zone;
  u.south = south;
  u.lon0 = (double)((zone - 1) * 6 - 180 + 3) * (kPi / 180.0);
  const double f = WGS84_F;
  const double n = f / (2.0 - f);
  const double n2 = n * n, n3 = n2 * n, n4 = n3 * n, n5 = n4 * n, n6 = n5 * n;
  // rectifying radius A = a/(1+n) * (1 + n^2/4 + n^4/64 + n^6/256)  (Karney eq. 14)
  const double A = WGS84_A / (1.0 + n) * (1.0 + n2 / 4.0 + n4 / 64.0 + n6 / 256.0);
  u.k0A = 0.9996 * A;
  u.e = std::sqrt(f * (2.0 - f));
  u.e2m = 1.0 - f * (2.0 - f);
  // Karney eq. 35 (alpha, forward) and eq. 36 (beta, inverse)
  u.alp[1] = n / 2.0 - 2.0 * n2 / 3.0 + 5.0 * n3 / 16.0 + 41.0 * n4 / 180.0 - 127.0 * n5 / 288.0 + 7891.0 * n6 / 37800.0;
  u.alp[2] = 13.0 * n2 / 48.0 - 3.0 * n3 / 5.0 + 557.0 * n4 / 1440.0 + 281.0 * n5 / 630.0 - 1983433.0 * n6 / 1935360.0;
  u.alp[3] = 61.0 * n3 / 240.0 - 103.0 * n4 / 140.0 + 15061.0 * n5 / 26880.0 + 167603.0 * n6 / 181440.0;
  u.alp[4] = 49561.0 * n4 / 161280.0 - 179.0 * n5 / 168.0 + 6601661.0 * n6 / 7257600.0;
  u.alp[5] = 34729.0 * n5 / 80640.0 - 3418889.0 * n6 / 1995840.0;
  u.alp[6] = 212378941.0 * n6 / 319334400.0;
  u.bet[1] = n / 2.0 - 2.0 * n2 / 3.0 + 37.0 * n3 / 96.0 - n4 / 360.0 - 81.0 * n5 / 512.0 + 96199.0 * n6 / 604800.0;
  u.bet[2] = n2 / 48.0 + n3 / 15.0 - 437.0 * n4 / 1440.0 + 46.0 * n5 / 105.0 - 1118711.0 * n6 / 3870720.0;
  u.bet[3] = 17.0 * n3 / 480.0 - 37.0 * n4 / 840.0 - 209.0 * n5 / 4480.0 + 5569.0 * n6 / 90720.0;
  u.bet[4] = 4397.0 * n4 / 161280.0 - 11.0 * n5 / 504.0 - 830251.0 * n6 / 7257600.0;
  u.bet[5] = 4583.0 * n5 / 161280.0 - 108847.0 * n6 / 3991680.0;
  u.bet[6] = 20648693.0 * n6 / 638668800.0;
  return u;
}

inline double adjlon(double lam) {  // wrap to [-pi, pi]
  while (lam > kPi) lam -= 2.0 * kPi;
  while (lam < -kPi) lam += 2.0 * kPi;
  return lam;
}

// sum_j c[j] * sin(2 j (xi + i eta)), returned as (re, im)
inline void krueger_sum(const double *c, double xi, double eta, double *re, double *im, bool crl) {
  double s1 = crl ? sd::crm::sin(2.0 * xi) : std::sin(2.0 * xi);
  double c1 = crl ? sd::crm::cos(2.0 * xi) : std::cos(2.0 * xi);
  double sh1 = crl ? sd::crm::sinh(2.0 * eta) : std::sinh(2.0 * eta);
  double ch1 = crl ? sd::crm::cosh(2.0 * eta) : std::cosh(2.0 * eta);
  // sin(2 zeta) and cos(2 zeta) for zeta = xi + i eta
  double sr = s1 * ch1, si = c1 * sh1;    // sin(2z)
  double cr = c1 * ch1, ci = -s1 * sh1;   // cos(2z)
  // Chebyshev recurrence: sin((j+1)w) = 2 cos(w) sin(jw) - sin((j-1)w)
  double pr = 0.0, pi = 0.0;  // sin(0 w)
  double qr = sr, qi = si;    // sin(1 w)
  double accr = 0.0, acci = 0.0;
  for (int j = 1; j <= 6; ++j) {
    accr += c[j] * qr;
    acci += c[j] * qi;
    double nr = 2.0 * (cr * qr - ci * qi) - pr;
    double ni = 2.0 * (cr * qi + ci * qr) - pi;
    pr = qr; pi = qi; qr = nr; qi = ni;
  }
  *re = accr;
  *im = acci;
}

inline double taupf(double tau, double e, bool cr) {  // tau' from tau (Karney eq. 7-9)
  if (cr) {
    double tau1 = sd::crm::hypot(1.0, tau);
    double sig = sd::crm::sinh(e * sd::crm::atanh(e * tau / tau1));
    return sd::crm::hypot(1.0, sig) * tau - sig * tau1;
  }
  double tau1 = std::hypot(1.0, tau);
  double sig = std::sinh(e * std::atanh(e * tau / tau1));
  return std::hypot(1.0, sig) * tau - sig * tau1;
}

inline double tauf(double taup, double e, double e2m) {  // inverse of taupf (eq. 19-21)
  double tau = taup / e2m;
  for (int i = 0; i < 6; ++i) {
    double taupa = taupf(tau, e, true);
    double dtau = (taup - taupa) * (1.0 + e2m * tau * tau) /
                  (e2m * sd::crm::hypot(1.0, tau) * sd::crm::hypot(1.0, taupa));
    tau += dtau;
    if (!(std::fabs(dtau) >= 1e-15 * std::max(1.0, std::fabs(tau)))) break;
  }
  return tau;
}

// lon, lat in radians -> easting, northing (m)
void utm_forward(const Utm &u, double lon, double lat, double *x, double *y) {
  const bool cr = cr_libm();
  double lam = adjlon(lon - u.lon0);
  double tau = cr ? sd::crm::tan(lat) : std::tan(lat);
  double taup = taupf(tau, u.e, cr);
  double xip, etap;
  if (cr) {
    xip = sd::crm::atan2(taup, sd::crm::cos(lam));
    etap = sd::crm::asinh(sd::crm::sin(lam) / sd::crm::hypot(taup, sd::crm::cos(lam)));
  } else {
    xip = std::atan2(taup, std::cos(lam));
    etap = std::asinh(std::sin(lam) / std::hypot(taup, std::cos(lam)));
  }
  double sr, si;
  krueger_sum(u.alp, xip, etap, &sr, &si, cr);
  double xi = xip + sr, eta = etap + si;
  *x = 500000.0 + u.k0A * eta;
  *y = (u.south ? 10000000.0 : 0.0) + u.k0A * xi;
}

// easting, northing (m) -> lon, lat in radians
void utm_inverse(const Utm &u, double x, double y, double *lon, double *lat) {
  double xi = (y - (u.south ? 10000000.0 : 0.0)) / u.k0A;
  double eta = (x - 500000.0) / u.k0A;
  double sr, si;
  krueger_sum(u.bet, xi, eta, &sr, &si, true);
  double xip = xi - sr, etap = eta - si;
  double s = sd::crm::sinh(etap), c = sd::crm::cos(xip);
  double taup = sd::crm::sin(xip) / sd::crm::hypot(s, c);
  double tau = tauf(taup, u.e, u.e2m);
  *lat = sd::crm::atan(tau);
  *lon = adjlon(sd::crm::atan2(s, c) + u.lon0);
}

// Projector::lonlat_to_xy / xy_to_lonlat (output_crs.rs:301-340): degrees in
// and out at the API; Rust to_radians is x*(PI/180), to_degrees x*(180/PI).
inline void lonlat_to_xy(const Utm &u, double lon_deg, double lat_deg, double *x, double *y) {
  utm_forward(u, lon_deg * (kPi / 180.0), lat_deg * (kPi / 180.0), x, y);
}
inline void xy_to_lonlat(const Utm &u, double x, double y, double *lon_deg, double *lat_deg) {
  double lo, la;
  utm_inverse(u, x, y, &lo, &la);
  *lon_deg = lo * (180.0 / kPi);
  *lat_deg = la * (180.0 / kPi);
}

// Projector::project_row (output_crs.rs:364-417)
void project_row(const Utm &u, double y, double x_start, double x_step, size_t n_cols,
                 size_t n_anchors, std::vector<double> &lon, std::vector<double> &lat) {
  lon.resize(n_cols);
  lat.resize(n_cols);
  if (n_cols == 0) return;
  n_anchors = std::min(n_anchors, n_cols);
  double x_end = x_start + ((double)n_cols - 1.0) * x_step;
  size_t n_pts = n_anchors + 1;
  double anchor_dx = (x_end - x_start) / (double)n_anchors;
  std::vector<double> ax(n_pts), alon(n_pts), alat(n_pts);
  for (size_t i = 0; i < n_pts; ++i) {
    double xi = x_start + (double)i * anchor_dx;
    ax[i] = xi;
    xy_to_lonlat(u, xi, y, &alon[i], &alat[i]);
  }
  size_t seg = 0;
  for (size_t col = 0; col < n_cols; ++col) {
    double x = x_start + (double)col * x_step;
    while (seg + 1 < n_anchors && x > ax[seg + 1]) seg++;
    double x0 = ax[seg], x1 = ax[seg + 1];
    double t = (x1 == x0) ? 0.0 : (x - x0) / (x1 - x0);
    lon[col] = alon[seg] + t * (alon[seg + 1] - alon[seg]);
    lat[col] = alat[seg] + t * (alat[seg + 1] - alat[seg]);
  }
}

// ── DEM (dem.rs:385-409 bilinear_on_grid; 351-371 Glo30Tile; 694-723 mosaic) ─
// Returns false for "no tile covers the point" (Err(OutOfBounds)); NaN for voids.
inline bool bilinear_on_grid(const float *data, size_t dim, double row_f, double col_f,
                             size_t max_rc, float *out) {
  size_t r0 = std::min<size_t>(f64_as_usize(row_f), max_rc == 0 ? 0 : max_rc - 1);
  size_t c0 = std::min<size_t>(f64_as_usize(col_f), dim < 2 ? 0 : dim - 2);
  size_t r1 = r0 + 1, c1 = c0 + 1;
  double dr = row_f - (double)r0;
  double dc = col_f - (double)c0;
  float v00 = data[r0 * dim + c0], v01 = data[r0 * dim + c1];
  float v10 = data[r1 * dim + c0], v11 = data[r1 * dim + c1];
  if (std::isnan(v00) || std::isnan(v01) || std::isnan(v10) || std::isnan(v11)) {
    *out = std::numeric_limits<float>::quiet_NaN();  // None -> caller treats as missing
    return true;
  }
  double v = (double)v00 * (1.0 - dr) * (1.0 - dc) + (double)v01 * (1.0 - dr) * dc +
             (double)v10 * dr * (1.0 - dc) + (double)v11 * dr * dc;
  *out = (float)v;
  return true;
}

struct Dem {
  sd_dem d;
  Utm utm;
};

// DemSource::elevation_at.  returns 0 = Ok(h) (h may be NaN), 1 = Err.
inline int dem_elevation(const Dem &dem, double lat_deg, double lon_deg, float *h) {
  const sd_dem &d = dem.d;
  double row_f, col_f;
  if (d.kind == SD_DEM_GEOGRAPHIC) {
    // DemMosaic::elevation_at normalises lon (dem.rs:697) before the tile lookup.
    double lon_norm = lon_deg >= 180.0 ? lon_deg - 360.0 : lon_deg;
    row_f = (d.origin_y - lat_deg) / d.pixel_size;
    col_f = (lon_norm - d.origin_x) / d.pixel_size;
  } else {
    double x, y;
    lonlat_to_xy(dem.utm, lon_deg, lat_deg, &x, &y);
    row_f = (d.origin_y - y) / d.pixel_size;
    col_f = (x - d.origin_x) / d.pixel_size;
  }
  double max_row = (double)(d.height - 1);
  double max_col = (double)(d.width - 1);
  const double margin = 0.5;
  if (row_f < -margin || row_f > max_row + margin || col_f < -margin || col_f > max_col + margin)
    return 1;
  // NaN coordinates fail every comparison above and reach here; the
  // reference's Glo30 tile then clamps NaN (clamp keeps NaN) and casts to 0.
  row_f = clamp_f64(row_f, 0.0, max_row);
  col_f = clamp_f64(col_f, 0.0, max_col);
  float v;
  bilinear_on_grid(d.data, d.width, row_f, col_f, d.height - 1, &v);
  *h = v;
  return 0;
}

// ── geoid (geoid.rs:220-251) ──────────────────────────────────────────────
inline double geoid_undulation(const sd_geoid &g, double lat_deg, double lon_deg) {
  if (g.kind == SD_GEOID_ZERO) return 0.0;
  const size_t NLAT = 73, NLON = 144;
  const double STEP = 2.5;
  double lon = std::fmod(lon_deg, 360.0);  // rem_euclid
  if (lon < 0.0) lon += 360.0;
  double row_f = (90.0 - clamp_f64(lat_deg, -90.0, 90.0)) / STEP;
  double col_f = lon / STEP;
  size_t r0 = std::min<size_t>(f64_as_usize(row_f), NLAT - 2);
  size_t r1 = r0 + 1;
  size_t c0 = f64_as_usize(col_f) % NLON;
  size_t c1 = (c0 + 1) % NLON;
  double dr = row_f - (double)r0;
  double dc = col_f - (double)c0;
  double v00 = g.undulations_m[r0 * NLON + c0], v01 = g.undulations_m[r0 * NLON + c1];
  double v10 = g.undulations_m[r1 * NLON + c0], v11 = g.undulations_m[r1 * NLON + c1];
  dc = clamp_f64(dc, 0.0, 1.0);
  return v00 * (1.0 - dr) * (1.0 - dc) + v01 * (1.0 - dr) * dc + v10 * dr * (1.0 - dc) +
         v11 * dr * dc;
}

// ── orbit (orbit.rs:498-596) ──────────────────────────────────────────────
enum { ORB_OK = 0, ORB_INSUFFICIENT = 1, ORB_OUTSIDE = 2 };

int interpolate_orbit_and_accel(const sd_state_vector *svs, size_t n, int64_t t, V3 *pos,
                                V3 *vel, V3 *acc) {
  const size_t DEG = 8;
  if (n < DEG) return ORB_INSUFFICIENT;
  if (t < svs[0].time_us || t > svs[n - 1].time_us) return ORB_OUTSIDE;
  const int64_t t_ref = svs[0].time_us;
  double t_sec = (double)(t - t_ref) / 1e6;
  // centre: largest i with svs[i].time <= t (the thread-local hint only
  // changes the walk length, never the result; orbit.rs:19-36)
  size_t lo = 0, hi = n;  // upper_bound
  while (lo < hi) {
    size_t mid = (lo + hi) / 2;
    if (svs[mid].time_us <= t) lo = mid + 1; else hi = mid;
  }
  size_t centre = lo - 1;
  const size_t half = DEG / 2;
  size_t start = centre < half ? 0 : (centre + half >= n ? n - DEG : centre - half + 1);
  double times[8];
  for (size_t i = 0; i < DEG; ++i) times[i] = (double)(svs[start + i].time_us - t_ref) / 1e6;
  double rdiff[8] = {0};
  double total_rdiff = 0.0;
  for (size_t j = 0; j < DEG; ++j) {
    double diff = t_sec - times[j];
    if (std::fabs(diff) > 1e-9) {
      rdiff[j] = 1.0 / diff;
      total_rdiff += rdiff[j];
    }
  }
  double p[3] = {0, 0, 0}, v[3] = {0, 0, 0}, a[3] = {0, 0, 0};
  for (size_t k = 0; k < DEG; ++k) {
    double basis = 1.0;
    for (size_t j = 0; j < DEG; ++j)
      if (j != k) basis *= (t_sec - times[j]) / (times[k] - times[j]);
    double d_basis = basis * (total_rdiff - rdiff[k]);
    const sd_state_vector &sv = svs[start + k];
    for (int c = 0; c < 3; ++c) {
      p[c] += basis * sv.position_m[c];
      v[c] += basis * sv.velocity_m_s[c];
      a[c] += d_basis * sv.velocity_m_s[c];
    }
  }
  *pos = {p[0], p[1], p[2]};
  *vel = {v[0], v[1], v[2]};
  *acc = {a[0], a[1], a[2]};
  return ORB_OK;
}

// ── zero-Doppler (terrain_correction.rs:1010-1073) ────────────────────────
enum { ZD_CONVERGED = 0, ZD_NOT_CONVERGED = 1, ZD_DEGENERATE = 2, ZD_ORBIT_ERROR = 3 };
struct ZdOut {
  int status;
  int64_t t;
  int iterations;
  V3 pos, vel;
  double residual;
};

ZdOut solve_zero_doppler(V3 target, const sd_state_vector *svs, size_t n, int64_t guess,
                         size_t max_iter, double tol) {
  const double DERIV_FLOOR = 1.0;
  ZdOut o{};
  int64_t t = guess;
  double last_delta = std::numeric_limits<double>::infinity();
  for (size_t i = 0; i < max_iter; ++i) {
    V3 pos, vel, acc;
    if (interpolate_orbit_and_accel(svs, n, t, &pos, &vel, &acc) != ORB_OK) {
      o.status = ZD_ORBIT_ERROR;
      o.t = t;
      return o;
    }
    V3 r = sub3(target, pos);
    double f = dot3(r, vel);
    double v_sq = dot3(vel, vel);
    double f_prime = -v_sq + dot3(r, acc);
    if (std::fabs(f_prime) < DERIV_FLOOR) {
      o.status = ZD_DEGENERATE;
      return o;
    }
    double delta = -f / f_prime;
    last_delta = delta;
    if (std::fabs(delta) < tol) {
      o.status = ZD_CONVERGED;
      o.t = t;
      o.iterations = (int)std::min<size_t>(i + 1, 255);
      o.pos = pos;
      o.vel = vel;
      o.residual = std::fabs(delta);
      return o;
    }
    t = t + f64_as_i64(delta * 1e6);
  }
  o.status = ZD_NOT_CONVERGED;
  o.residual = std::fabs(last_delta);
  return o;
}

// ── azimuth-time LUT (terrain_correction.rs:1080-1137) ───────────────────
struct LutPt { double lat; int64_t t; };

std::vector<LutPt> build_azimuth_time_lut(const sd_geo_grid_point *pts, size_t n) {
  std::vector<LutPt> lut;
  for (size_t i = 0; i < n; ++i) lut.push_back({pts[i].latitude_deg, pts[i].azimuth_time_us});
  std::stable_sort(lut.begin(), lut.end(), [](const LutPt &a, const LutPt &b) { return a.lat < b.lat; });
  std::vector<LutPt> out;
  for (const LutPt &p : lut) {
    if (!out.empty() && std::fabs(p.lat - out.back().lat) < 1e-6) continue;  // dedup_by keeps first
    out.push_back(p);
  }
  return out;
}

int64_t guess_azimuth_time(const std::vector<LutPt> &lut, double lat) {
  if (lut.size() == 1) return lut[0].t;
  // binary_search_by over sorted latitudes
  size_t lo = 0, hi = lut.size();
  while (lo < hi) {
    size_t mid = lo + (hi - lo) / 2;
    if (lut[mid].lat < lat) lo = mid + 1;
    else if (lut[mid].lat > lat) hi = mid;
    else return lut[mid].t;  // Ok(i)
  }
  size_t idx = lo;
  if (idx == 0) return lut[0].t;
  if (idx >= lut.size()) return lut.back().t;
  const LutPt &a = lut[idx - 1], &b = lut[idx];
  double frac = (lat - a.lat) / (b.lat - a.lat);
  double dt_us = (double)(b.t - a.t);
  return a.t + f64_as_i64(frac * dt_us);
}

// ── resampling (terrain_correction.rs:770-983) ────────────────────────────
float bilinear_sample_slice(const float *data, size_t n_lines, size_t n_samples, double line,
                            double sample) {
  int64_t max_line = n_lines == 0 ? 0 : (int64_t)n_lines - 1;
  int64_t max_sample = n_samples == 0 ? 0 : (int64_t)n_samples - 1;
  int64_t l0 = clamp_i64(f64_as_isize(std::floor(line)), 0, max_line);
  int64_t l1 = std::min<int64_t>(l0 + 1, max_line);
  int64_t s0 = clamp_i64(f64_as_isize(std::floor(sample)), 0, max_sample);
  int64_t s1 = std::min<int64_t>(s0 + 1, max_sample);
  double dl = line - (double)l0;
  double ds = sample - (double)s0;
  float v00 = data[l0 * n_samples + s0], v01 = data[l0 * n_samples + s1];
  float v10 = data[l1 * n_samples + s0], v11 = data[l1 * n_samples + s1];
  if (std::isnan(v00) || std::isnan(v01) || std::isnan(v10) || std::isnan(v11))
    return std::numeric_limits<float>::quiet_NaN();
  double w00 = (1.0 - dl) * (1.0 - ds);
  double w01 = (1.0 - dl) * ds;
  double w10 = dl * (1.0 - ds);
  double w11 = dl * ds;
  return (float)((double)v00 * w00 + (double)v01 * w01 + (double)v10 * w10 + (double)v11 * w11);
}

inline double keys_weight(double t) {
  t = std::fabs(t);
  if (t < 1.0) return 1.5 * t * t * t - 2.5 * t * t + 1.0;
  if (t < 2.0) return -0.5 * t * t * t + 2.5 * t * t - 4.0 * t + 2.0;
  return 0.0;
}

float bicubic_sample_slice(const float *data, size_t n_lines, size_t n_samples, double line,
                           double sample) {
  int64_t max_l = (int64_t)n_lines - 1, max_s = (int64_t)n_samples - 1;
  int64_t l_floor = f64_as_isize(std::floor(line));
  int64_t s_floor = f64_as_isize(std::floor(sample));
  double dl = line - (double)l_floor;
  double ds = sample - (double)s_floor;
  double acc = 0.0;
  for (int64_t li = -1; li <= 2; ++li) {
    int64_t row = clamp_i64(l_floor + li, 0, max_l);
    double wl = keys_weight((double)li - dl);
    for (int64_t si = -1; si <= 2; ++si) {
      int64_t col = clamp_i64(s_floor + si, 0, max_s);
      float v = data[row * (int64_t)n_samples + col];
      if (std::isnan(v)) return std::numeric_limits<float>::quiet_NaN();
      acc += (double)v * wl * keys_weight((double)si - ds);
    }
  }
  return (float)acc;
}

inline double lanczos_weight(double x) {
  const double A = 3.0;
  double ax = std::fabs(x);
  if (ax < 1e-10) return 1.0;
  if (ax < A) {
    double px = kPi * x;
    double pxa = kPi * x / A;
    return std::sin(px) * std::sin(pxa) / (px * pxa);
  }
  return 0.0;
}

float lanczos_sample_slice(const float *data, size_t n_lines, size_t n_samples, double line,
                           double sample) {
  int64_t max_l = (int64_t)n_lines - 1, max_s = (int64_t)n_samples - 1;
  int64_t l_floor = f64_as_isize(std::floor(line));
  int64_t s_floor = f64_as_isize(std::floor(sample));
  double acc = 0.0;
  for (int64_t li = -2; li <= 3; ++li) {
    int64_t row = clamp_i64(l_floor + li, 0, max_l);
    double wl = lanczos_weight(line - (double)(l_floor + li));
    for (int64_t si = -2; si <= 3; ++si) {
      int64_t col = clamp_i64(s_floor + si, 0, max_s);
      float v = data[row * (int64_t)n_samples + col];
      if (std::isnan(v)) return std::numeric_limits<float>::quiet_NaN();
      acc += (double)v * wl * lanczos_weight(sample - (double)(s_floor + si));
    }
  }
  return (float)acc;
}

// ── terrain geometry (terrain_correction.rs:576-651) ─────────────────────
enum { GEOM_VALID = 0, GEOM_FORESHORTENING = 1, GEOM_LAYOVER = 2, GEOM_SHADOW = 3 };

double flat_cell_area(double lat, double lon, double sp) {
  V3 fe = geodetic_to_ecef(lat, lon + sp, 0.0);
  V3 fw = geodetic_to_ecef(lat, lon - sp, 0.0);
  V3 fn = geodetic_to_ecef(lat + sp, lon, 0.0);
  V3 fs = geodetic_to_ecef(lat - sp, lon, 0.0);
  return norm3(cross3(sub3(fe, fw), sub3(fn, fs)));
}

int terrain_geometry(double lat, double lon, double he, double hw, double hn, double hs,
                     V3 sat, V3 target, double sp, double flat_area, double *w_out,
                     double *cos_lia_out) {
  V3 pe = geodetic_to_ecef(lat, lon + sp, he);
  V3 pw = geodetic_to_ecef(lat, lon - sp, hw);
  V3 pn = geodetic_to_ecef(lat + sp, lon, hn);
  V3 ps = geodetic_to_ecef(lat - sp, lon, hs);
  V3 normal = cross3(sub3(pe, pw), sub3(pn, ps));
  V3 look = normalize3(sub3(sat, target));
  double local_proj = dot3(normal, look);
  if (local_proj <= 0.0) return GEOM_SHADOW;
  double area = norm3(normal);
  if (area == 0.0) return GEOM_SHADOW;
  double cos_lia = clamp_f64(local_proj / area, 0.0, 1.0);
  double w = local_proj / flat_area;
  *cos_lia_out = cos_lia;
  *w_out = w;
  if (w < 0.05) return GEOM_FORESHORTENING;
  if (w > 2.0) return GEOM_LAYOVER;
  return GEOM_VALID;
}

}  // namespace

// ═══════════════════════════════════════════════════════════════════════════
// extern "C" surface used by tests/ and bench.py (ctypes)
// ═══════════════════════════════════════════════════════════════════════════
extern "C" {

// Worker threads for the parallel loops (0 = all hardware threads).
void orc_set_threads(int n) { g_threads.store(n < 0 ? 0 : n); }
int orc_get_threads(void) { return n_threads(); }

// Sines and cosines of geodetic_to_ecef and the forward UTM projection's
// functions: 0 = the platform libm (default, the reference's), 1 = crmath.cuh.
void orc_set_libm(int correctly_rounded) { g_cr_libm.store(correctly_rounded ? 1 : 0); }
int orc_get_libm(void) { return g_cr_libm.load(); }

// Correctly rounded sin and cos of n doubles (the reference values the device's are tested against).
void orc_cr_sincos(const double *x, uint64_t n, double *s, double *c) {
  for (uint64_t i = 0; i < n; ++i) sd::crm::sincos(x[i], s + i, c + i);
}

int orc_interpolate_orbit_and_accel(const sd_state_vector *svs, uint64_t n, int64_t t,
                                    double *pos, double *vel, double *acc) {
  V3 p, v, a;
  int rc = interpolate_orbit_and_accel(svs, n, t, &p, &v, &a);
  if (rc != ORB_OK) return rc;
  pos[0] = p.x; pos[1] = p.y; pos[2] = p.z;
  vel[0] = v.x; vel[1] = v.y; vel[2] = v.z;
  acc[0] = a.x; acc[1] = a.y; acc[2] = a.z;
  return 0;
}

int orc_solve_zero_doppler(const double *target, const sd_state_vector *svs, uint64_t n,
                           int64_t guess, uint64_t max_iter, double tol, int64_t *t_out,
                           int32_t *iters_out, double *residual_out) {
  ZdOut o = solve_zero_doppler({target[0], target[1], target[2]}, svs, n, guess, max_iter, tol);
  *t_out = o.t;
  *iters_out = o.iterations;
  *residual_out = o.residual;
  return o.status;
}

void orc_geodetic_to_ecef(double lat, double lon, double h, double *out) {
  V3 p = geodetic_to_ecef(lat, lon, h);
  out[0] = p.x; out[1] = p.y; out[2] = p.z;
}

void orc_utm_lonlat_to_xy(int zone, int south, double lon, double lat, double *x, double *y) {
  Utm u = make_utm(zone, south != 0);
  lonlat_to_xy(u, lon, lat, x, y);
}
void orc_utm_xy_to_lonlat(int zone, int south, double x, double y, double *lon, double *lat) {
  Utm u = make_utm(zone, south != 0);
  xy_to_lonlat(u, x, y, lon, lat);
}
void orc_project_row(int zone, int south, double y, double x_start, double x_step,
                     uint64_t n_cols, uint64_t n_anchors, double *lon, double *lat) {
  Utm u = make_utm(zone, south != 0);
  std::vector<double> lo, la;
  project_row(u, y, x_start, x_step, n_cols, n_anchors, lo, la);
  std::memcpy(lon, lo.data(), n_cols * sizeof(double));
  std::memcpy(lat, la.data(), n_cols * sizeof(double));
}

float orc_bilinear_sample(const float *d, uint64_t nl, uint64_t ns, double l, double s) {
  return bilinear_sample_slice(d, nl, ns, l, s);
}
float orc_bicubic_sample(const float *d, uint64_t nl, uint64_t ns, double l, double s) {
  return bicubic_sample_slice(d, nl, ns, l, s);
}
float orc_lanczos_sample(const float *d, uint64_t nl, uint64_t ns, double l, double s) {
  return lanczos_sample_slice(d, nl, ns, l, s);
}
double orc_keys_weight(double t) { return keys_weight(t); }
double orc_lanczos_weight(double x) { return lanczos_weight(x); }
double orc_flat_cell_area(double lat, double lon, double sp) { return flat_cell_area(lat, lon, sp); }
int orc_terrain_geometry(double lat, double lon, double he, double hw, double hn, double hs,
                         const double *sat, const double *target, double sp, double flat_area,
                         double *w, double *cos_lia) {
  return terrain_geometry(lat, lon, he, hw, hn, hs, {sat[0], sat[1], sat[2]},
                          {target[0], target[1], target[2]}, sp, flat_area, w, cos_lia);
}
double orc_geoid_undulation(const sd_geoid *g, double lat, double lon) {
  return geoid_undulation(*g, lat, lon);
}
int orc_dem_elevation(const sd_dem *d, double lat, double lon, float *h) {
  Dem dem{*d, make_utm(d->utm_zone > 0 ? d->utm_zone : 1, d->utm_south != 0)};
  return dem_elevation(dem, lat, lon, h);
}
int64_t orc_guess_azimuth_time(const sd_geo_grid_point *pts, uint64_t n, double lat) {
  auto lut = build_azimuth_time_lut(pts, n);
  if (lut.empty()) return 0;
  return guess_azimuth_time(lut, lat);
}

// compute_output_grid_extent + grid size (terrain_correction.rs:1174-1216, 1297-1320)
int orc_tc_output_grid(const sd_scene *scene, const sd_tc_config *cfg, sd_geocoded_info *info) {
  std::memset(info, 0, sizeof(*info));
  if (!(cfg->pixel_spacing > 0.0)) return SD_ERR_TC_CONFIG;
  double sp = cfg->pixel_spacing;
  double n, s, w, e;
  if (cfg->crs == SD_CRS_WGS84) {
    n = std::ceil(scene->max_lat_deg / sp) * sp;
    s = std::floor(scene->min_lat_deg / sp) * sp;
    w = std::floor(scene->min_lon_deg / sp) * sp;
    e = std::ceil(scene->max_lon_deg / sp) * sp;
  } else {
    Utm u = make_utm(cfg->utm_zone, cfg->crs == SD_CRS_UTM_SOUTH);
    double corners[4][2] = {{scene->min_lon_deg, scene->min_lat_deg},
                            {scene->min_lon_deg, scene->max_lat_deg},
                            {scene->max_lon_deg, scene->min_lat_deg},
                            {scene->max_lon_deg, scene->max_lat_deg}};
    double xmin = INFINITY, xmax = -INFINITY, ymin = INFINITY, ymax = -INFINITY;
    for (auto &c : corners) {
      double x, y;
      lonlat_to_xy(u, c[0], c[1], &x, &y);
      if (x < xmin) xmin = x;
      if (x > xmax) xmax = x;
      if (y < ymin) ymin = y;
      if (y > ymax) ymax = y;
    }
    n = std::ceil(ymax / sp) * sp;
    s = std::floor(ymin / sp) * sp;
    w = std::floor(xmin / sp) * sp;
    e = std::ceil(xmax / sp) * sp;
  }
  uint64_t rows = f64_as_usize(std::round((n - s) / sp));
  uint64_t cols = f64_as_usize(std::round((e - w) / sp));
  info->rows = rows;
  info->cols = cols;
  info->origin_lat_deg = n;
  info->origin_lon_deg = w;
  info->pixel_spacing = sp;
  info->geotransform[0] = w; info->geotransform[1] = sp; info->geotransform[2] = 0.0;
  info->geotransform[3] = n; info->geotransform[4] = 0.0; info->geotransform[5] = -sp;
  info->total_pixel_count = rows * cols;
  if (rows == 0 || cols == 0) return SD_ERR_TC_CONFIG;
  return SD_OK;
}

// terrain_correction (terrain_correction.rs:1245-1836).  Rows [row_begin,
// row_end) only (row_end = 0 means all rows): the per-row chain makes any row
// band an exact sub-problem, which the CPU baseline uses as its sample.
// out_t_us / out_iters (optional) receive the converged azimuth time and the
// Newton iteration count per pixel (INT64_MIN / 0 where no solve converged).
static int tc_impl(const sd_radar_image *img, const sd_scene *scene, const sd_dem *dem_in,
                   const sd_geoid *geoid, const sd_geo_grid_point *grid, uint64_t n_grid,
                   const sd_tc_config *cfg, const double *forced_grid, uint64_t row_begin,
                   uint64_t row_end, float *out_data, float *out_cos_lia, uint8_t *out_mask,
                   int64_t *out_t_us, uint8_t *out_iters, sd_geocoded_info *info) {
  if (n_grid == 0) return SD_ERR_TC_NO_GRID_POINTS;
  if (!(cfg->pixel_spacing > 0.0)) return SD_ERR_TC_CONFIG;
  if (scene->n_sub_swaths <= 0) return SD_ERR_TC_NO_SUBSWATHS;
  const double ati = scene->azimuth_time_interval_s;
  if (!std::isfinite(ati) || ati <= 0.0) return SD_ERR_TC_CONFIG;
  const double near_range_m = img->near_slant_range_time_s * SPEED_OF_LIGHT / 2.0;
  const double rps = img->range_pixel_spacing_m;
  auto lut = build_azimuth_time_lut(grid, n_grid);
  if (lut.empty()) return SD_ERR_TC_NO_GRID_POINTS;
  int rc = SD_OK;
  if (forced_grid) {
    // an explicit grid {west edge, north edge, rows, cols}: the output grid
    // terrain_correction derives from a bounding box that snaps to it
    std::memset(info, 0, sizeof *info);
    info->origin_lon_deg = forced_grid[0];
    info->origin_lat_deg = forced_grid[1];
    info->rows = (uint64_t)forced_grid[2];
    info->cols = (uint64_t)forced_grid[3];
    info->pixel_spacing = cfg->pixel_spacing;
    info->geotransform[0] = forced_grid[0];
    info->geotransform[1] = cfg->pixel_spacing;
    info->geotransform[3] = forced_grid[1];
    info->geotransform[5] = -cfg->pixel_spacing;
    info->total_pixel_count = info->rows * info->cols;
    if (info->rows == 0 || info->cols == 0) return SD_ERR_TC_CONFIG;
  } else {
    rc = orc_tc_output_grid(scene, cfg, info);
  }
  if (rc != SD_OK) return rc;
  if (cfg->projector_anchors <= 0) return SD_ERR_TC_CONFIG;
  const bool utm = cfg->crs != SD_CRS_WGS84;
  Utm proj;
  if (utm) proj = make_utm(cfg->utm_zone, cfg->crs == SD_CRS_UTM_SOUTH);
  Dem dem{*dem_in, make_utm(dem_in->utm_zone > 0 ? dem_in->utm_zone : 1, dem_in->utm_south != 0)};
  const uint64_t n_rows = info->rows, n_cols = info->cols;
  const double sp = cfg->pixel_spacing;
  const double lat_north = info->origin_lat_deg, lon_west = info->origin_lon_deg;
  const double step_deg = utm ? sp / 111320.0 : sp;  // cardinal_neighbour_step_deg (452-465)
  const bool need_geom = cfg->flatten || cfg->compute_lia;
  const bool nesz_mask = std::isfinite(cfg->noise_floor_margin_db) && img->nesz != nullptr;
  const float nesz_factor = nesz_mask ? std::pow(10.0f, cfg->noise_floor_margin_db / 10.0f) : 0.0f;
  if (row_end == 0 || row_end > n_rows) row_end = n_rows;
  const float fnan = std::numeric_limits<float>::quiet_NaN();

  uint64_t c_valid = 0, c_dem = 0, c_out = 0, c_nc = 0, c_deg = 0, c_flat = 0, c_noise = 0;
  uint64_t hist[SD_NEWTON_ITER_HIST_SIZE] = {0};
  std::atomic<int> orbit_error{0};

  std::mutex mu;
  parallel_for((int64_t)(row_end - row_begin), 1, [&](int64_t rb, int64_t re, int) {
    uint64_t l_valid = 0, l_dem = 0, l_out = 0, l_nc = 0, l_deg = 0, l_flat = 0, l_noise = 0;
    uint64_t l_hist[SD_NEWTON_ITER_HIST_SIZE] = {0};
    std::vector<double> rlon, rlat;
    for (int64_t row_i = (int64_t)row_begin + rb; row_i < (int64_t)row_begin + re; ++row_i) {
      if (orbit_error.load(std::memory_order_relaxed)) continue;
      const uint64_t row = (uint64_t)row_i;
      const double row_y = lat_north - ((double)row + 0.5) * sp;
      double row_lat_seed = row_y;
      if (utm) {
        double mid_x = lon_west + ((double)n_cols / 2.0) * sp;
        double lo;
        xy_to_lonlat(proj, mid_x, row_y, &lo, &row_lat_seed);
      }
      int64_t prev = guess_azimuth_time(lut, row_lat_seed);
      if (utm) project_row(proj, row_y, lon_west + 0.5 * sp, sp, n_cols, (size_t)cfg->projector_anchors, rlon, rlat);
      double row_flat_area = 0.0;
      if (need_geom) {
        double mid_lon = lon_west + ((double)n_cols / 2.0) * sp;
        double ref_lon = utm ? rlon[n_cols / 2] : mid_lon;
        row_flat_area = flat_cell_area(row_lat_seed, ref_lon, step_deg);
      }
      const size_t base = (size_t)((row - row_begin) * n_cols);
      for (uint64_t col = 0; col < n_cols; ++col) {
        const size_t o = base + col;
        out_data[o] = fnan;
        if (cfg->compute_lia) { out_cos_lia[o] = fnan; out_mask[o] = SD_MASK_OUTSIDE_FOOTPRINT; }
        if (out_t_us) out_t_us[o] = INT64_MIN;
        if (out_iters) out_iters[o] = 0;
        double lon, lat;
        if (utm) { lon = rlon[col]; lat = rlat[col]; }
        else { lon = lon_west + ((double)col + 0.5) * sp; lat = row_y; }
        float hf;
        if (dem_elevation(dem, lat, lon, &hf) != 0 || !std::isfinite(hf)) {
          l_dem++;
          if (cfg->compute_lia) out_mask[o] = SD_MASK_DEM_MISSING;
          continue;
        }
        double h = (double)hf;
        double h_ell = h + geoid_undulation(*geoid, lat, lon);
        V3 target = geodetic_to_ecef(lat, lon, h_ell);
        ZdOut zd = solve_zero_doppler(target, scene->state_vectors, scene->n_state_vectors, prev,
                                      (size_t)std::max(0, cfg->max_newton_iterations), cfg->newton_tolerance_s);
        if (zd.status == ZD_ORBIT_ERROR) { orbit_error.store(1); break; }
        if (zd.status == ZD_NOT_CONVERGED) {
          l_nc++;
          if (cfg->compute_lia) out_mask[o] = SD_MASK_NON_CONVERGED;
          continue;
        }
        if (zd.status == ZD_DEGENERATE) {
          l_deg++;
          if (cfg->compute_lia) out_mask[o] = SD_MASK_DEGENERATE_GEOMETRY;
          continue;
        }
        l_hist[std::min<int>(zd.iterations, SD_NEWTON_ITER_HIST_SIZE - 1)]++;
        prev = zd.t;
        if (out_t_us) out_t_us[o] = zd.t;
        if (out_iters) out_iters[o] = (uint8_t)zd.iterations;
        double slant = norm3(sub3(target, zd.pos));
        // RadarGeometry::to_image_coords (745-762)
        double dt_s = (double)(zd.t - img->azimuth_start_time_us) / 1e6;
        double line = dt_s / ati;
        double sample = (slant - near_range_m) / rps;
        if (line < -0.5 || line > ((double)img->lines - 0.5) || sample < -0.5 ||
            sample > ((double)img->samples - 0.5)) {
          l_out++;
          if (cfg->compute_lia) out_mask[o] = SD_MASK_OUTSIDE_FOOTPRINT;
          continue;
        }
        float sigma0;
        if (cfg->resampling == SD_RESAMPLE_BICUBIC) sigma0 = bicubic_sample_slice(img->data, img->lines, img->samples, line, sample);
        else if (cfg->resampling == SD_RESAMPLE_LANCZOS3) sigma0 = lanczos_sample_slice(img->data, img->lines, img->samples, line, sample);
        else sigma0 = bilinear_sample_slice(img->data, img->lines, img->samples, line, sample);
        if (std::isnan(sigma0)) {
          l_out++;
          if (cfg->compute_lia) out_mask[o] = SD_MASK_OUTSIDE_FOOTPRINT;
          continue;
        }
        if (need_geom) {
          float he = 0.0f, hw = 0.0f, hn = 0.0f, hs = 0.0f;
          int e1 = dem_elevation(dem, lat, lon + step_deg, &he);
          int e2 = dem_elevation(dem, lat, lon - step_deg, &hw);
          int e3 = dem_elevation(dem, lat + step_deg, lon, &hn);
          int e4 = dem_elevation(dem, lat - step_deg, lon, &hs);
          bool all_finite = e1 == 0 && e2 == 0 && e3 == 0 && e4 == 0 && std::isfinite(he) &&
                            std::isfinite(hw) && std::isfinite(hn) && std::isfinite(hs);
          if (!all_finite) {
            if (cfg->compute_lia) out_mask[o] = SD_MASK_DEM_NEIGHBOUR_MISSING;
            if (cfg->flatten) { l_flat++; continue; }
          } else {
            double w = 0.0, cl = 0.0;
            int g = terrain_geometry(lat, lon, (double)he, (double)hw, (double)hn, (double)hs, zd.pos,
                                     target, step_deg, row_flat_area, &w, &cl);
            if (g == GEOM_VALID) {
              if (cfg->compute_lia) out_cos_lia[o] = (float)cl;
              if (cfg->flatten) sigma0 /= (float)w;
            } else if (g == GEOM_FORESHORTENING || g == GEOM_LAYOVER) {
              if (cfg->compute_lia) {
                out_cos_lia[o] = (float)cl;
                out_mask[o] = g == GEOM_LAYOVER ? SD_MASK_LAYOVER : SD_MASK_FORESHORTENING;
              }
              if (cfg->flatten) { l_flat++; continue; }
            } else {
              if (cfg->compute_lia) out_mask[o] = SD_MASK_SHADOW;
              if (cfg->flatten) { l_flat++; continue; }
            }
          }
        }
        if (nesz_mask) {
          float nesz = bilinear_sample_slice(img->nesz, img->lines, img->samples, line, sample);
          if (!std::isnan(nesz)) {
            float thr = nesz * nesz_factor;
            if (sigma0 <= thr) {
              l_noise++;
              if (cfg->compute_lia) out_mask[o] = SD_MASK_NOISE_MASKED;
              continue;
            }
          }
        }
        out_data[o] = sigma0;
        if (cfg->compute_lia) out_mask[o] = SD_MASK_VALID;
        l_valid++;
      }
    }
    std::lock_guard<std::mutex> lk(mu);
    c_valid += l_valid; c_dem += l_dem; c_out += l_out; c_nc += l_nc; c_deg += l_deg;
    c_flat += l_flat; c_noise += l_noise;
    for (int i = 0; i < SD_NEWTON_ITER_HIST_SIZE; ++i) hist[i] += l_hist[i];
  });
  if (orbit_error.load()) return SD_ERR_TC_ORBIT;
  info->valid_pixel_count = c_valid;
  info->dem_missing_count = c_dem;
  info->outside_footprint_count = c_out;
  info->non_converged_count = c_nc;
  info->degenerate_geometry_count = c_deg;
  info->flat_masked_count = c_flat;
  info->noise_masked_count = c_noise;
  std::memcpy(info->newton_iter_histogram, hist, sizeof(hist));
  return SD_OK;
}

int orc_terrain_correction(const sd_radar_image *img, const sd_scene *scene, const sd_dem *dem_in,
                           const sd_geoid *geoid, const sd_geo_grid_point *grid, uint64_t n_grid,
                           const sd_tc_config *cfg, uint64_t row_begin, uint64_t row_end,
                           float *out_data, float *out_cos_lia, uint8_t *out_mask,
                           int64_t *out_t_us, uint8_t *out_iters, sd_geocoded_info *info) {
  return tc_impl(img, scene, dem_in, geoid, grid, n_grid, cfg, nullptr, row_begin, row_end, out_data,
                 out_cos_lia, out_mask, out_t_us, out_iters, info);
}

// terrain_correction on an explicit output grid (west edge, north edge,
// rows, cols in the config's CRS) instead of the grid of the scene's bbox.
int orc_terrain_correction_grid(const sd_radar_image *img, const sd_scene *scene, const sd_dem *dem_in,
                                const sd_geoid *geoid, const sd_geo_grid_point *grid, uint64_t n_grid,
                                const sd_tc_config *cfg, double origin_x, double origin_y, uint64_t rows,
                                uint64_t cols, float *out_data, float *out_cos_lia, uint8_t *out_mask,
                                int64_t *out_t_us, sd_geocoded_info *info) {
  const double g[4] = {origin_x, origin_y, (double)rows, (double)cols};
  return tc_impl(img, scene, dem_in, geoid, grid, n_grid, cfg, g, 0, 0, out_data, out_cos_lia, out_mask,
                 out_t_us, nullptr, info);
}

// ── deburst (deburst.rs:172-344) ─────────────────────────────────────────
int orc_compute_overlap_lines(const sd_burst *bk, const sd_burst *bk1, double ati, uint64_t lps,
                              int64_t *overlap) {
  int64_t dt_us = bk1->azimuth_time_us - bk->azimuth_time_us;
  double dt_s = (double)dt_us * 1e-6;
  int64_t step_lines = f64_as_i64(std::round(dt_s / ati));
  int64_t ov = (int64_t)lps - step_lines;
  *overlap = ov;
  if (ov <= 0) return SD_ERR_DEBURST_INVALID_OVERLAP;
  if (ov < 50 || ov > 400) return SD_ERR_DEBURST_IMPLAUSIBLE_OVERLAP;
  return SD_OK;
}

int orc_deburst_plan(const sd_subswath *sw, const sd_burst *bursts, uint64_t n, uint64_t tiff_height,
                     uint64_t *lines, uint64_t *samples, uint64_t *offset, uint64_t *first_out,
                     uint64_t *end_out) {
  if (n == 0) return SD_ERR_DEBURST_NO_BURSTS;
  if (n != sw->burst_count) return SD_ERR_DEBURST_BURST_COUNT_MISMATCH;
  uint64_t lps = sw->lines_per_burst;
  if (tiff_height < n * lps) return SD_ERR_DEBURST_TIFF_TOO_SMALL;
  uint64_t fv = 0, lv = UINT64_MAX;
  for (uint64_t i = 0; i < n; ++i) {
    fv = std::max<uint64_t>(fv, bursts[i].first_valid_sample);
    lv = std::min<uint64_t>(lv, bursts[i].last_valid_sample);
  }
  if (fv >= lv) return SD_ERR_DEBURST_EMPTY_VALID_WINDOW;
  std::vector<uint64_t> ovs;
  for (uint64_t k = 0; k + 1 < n; ++k) {
    int64_t ov;
    int rc = orc_compute_overlap_lines(&bursts[k], &bursts[k + 1], sw->azimuth_time_interval_s, lps, &ov);
    if (rc != SD_OK) return rc;
    ovs.push_back((uint64_t)ov);
  }
  uint64_t total = 0;
  for (uint64_t k = 0; k < n; ++k) {
    uint64_t lf = k == 0 ? 0 : (ovs[k - 1] + 1) / 2;
    uint64_t le = k == n - 1 ? lps : lps - ovs[k] / 2;
    if (first_out) first_out[k] = lf;
    if (end_out) end_out[k] = le;
    total += le - lf;
  }
  *lines = total;
  *samples = lv - fv;
  *offset = fv;
  return SD_OK;
}

int orc_deburst_subswath(const int16_t *slc, uint64_t tiff_width, uint64_t tiff_height,
                         const sd_subswath *sw, const sd_burst *bursts, uint64_t n, int16_t *out) {
  uint64_t lines, samples, off;
  std::vector<uint64_t> lf(n), le(n);
  int rc = orc_deburst_plan(sw, bursts, n, tiff_height, &lines, &samples, &off, lf.data(), le.data());
  if (rc != SD_OK) return rc;
  uint64_t out_line = 0;
  for (uint64_t k = 0; k < n; ++k) {
    uint64_t nl = le[k] - lf[k];
    uint64_t tiff_first = bursts[k].first_line + lf[k];
    for (uint64_t l = 0; l < nl; ++l) {
      const int16_t *src = slc + ((tiff_first + l) * tiff_width + off) * 2;
      std::memcpy(out + (out_line + l) * samples * 2, src, samples * 2 * sizeof(int16_t));
    }
    out_line += nl;
  }
  return SD_OK;
}

// ── calibration (apply_calibration.rs:128-572) ───────────────────────────
namespace {
inline float lerp(float a, float b, float t) {
  t = clamp_f32(t, 0.0f, 1.0f);
  return a + (b - a) * t;
}
void bracket_azimuth(const std::vector<int64_t> &lines, int64_t tl, size_t *lo, size_t *hi) {
  size_t a = 0, b = lines.size();
  while (a < b) {
    size_t mid = a + (b - a) / 2;
    if (lines[mid] < tl) a = mid + 1;
    else if (lines[mid] > tl) b = mid;
    else { *lo = *hi = mid; return; }
  }
  if (a == 0) { *lo = *hi = 0; return; }
  if (a >= lines.size()) { *lo = *hi = lines.size() - 1; return; }
  *lo = a - 1;
  *hi = a;
}
inline float lut_cursor_eval(const uint32_t *px, const float *v, size_t n, size_t cur, uint32_t col) {
  if (px[cur] > col) return v[0];
  if (cur + 1 < n) {
    float t = (float)(col - px[cur]) / (float)(px[cur + 1] - px[cur]);
    return lerp(v[cur], v[cur + 1], t);
  }
  return v[cur];
}
void bilinear_row_into(const sd_lut_vector *vecs, const std::vector<int64_t> &lines, int64_t tl,
                       size_t col_offset, float *buf, size_t n_cols) {
  size_t lo, hi;
  bracket_azimuth(lines, tl, &lo, &hi);
  const sd_lut_vector &L = vecs[lo];
  size_t cur_lo = 0;
  if (lo == hi) {
    for (size_t c = 0; c < n_cols; ++c) {
      uint32_t col = (uint32_t)(c + col_offset);
      while (cur_lo + 1 < L.n && L.pixels[cur_lo + 1] <= col) cur_lo++;
      buf[c] = lut_cursor_eval(L.pixels, L.values, L.n, cur_lo, col);
    }
  } else {
    float t_line = (float)(tl - lines[lo]) / (float)(lines[hi] - lines[lo]);
    const sd_lut_vector &H = vecs[hi];
    size_t cur_hi = 0;
    for (size_t c = 0; c < n_cols; ++c) {
      uint32_t col = (uint32_t)(c + col_offset);
      while (cur_lo + 1 < L.n && L.pixels[cur_lo + 1] <= col) cur_lo++;
      while (cur_hi + 1 < H.n && H.pixels[cur_hi + 1] <= col) cur_hi++;
      float vl = lut_cursor_eval(L.pixels, L.values, L.n, cur_lo, col);
      float vh = lut_cursor_eval(H.pixels, H.values, H.n, cur_hi, col);
      buf[c] = lerp(vl, vh, t_line);
    }
  }
}
}  // namespace

int orc_apply_calibration(const int16_t *iq, uint64_t lines, uint64_t samples, uint64_t col_offset,
                          const sd_lut_vector *cal, uint64_t n_cal, const sd_lut_vector *nr,
                          uint64_t n_nr, const sd_noise_azimuth *az, uint64_t tiff_line_origin,
                          float *out, float *nesz, uint32_t *cal_gap, uint32_t *noise_gap) {
  if (n_cal == 0) return SD_ERR_CAL_NO_CALIBRATION_VECTORS;
  if (n_nr == 0) return SD_ERR_CAL_NO_NOISE_RANGE_VECTORS;
  const uint32_t SLACK = 600;
  uint64_t req64 = col_offset + samples;
  uint32_t required_last = (uint32_t)(req64 == 0 ? 0 : req64 - 1);
  uint32_t max_cal_gap = 0, max_nr_gap = 0;
  for (uint64_t i = 0; i < n_cal; ++i) {
    if (cal[i].n == 0) return SD_ERR_CAL_NO_CALIBRATION_VECTORS;
    uint32_t m = cal[i].pixels[cal[i].n - 1];
    if (m < required_last) {
      uint32_t gap = required_last - m;
      if (gap > SLACK) return SD_ERR_CAL_LUT_RANGE_INSUFFICIENT;
      max_cal_gap = std::max(max_cal_gap, gap);
    }
  }
  for (uint64_t i = 0; i < n_nr; ++i) {
    if (nr[i].n == 0) return SD_ERR_CAL_NO_NOISE_RANGE_VECTORS;
    uint32_t m = nr[i].pixels[nr[i].n - 1];
    if (m < required_last) {
      uint32_t gap = required_last - m;
      if (gap > SLACK) return SD_ERR_CAL_LUT_RANGE_INSUFFICIENT;
      max_nr_gap = std::max(max_nr_gap, gap);
    }
  }
  *cal_gap = max_cal_gap;
  *noise_gap = max_nr_gap;
  std::vector<int64_t> cal_lines(n_cal), nr_lines(n_nr), az_lines;
  for (uint64_t i = 0; i < n_cal; ++i) cal_lines[i] = cal[i].line;
  for (uint64_t i = 0; i < n_nr; ++i) nr_lines[i] = nr[i].line;
  bool az_avail = az != nullptr && az->n > 0;
  if (az_avail)
    for (uint64_t i = 0; i < az->n; ++i) az_lines.push_back(az->lines[i]);
  parallel_for((int64_t)lines, 64, [&](int64_t lb, int64_t le, int) {
    std::vector<float> k_row(samples), nr_row(samples);
    for (int64_t ol = lb; ol < le; ++ol) {
      int64_t tl = (int64_t)(tiff_line_origin + (uint64_t)ol);
      bilinear_row_into(cal, cal_lines, tl, col_offset, k_row.data(), samples);
      bilinear_row_into(nr, nr_lines, tl, col_offset, nr_row.data(), samples);
      float az_factor = 1.0f;
      if (az_avail && !az_lines.empty()) {
        size_t lo, hi;
        bracket_azimuth(az_lines, tl, &lo, &hi);
        if (az_lines[hi] == az_lines[lo]) az_factor = az->values[lo];
        else {
          float t = (float)(tl - az_lines[lo]) / (float)(az_lines[hi] - az_lines[lo]);
          az_factor = lerp(az->values[lo], az->values[hi], t);
        }
      }
      const int16_t *row = iq + (size_t)ol * samples * 2;
      float *o = out + (size_t)ol * samples;
      float *nz = nesz + (size_t)ol * samples;
      for (uint64_t c = 0; c < samples; ++c) {
        int32_t i = row[2 * c], q = row[2 * c + 1];
        // i32 arithmetic wraps in release builds; do it in u32 to match.
        float power = (float)(int32_t)((uint32_t)(i * i) + (uint32_t)(q * q));
        float k = k_row[c];
        float k2 = k * k;
        float valid = (k2 > 0.0f) ? 1.0f : 0.0f;
        float inv_k2 = (k2 > 0.0f) ? 1.0f / k2 : 0.0f;
        float noise_val = nr_row[c] * az_factor;
        o[c] = max_f32(power - noise_val, 0.0f) * inv_k2 * valid;
        nz[c] = noise_val * inv_k2 * valid;
      }
    }
  });
  return SD_OK;
}

// ── merge (merge_subswaths.rs:207-450) ───────────────────────────────────
int orc_merge_plan(int32_t n, const uint64_t *lines, const uint64_t *samples, const uint64_t *voff,
                   const sd_subswath *sw, const int64_t *az_start, sd_merged_info *info) {
  std::memset(info, 0, sizeof(*info));
  if (n <= 0) return SD_ERR_MERGE_EMPTY_INPUTS;
  if (n > 8) return SD_ERR_INVALID_ARGUMENT;
  info->n_swaths = n;
  if (n == 1) {
    if (samples[0] == 0) return SD_ERR_MERGE_EMPTY_SWATH;
    double rps = sw[0].range_pixel_spacing_m;
    double dt = rps * 2.0 / SPEED_OF_LIGHT;
    info->lines = lines[0];
    info->samples = samples[0];
    info->near_slant_range_time_s = sw[0].slant_range_time_s + (double)voff[0] * dt;
    info->range_pixel_spacing_s = dt;
    info->range_pixel_spacing_m = rps;
    info->azimuth_start_time_us = az_start[0];
    info->swath_out_offset[0] = 0;
    info->swath_seam[0] = samples[0];
    info->swath_lines[0] = lines[0];
    info->swath_valid_offset[0] = voff[0];
    return SD_OK;
  }
  double rps = sw[0].range_pixel_spacing_m;
  for (int32_t i = 1; i < n; ++i)
    if (std::fabs(sw[i].range_pixel_spacing_m - rps) > 1e-3) return SD_ERR_MERGE_INCONSISTENT_PIXEL_SPACING;
  for (int32_t i = 0; i < n; ++i)
    if (samples[i] == 0) return SD_ERR_MERGE_EMPTY_SWATH;
  double dt = rps * 2.0 / SPEED_OF_LIGHT;
  std::vector<double> st(n);
  for (int32_t i = 0; i < n; ++i) st[i] = sw[i].slant_range_time_s + (double)voff[i] * dt;
  double t0 = st[0];
  std::vector<int64_t> offs(n), ends(n);
  for (int32_t i = 0; i < n; ++i) {
    offs[i] = f64_as_i64(std::round((st[i] - t0) / dt));
    ends[i] = offs[i] + (int64_t)samples[i];
  }
  uint64_t out_cols = (uint64_t)ends[n - 1];
  uint64_t out_lines = UINT64_MAX;
  for (int32_t i = 0; i < n; ++i) out_lines = std::min(out_lines, lines[i]);
  int64_t azmin = az_start[0];
  for (int32_t i = 1; i < n; ++i) azmin = std::min(azmin, az_start[i]);
  info->lines = out_lines;
  info->samples = out_cols;
  info->near_slant_range_time_s = t0;
  info->range_pixel_spacing_s = dt;
  info->range_pixel_spacing_m = rps;
  info->azimuth_start_time_us = azmin;
  for (int32_t i = 0; i < n; ++i) {
    info->swath_out_offset[i] = offs[i];
    info->swath_lines[i] = lines[i];
    info->swath_valid_offset[i] = voff[i];
    info->swath_seam[i] = (i + 1 < n) ? (uint64_t)((ends[i] + offs[i + 1]) / 2) : out_cols;
  }
  return SD_OK;
}

int orc_merge_subswaths(int32_t n, const float *const *sig, const float *const *nesz,
                        const uint64_t *lines, const uint64_t *samples, const uint64_t *voff,
                        const uint32_t *cal_gap, const uint32_t *noise_gap, const sd_subswath *sw,
                        const int64_t *az_start, float *out, float *out_nesz, sd_merged_info *info) {
  int rc = orc_merge_plan(n, lines, samples, voff, sw, az_start, info);
  if (rc != SD_OK) return rc;
  uint32_t cg = 0, ng = 0;
  for (int32_t i = 0; i < n; ++i) { cg = std::max(cg, cal_gap[i]); ng = std::max(ng, noise_gap[i]); }
  info->cal_lut_extrapolation_gap_px = cg;
  info->noise_lut_extrapolation_gap_px = ng;
  if (!out) return SD_OK;
  const uint64_t out_lines = info->lines, out_cols = info->samples;
  const float fnan = std::numeric_limits<float>::quiet_NaN();
  if (n == 1) {
    std::memcpy(out, sig[0], out_lines * out_cols * sizeof(float));
    std::memcpy(out_nesz, nesz[0], out_lines * out_cols * sizeof(float));
    return SD_OK;
  }
  struct FR { uint64_t col_start, col_end, vs, ve, in_start; };
  std::vector<FR> fr(n);
  for (int32_t i = 0; i < n; ++i) {
    uint64_t cs = i == 0 ? 0 : info->swath_seam[i - 1];
    uint64_t ce = i == n - 1 ? out_cols : info->swath_seam[i];
    uint64_t off = (uint64_t)info->swath_out_offset[i];
    uint64_t vs = std::max(cs, off);
    uint64_t ve = std::min(ce, off + samples[i]);
    uint64_t in_start = vs >= off ? vs - off : 0;
    fr[i] = {cs, ce, vs, ve, in_start};
  }
  parallel_for((int64_t)out_lines, 64, [&](int64_t lb, int64_t lend, int) {
  for (int64_t l = lb; l < lend; ++l) {
    float *orow = out + (size_t)l * out_cols;
    float *nrow = out_nesz + (size_t)l * out_cols;
    uint64_t fill_end = 0;
    for (int32_t i = 0; i < n; ++i) {
      const FR &f = fr[i];
      for (uint64_t c = fill_end; c < f.vs; ++c) { orow[c] = fnan; nrow[c] = fnan; }
      if (f.vs < f.ve) {
        size_t b = (size_t)l * samples[i] + f.in_start;
        std::memcpy(orow + f.vs, sig[i] + b, (f.ve - f.vs) * sizeof(float));
        std::memcpy(nrow + f.vs, nesz[i] + b, (f.ve - f.vs) * sizeof(float));
      }
      for (uint64_t c = f.ve; c < f.col_end; ++c) { orow[c] = fnan; nrow[c] = fnan; }
      fill_end = f.col_end;
    }
    for (uint64_t c = fill_end; c < out_cols; ++c) { orow[c] = fnan; nrow[c] = fnan; }
  }
  });
  return SD_OK;
}

// ── speckle (speckle.rs:131-569) ─────────────────────────────────────────
namespace {
struct WStats { bool ok; float mean, var; };
inline WStats window_mean_var(const float *d, int64_t cols, int64_t rows, int64_t r, int64_t c, int half) {
  double sum = 0.0, sum_sq = 0.0;
  size_t n = 0;
  for (int dy = -half; dy <= half; ++dy)
    for (int dx = -half; dx <= half; ++dx) {
      int64_t rr = r + dy, cc = c + dx;
      if (rr < 0 || cc < 0 || rr >= rows || cc >= cols) continue;
      float v = d[rr * cols + cc];
      if (!std::isfinite(v)) continue;
      double vd = (double)v;
      sum += vd;
      sum_sq += vd * vd;
      n++;
    }
  if (n == 0) return {false, 0.0f, 0.0f};
  double mean = sum / (double)n;
  double var = max_f64(sum_sq / (double)n - mean * mean, 0.0);
  return {true, (float)mean, (float)var};
}
inline bool rl_in_mask(int dir, int dy, int dx) {
  if (dy == 0 && dx == 0) return false;
  switch (dir) {
    case 0: return dy >= 1 && dy <= 3;
    case 1: return dy >= -3 && dy <= -1;
    case 2: return dx >= 1 && dx <= 3;
    case 3: return dx >= -3 && dx <= -1;
    case 4: return std::abs(dy - dx) <= 1 && (dy + dx) >= 1;
    case 5: return std::abs(dy - dx) <= 1 && (dy + dx) <= -1;
    case 6: return std::abs(dy + dx) <= 1 && (dx - dy) >= 1;
    case 7: return std::abs(dy + dx) <= 1 && (dx - dy) <= -1;
  }
  return false;
}
}  // namespace

int orc_speckle(const float *d, uint64_t len, uint64_t cols_u, uint64_t rows_u, int kind,
                uint64_t window, float enl, float damping, float *out) {
  if (cols_u != 0 && rows_u > UINT64_MAX / cols_u) return SD_ERR_SPECKLE_DIMENSION_MISMATCH;
  if (len != cols_u * rows_u) return SD_ERR_SPECKLE_DIMENSION_MISMATCH;
  uint64_t win = kind == SD_SPECKLE_REFINED_LEE ? 7 : window;
  if (win < 3 || win % 2 == 0) return SD_ERR_SPECKLE_BAD_WINDOW;
  if (kind == SD_SPECKLE_LEE || kind == SD_SPECKLE_GAMMA_MAP || kind == SD_SPECKLE_REFINED_LEE) {
    if (!(enl > 0.0f) || !std::isfinite(enl)) return SD_ERR_SPECKLE_BAD_ENL;
  }
  if (kind == SD_SPECKLE_FROST) {
    if (!std::isfinite(damping) || damping < 0.0f) return SD_ERR_SPECKLE_BAD_DAMPING;
  }
  const int64_t cols = (int64_t)cols_u, rows = (int64_t)rows_u;
  const int half = (int)(win / 2);
  const float fnan = std::numeric_limits<float>::quiet_NaN();
  const float cv_n_sq = 1.0f / enl;
  const float cv_max_sq = cv_n_sq < 1.0f ? 2.0f * cv_n_sq / (1.0f - cv_n_sq) : INFINITY;
  parallel_for(rows, 4, [&](int64_t rb, int64_t rend, int) {
  for (int64_t r = rb; r < rend; ++r) {
    for (int64_t c = 0; c < cols; ++c) {
      float &o = out[r * cols + c];
      o = fnan;
      float centre = d[r * cols + c];
      if (!std::isfinite(centre)) continue;
      if (kind == SD_SPECKLE_REFINED_LEE) {
        float best_cv = INFINITY, best_mean = centre, best_var = 0.0f;
        for (int dir = 0; dir < 8; ++dir) {
          double sum = 0.0, sum_sq = 0.0;
          size_t n = 0;
          for (int dy = -3; dy <= 3; ++dy)
            for (int dx = -3; dx <= 3; ++dx) {
              if (!rl_in_mask(dir, dy, dx)) continue;
              int64_t rr = r + dy, cc = c + dx;
              if (rr < 0 || cc < 0 || rr >= rows || cc >= cols) continue;
              float v = d[rr * cols + cc];
              if (!std::isfinite(v)) continue;
              double vd = (double)v;
              sum += vd;
              sum_sq += vd * vd;
              n++;
            }
          if (n == 0) continue;
          double meand = sum / (double)n;
          double vard = max_f64(sum_sq / (double)n - meand * meand, 0.0);
          float mean = (float)meand, var = (float)vard;
          if (!(mean > 0.0f)) continue;
          float cv = var / (mean * mean);
          if (cv < best_cv) { best_cv = cv; best_mean = mean; best_var = var; }
        }
        if (!std::isfinite(best_cv)) { o = centre; continue; }
        float noise_var = best_mean * best_mean * cv_n_sq;
        float signal_var = max_f32(best_var - noise_var, 0.0f);
        float denom = signal_var + noise_var;
        float k = denom > 0.0f ? signal_var / denom : 0.0f;
        o = best_mean + k * (centre - best_mean);
        continue;
      }
      WStats s = window_mean_var(d, cols, rows, r, c, half);
      if (!s.ok) continue;
      float mean = s.mean, var = s.var;
      if (kind == SD_SPECKLE_BOXCAR) {
        o = mean;
      } else if (kind == SD_SPECKLE_LEE) {
        float noise_var = mean * mean * cv_n_sq;
        float signal_var = max_f32(var - noise_var, 0.0f);
        float denom = signal_var + noise_var;
        float k = denom > 0.0f ? signal_var / denom : 0.0f;
        o = mean + k * (centre - mean);
      } else if (kind == SD_SPECKLE_FROST) {
        float cv_sq = mean > 0.0f ? var / (mean * mean) : 0.0f;
        float alpha = damping * cv_sq;
        double wsum = 0.0, vwsum = 0.0;
        for (int dy = -half; dy <= half; ++dy)
          for (int dx = -half; dx <= half; ++dx) {
            int64_t rr = r + dy, cc = c + dx;
            if (rr < 0 || cc < 0 || rr >= rows || cc >= cols) continue;
            float v = d[rr * cols + cc];
            if (!std::isfinite(v)) continue;
            float dd = (float)(std::abs(dy) + std::abs(dx));
            double w = (double)std::exp(-alpha * dd);
            wsum += w;
            vwsum += w * (double)v;
          }
        if (wsum > 0.0) o = (float)(vwsum / wsum);
      } else {  // gamma map
        float cv_sq = mean > 0.0f ? var / (mean * mean) : 0.0f;
        if (cv_sq <= cv_n_sq) { o = mean; continue; }
        if (cv_sq >= cv_max_sq) { o = centre; continue; }
        float alpha = (1.0f + cv_n_sq) / (cv_sq - cv_n_sq);
        float b = (alpha - enl - 1.0f) * mean;
        float disc = b * b + 4.0f * alpha * enl * mean * centre;
        o = disc >= 0.0f ? ((enl - alpha + 1.0f) * mean + std::sqrt(disc)) / (2.0f * enl) : mean;
      }
    }
  }
  });
  return SD_OK;
}

}  // extern "C"
