// geo.cuh — geometry primitives of the terrain correction, written once for
// host and device.  Every function reproduces the reference's arithmetic
// operation by operation (IEEE f64/f32, left-to-right, no contraction: the
// library is compiled with --fmad=false), so that integer outcomes (masks,
// microsecond azimuth times, iteration counts) match the reference.
//
// Reference files: sardine/src/geodesy.rs, orbit.rs, dem.rs, geoid.rs,
// terrain_correction.rs, output_crs.rs.
#pragma once

#include <cmath>
#include <cstdint>

#include "../../include/sardine_b200.h"
#include "crmath.cuh"

#if defined(__CUDACC__)
#define SD_HD __host__ __device__ __forceinline__
#define SD_HD_COLD static __host__ __device__ __noinline__  // rare paths, kept out of line
#else
#define SD_HD inline
#define SD_HD_COLD inline
#endif

namespace sd {

constexpr double kPi = 3.14159265358979323846;  // std::f64::consts::PI
constexpr double WGS84_A = 6378137.0;           // geodesy.rs:13
constexpr double WGS84_F = 1.0 / 298.257223563; // geodesy.rs:16
constexpr double WGS84_E2 = 2.0 * WGS84_F - WGS84_F * WGS84_F;  // geodesy.rs:22
constexpr double SPEED_OF_LIGHT = 299792458.0;  // types.rs:11

// Rust `x as i64` (saturating, NaN -> 0).
SD_HD int64_t f2i64(double x) {
  if (x != x) return 0;
  if (x >= 9223372036854775807.0) return INT64_MAX;
  if (x <= -9223372036854775808.0) return INT64_MIN;
  return (int64_t)x;
}
// Rust `x as usize` (saturating at 0).
SD_HD uint64_t f2u64(double x) {
  if (x != x || x <= 0.0) return 0;
  if (x >= 18446744073709551615.0) return UINT64_MAX;
  return (uint64_t)x;
}
SD_HD double clampd(double x, double lo, double hi) {
  if (x < lo) x = lo;
  if (x > hi) x = hi;
  return x;
}
SD_HD int64_t clampi(int64_t x, int64_t lo, int64_t hi) { return x < lo ? lo : (x > hi ? hi : x); }
SD_HD float maxf_nan(float a, float b) {  // f32::max
  return (a != a) ? b : ((b != b) ? a : (a > b ? a : b));
}
SD_HD double maxd_nan(double a, double b) {
  return (a != a) ? b : ((b != b) ? a : (a > b ? a : b));
}

struct V3 {
  double x, y, z;
};
SD_HD double dot3(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
SD_HD double norm3(V3 v) { return sqrt(dot3(v, v)); }
SD_HD V3 sub3(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
SD_HD V3 cross3(V3 a, V3 b) {
  return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
SD_HD V3 normalize3(V3 v) {
  double n = norm3(v);
  if (n == 0.0) return {0.0, 0.0, 0.0};
  return {v.x / n, v.y / n, v.z / n};
}

// geodetic_to_ecef (geodesy.rs:38-55), with correctly rounded sines and
// cosines (crmath.cuh): equal to the reference's wherever its libm rounds
// correctly.
SD_HD V3 geodetic_to_ecef(double lat_deg, double lon_deg, double h) {
  double lat = lat_deg * kPi / 180.0;
  double lon = lon_deg * kPi / 180.0;
  double sin_lat, cos_lat, sin_lon, cos_lon;
  crm::sincos(lat, &sin_lat, &cos_lat);
  crm::sincos(lon, &sin_lon, &cos_lon);
  double n = WGS84_A / sqrt(1.0 - WGS84_E2 * sin_lat * sin_lat);
  return {(n + h) * cos_lat * cos_lon, (n + h) * cos_lat * sin_lon,
          (n * (1.0 - WGS84_E2) + h) * sin_lat};
}

// ── UTM: transverse Mercator by Krueger's n-series to sixth order, as given
// by C. F. F. Karney (2011), J. Geodesy 85:475-485, eqs. 7-11, 14, 19-21, 35,
// 36.  (The reference delegates UTM to the proj4rs crate.)
struct Utm {
  int32_t zone;
  int32_t south;
  double lon0;  // central meridian, radians
  double k0A;
  double e, e2m;
  double alp[7], bet[7];
};

inline Utm make_utm(int zone, bool south) {
  Utm u{};
  u.zone = zone;
  u.south = south ? 1 : 0;
  u.lon0 = (double)((zone - 1) * 6 - 180 + 3) * (kPi / 180.0);
  const double f = WGS84_F;
  const double n = f / (2.0 - f);
  const double n2 = n * n, n3 = n2 * n, n4 = n3 * n, n5 = n4 * n, n6 = n5 * n;
  const double A = WGS84_A / (1.0 + n) * (1.0 + n2 / 4.0 + n4 / 64.0 + n6 / 256.0);
  u.k0A = 0.9996 * A;
  u.e = std::sqrt(f * (2.0 - f));
  u.e2m = 1.0 - f * (2.0 - f);
  u.alp[0] = 0.0;
  u.alp[1] = n / 2.0 - 2.0 * n2 / 3.0 + 5.0 * n3 / 16.0 + 41.0 * n4 / 180.0 - 127.0 * n5 / 288.0 + 7891.0 * n6 / 37800.0;
  u.alp[2] = 13.0 * n2 / 48.0 - 3.0 * n3 / 5.0 + 557.0 * n4 / 1440.0 + 281.0 * n5 / 630.0 - 1983433.0 * n6 / 1935360.0;
  u.alp[3] = 61.0 * n3 / 240.0 - 103.0 * n4 / 140.0 + 15061.0 * n5 / 26880.0 + 167603.0 * n6 / 181440.0;
  u.alp[4] = 49561.0 * n4 / 161280.0 - 179.0 * n5 / 168.0 + 6601661.0 * n6 / 7257600.0;
  u.alp[5] = 34729.0 * n5 / 80640.0 - 3418889.0 * n6 / 1995840.0;
  u.alp[6] = 212378941.0 * n6 / 319334400.0;
  u.bet[0] = 0.0;
  u.bet[1] = n / 2.0 - 2.0 * n2 / 3.0 + 37.0 * n3 / 96.0 - n4 / 360.0 - 81.0 * n5 / 512.0 + 96199.0 * n6 / 604800.0;
  u.bet[2] = n2 / 48.0 + n3 / 15.0 - 437.0 * n4 / 1440.0 + 46.0 * n5 / 105.0 - 1118711.0 * n6 / 3870720.0;
  u.bet[3] = 17.0 * n3 / 480.0 - 37.0 * n4 / 840.0 - 209.0 * n5 / 4480.0 + 5569.0 * n6 / 90720.0;
  u.bet[4] = 4397.0 * n4 / 161280.0 - 11.0 * n5 / 504.0 - 830251.0 * n6 / 7257600.0;
  u.bet[5] = 4583.0 * n5 / 161280.0 - 108847.0 * n6 / 3991680.0;
  u.bet[6] = 20648693.0 * n6 / 638668800.0;
  return u;
}

SD_HD double adjlon(double lam) {
  while (lam > kPi) lam -= 2.0 * kPi;
  while (lam < -kPi) lam += 2.0 * kPi;
  return lam;
}

// The exact forward and inverse transforms take their elementary functions
// from crmath.cuh, the arithmetic the oracle's restatement uses for them.
// sum_{j=1..6} c[j] sin(2 j zeta), zeta = xi + i eta  (complex Chebyshev recurrence)
SD_HD void krueger_sum(const double *c, double xi, double eta, double *re, double *im) {
  double s1, c1;
  crm::sincos(2.0 * xi, &s1, &c1);
  double sh1 = crm::sinh(2.0 * eta), ch1 = crm::cosh(2.0 * eta);
  double sr = s1 * ch1, si = c1 * sh1;
  double cr = c1 * ch1, ci = -s1 * sh1;
  double pr = 0.0, pi = 0.0, qr = sr, qi = si, ar = 0.0, ai = 0.0;
  for (int j = 1; j <= 6; ++j) {
    ar += c[j] * qr;
    ai += c[j] * qi;
    double nr = 2.0 * (cr * qr - ci * qi) - pr;
    double ni = 2.0 * (cr * qi + ci * qr) - pi;
    pr = qr; pi = qi; qr = nr; qi = ni;
  }
  *re = ar;
  *im = ai;
}

SD_HD double taupf(double tau, double e) {
  double tau1 = crm::hypot(1.0, tau);
  double sig = crm::sinh(e * crm::atanh(e * tau / tau1));
  return crm::hypot(1.0, sig) * tau - sig * tau1;
}

SD_HD double tauf(double taup, double e, double e2m) {
  double tau = taup / e2m;
  for (int i = 0; i < 6; ++i) {
    double taupa = taupf(tau, e);
    double dtau = (taup - taupa) * (1.0 + e2m * tau * tau) / (e2m * crm::hypot(1.0, tau) * crm::hypot(1.0, taupa));
    tau += dtau;
    double lim = fabs(tau) > 1.0 ? fabs(tau) : 1.0;
    if (!(fabs(dtau) >= 1e-15 * lim)) break;
  }
  return tau;
}

// lon/lat in degrees -> easting/northing (Projector::lonlat_to_xy, output_crs.rs:301-315)
SD_HD void utm_lonlat_to_xy(const Utm &u, double lon_deg, double lat_deg, double *x, double *y) {
  double lam = adjlon(lon_deg * (kPi / 180.0) - u.lon0);
  double tau = crm::tan(lat_deg * (kPi / 180.0));
  double taup = taupf(tau, u.e);
  double sl, cl;
  crm::sincos(lam, &sl, &cl);
  double xip = crm::atan2(taup, cl);
  double etap = crm::asinh(sl / crm::hypot(taup, cl));
  double sr, si;
  krueger_sum(u.alp, xip, etap, &sr, &si);
  *x = 500000.0 + u.k0A * (etap + si);
  *y = (u.south ? 10000000.0 : 0.0) + u.k0A * (xip + sr);
}

// easting/northing -> lon/lat in degrees (Projector::xy_to_lonlat, output_crs.rs:318-340)
SD_HD void utm_xy_to_lonlat(const Utm &u, double x, double y, double *lon_deg, double *lat_deg) {
  double xi = (y - (u.south ? 10000000.0 : 0.0)) / u.k0A;
  double eta = (x - 500000.0) / u.k0A;
  double sr, si;
  krueger_sum(u.bet, xi, eta, &sr, &si);
  double xip = xi - sr, etap = eta - si;
  double sx, c;
  crm::sincos(xip, &sx, &c);
  double s = crm::sinh(etap);
  double taup = sx / crm::hypot(s, c);
  double tau = tauf(taup, u.e, u.e2m);
  *lat_deg = crm::atan(tau) * (180.0 / kPi);
  *lon_deg = adjlon(crm::atan2(s, c) + u.lon0) * (180.0 / kPi);
}

// The forward projection split into its latitude-only and longitude-only
// parts, so lookups that share a latitude or a longitude share that work.
// utm_xy_from(u, utm_taup(u, lat), utm_lam(u, lon)) performs exactly the
// operations of utm_lonlat_to_xy(u, lon, lat).
SD_HD double utm_taup(const Utm &u, double lat_deg) { return taupf(tan(lat_deg * (kPi / 180.0)), u.e); }
struct LamSC {
  double s, c;
};
SD_HD LamSC utm_lam(const Utm &u, double lon_deg) {
  double lam = adjlon(lon_deg * (kPi / 180.0) - u.lon0);
  return {sin(lam), cos(lam)};
}
SD_HD void utm_xy_from(const Utm &u, double taup, LamSC L, double *x, double *y) {
  double xip = atan2(taup, L.c);
  double etap = asinh(L.s / hypot(taup, L.c));
  double sr, si;
  krueger_sum(u.alp, xip, etap, &sr, &si);
  *x = 500000.0 + u.k0A * (etap + si);
  *y = (u.south ? 10000000.0 : 0.0) + u.k0A * (xip + sr);
}

// Local expansion of the forward projection around one point, for lookups a
// few metres away (the four cardinal DEM neighbours of an output pixel).
// With w = psi + i*lam (isometric latitude, longitude) the spherical step is
// zeta' = gd(w), so d zeta'/dw = cos(zeta') and d2 zeta'/dw2 =
// -cos(zeta') sin(zeta'); the Krueger series adds d zeta/d zeta' =
// 1 + sum 2j a_j cos(2j zeta') and d2 zeta/d zeta'2 = -sum 4j^2 a_j sin(2j zeta').
// A second-order step of |dw| ~ 2e-6 is exact to ~3e-11 m (the third-order
// term), below the rounding of the projected coordinates themselves.
struct UtmLocal {
  double x, y;             // projected point
  double zw_re, zw_im;     // d zeta / dw
  double zww_re, zww_im;   // d2 zeta / dw2
  double dpsi1, dpsi2;     // d psi/d phi, d2 psi/d phi2 (phi in radians)
};

SD_HD void utm_local(const Utm &u, double lat_deg, double taup, LamSC L, UtmLocal *o) {
  const double xip = atan2(taup, L.c);
  const double etap = asinh(L.s / hypot(taup, L.c));
  // sin/cos of zeta' and of 2 zeta'
  const double sx = sin(xip), cx = cos(xip);
  const double ex = exp(etap), emx = 1.0 / ex;
  const double sh = 0.5 * (ex - emx), ch = 0.5 * (ex + emx);
  const double s_re = sx * ch, s_im = cx * sh;    // sin(zeta')
  const double c_re = cx * ch, c_im = -sx * sh;   // cos(zeta')
  const double s2_re = 2.0 * (s_re * c_re - s_im * c_im), s2_im = 2.0 * (s_re * c_im + s_im * c_re);
  const double c2_re = c_re * c_re - c_im * c_im - (s_re * s_re - s_im * s_im);
  const double c2_im = 2.0 * (c_re * c_im - s_re * s_im);
  // Chebyshev recurrences for sin(2j z) and cos(2j z): S = sum a_j sin(2jz),
  // D1 = sum 2j a_j cos(2jz), D2 = sum 4j^2 a_j sin(2jz)
  double ps_re = 0.0, ps_im = 0.0, qs_re = s2_re, qs_im = s2_im;   // sin(0), sin(2z)
  double pc_re = 1.0, pc_im = 0.0, qc_re = c2_re, qc_im = c2_im;   // cos(0), cos(2z)
  double S_re = 0.0, S_im = 0.0, D1_re = 0.0, D1_im = 0.0, D2_re = 0.0, D2_im = 0.0;
  for (int j = 1; j <= 6; ++j) {
    const double a = u.alp[j];
    S_re += a * qs_re;
    S_im += a * qs_im;
    D1_re += 2.0 * j * a * qc_re;
    D1_im += 2.0 * j * a * qc_im;
    D2_re += 4.0 * j * j * a * qs_re;
    D2_im += 4.0 * j * j * a * qs_im;
    const double ns_re = 2.0 * (c2_re * qs_re - c2_im * qs_im) - ps_re;
    const double ns_im = 2.0 * (c2_re * qs_im + c2_im * qs_re) - ps_im;
    const double nc_re = 2.0 * (c2_re * qc_re - c2_im * qc_im) - pc_re;
    const double nc_im = 2.0 * (c2_re * qc_im + c2_im * qc_re) - pc_im;
    ps_re = qs_re; ps_im = qs_im; qs_re = ns_re; qs_im = ns_im;
    pc_re = qc_re; pc_im = qc_im; qc_re = nc_re; qc_im = nc_im;
  }
  o->x = 500000.0 + u.k0A * (etap + S_im);
  o->y = (u.south ? 10000000.0 : 0.0) + u.k0A * (xip + S_re);
  // d zeta/dw = (1 + D1) cos z ;  d2 zeta/dw2 = -D2 cos^2 z - (1 + D1) cos z sin z
  const double g_re = 1.0 + D1_re, g_im = D1_im;
  o->zw_re = g_re * c_re - g_im * c_im;
  o->zw_im = g_re * c_im + g_im * c_re;
  const double cc_re = c_re * c_re - c_im * c_im, cc_im = 2.0 * c_re * c_im;
  const double cs_re = c_re * s_re - c_im * s_im, cs_im = c_re * s_im + c_im * s_re;
  o->zww_re = -(D2_re * cc_re - D2_im * cc_im) - (g_re * cs_re - g_im * cs_im);
  o->zww_im = -(D2_re * cc_im + D2_im * cc_re) - (g_re * cs_im + g_im * cs_re);
  // isometric latitude derivatives: psi' = (1-e2)/(cos(phi)(1-e2 sin^2 phi))
  const double phi = lat_deg * (kPi / 180.0);
  const double sp = sin(phi), cp = cos(phi);
  const double e2 = 1.0 - u.e2m;
  const double q = 1.0 - e2 * sp * sp;
  const double D = cp * q;
  o->dpsi1 = u.e2m / D;
  o->dpsi2 = u.e2m * (sp * q + 2.0 * e2 * sp * cp * cp) / (D * D);
}

// Projected coordinates of a point displaced by (dphi, dlam) radians.
// The device fuses its multiply-adds here and in utm_local_hermite: these
// positions only feed certified DEM lookups, whose allowance (kDemPosEps,
// 3e-8 m) is far above the rounding of either form (~1e-9 m).
SD_HD void utm_local_step(const Utm &u, const UtmLocal &l, double dphi, double dlam, double *x, double *y) {
  const double dw_im = dlam;
#if defined(__CUDA_ARCH__)
  const double dw_re = fma(0.5 * l.dpsi2 * dphi, dphi, l.dpsi1 * dphi);
  const double w2_re = fma(dw_re, dw_re, -dw_im * dw_im), w2_im = 2.0 * dw_re * dw_im;
  const double dz_re = fma(l.zw_re, dw_re, fma(-l.zw_im, dw_im, 0.5 * fma(l.zww_re, w2_re, -l.zww_im * w2_im)));
  const double dz_im = fma(l.zw_re, dw_im, fma(l.zw_im, dw_re, 0.5 * fma(l.zww_re, w2_im, l.zww_im * w2_re)));
  *x = fma(u.k0A, dz_im, l.x);
  *y = fma(u.k0A, dz_re, l.y);
#else
  const double dw_re = l.dpsi1 * dphi + 0.5 * l.dpsi2 * dphi * dphi;
  const double w2_re = dw_re * dw_re - dw_im * dw_im, w2_im = 2.0 * dw_re * dw_im;
  const double dz_re = l.zw_re * dw_re - l.zw_im * dw_im + 0.5 * (l.zww_re * w2_re - l.zww_im * w2_im);
  const double dz_im = l.zw_re * dw_im + l.zw_im * dw_re + 0.5 * (l.zww_re * w2_im + l.zww_im * w2_re);
  *x = l.x + u.k0A * dz_im;
  *y = l.y + u.k0A * dz_re;
#endif
}

// Projected point (and local expansion) at position t of the segment between
// two anchors A, B whose lon/lat differ by (dphi, dlam) radians: a cubic
// Hermite through the anchors' projected points and their derivatives along
// the segment (d/dt = dzeta/dw . (psi' dphi + i dlam)); the local-expansion
// terms are interpolated linearly.
SD_HD void utm_local_hermite(const UtmLocal &A, const UtmLocal &B, double dphi, double dlam, double k0A,
                             double t, UtmLocal *o) {
  const double aw = A.dpsi1 * dphi, bw = B.dpsi1 * dphi;
  const double ax_ = k0A * (A.zw_re * dlam + A.zw_im * aw), ay_ = k0A * (A.zw_re * aw - A.zw_im * dlam);
  const double bx_ = k0A * (B.zw_re * dlam + B.zw_im * bw), by_ = k0A * (B.zw_re * bw - B.zw_im * dlam);
  const double t2 = t * t, t3 = t2 * t;
  const double h00 = 2.0 * t3 - 3.0 * t2 + 1.0, h10 = t3 - 2.0 * t2 + t;
  const double h01 = -2.0 * t3 + 3.0 * t2, h11 = t3 - t2;
  const double u = 1.0 - t;
#if defined(__CUDA_ARCH__)
  o->x = fma(h00, A.x, fma(h01, B.x, fma(h10, ax_, h11 * bx_)));
  o->y = fma(h00, A.y, fma(h01, B.y, fma(h10, ay_, h11 * by_)));
  o->zw_re = fma(u, A.zw_re, t * B.zw_re);
  o->zw_im = fma(u, A.zw_im, t * B.zw_im);
  o->zww_re = fma(u, A.zww_re, t * B.zww_re);
  o->zww_im = fma(u, A.zww_im, t * B.zww_im);
  o->dpsi1 = fma(u, A.dpsi1, t * B.dpsi1);
  o->dpsi2 = fma(u, A.dpsi2, t * B.dpsi2);
#else
  o->x = h00 * A.x + h10 * ax_ + h01 * B.x + h11 * bx_;
  o->y = h00 * A.y + h10 * ay_ + h01 * B.y + h11 * by_;
  o->zw_re = u * A.zw_re + t * B.zw_re;
  o->zw_im = u * A.zw_im + t * B.zw_im;
  o->zww_re = u * A.zww_re + t * B.zww_re;
  o->zww_im = u * A.zww_im + t * B.zww_im;
  o->dpsi1 = u * A.dpsi1 + t * B.dpsi1;
  o->dpsi2 = u * A.dpsi2 + t * B.dpsi2;
#endif
}

// sin/cos of a + b from sin/cos of a, for |b| < 1e-4 (series to b^4).
SD_HD void sincos_add(double sa, double ca, double b, double *s, double *c) {
  const double b2 = b * b;
  const double sb = b * (1.0 - b2 * (1.0 / 6.0) * (1.0 - b2 * (1.0 / 20.0)));
  const double cb = 1.0 - 0.5 * b2 * (1.0 - b2 * (1.0 / 12.0));
  *s = sa * cb + ca * sb;
  *c = ca * cb - sa * sb;
}

// geodetic_to_ecef with sin/cos of latitude and longitude supplied
// (same operations as geodetic_to_ecef).
SD_HD V3 ecef_sc(double sin_lat, double cos_lat, double sin_lon, double cos_lon, double h) {
  double n = WGS84_A / sqrt(1.0 - WGS84_E2 * sin_lat * sin_lat);
  return {(n + h) * cos_lat * cos_lon, (n + h) * cos_lat * sin_lon, (n * (1.0 - WGS84_E2) + h) * sin_lat};
}
SD_HD double deg2rad_ecef(double deg) { return deg * kPi / 180.0; }  // geodesy.rs:39-40

// ── DEM: DemSource::elevation_at for one grid (dem.rs:351-409, 694-723) ────
struct DemView {
  const float *data;
  uint64_t width, height;
  double origin_y, origin_x, pixel_size;
  double inv_ps;  // 1 / pixel_size: fractional indices by multiplication (within an ulp of the quotient)
  int32_t kind;
  Utm utm;
};

// A DEM cell read on the device (bounds-checked in SD_BOUNDS_CHECK builds).
#if defined(__CUDA_ARCH__) && defined(SD_IN_BOUNDS)
#define SD_DEM_LD(d, i)                                                                          \
  (SD_IN_BOUNDS(::sd::BS_DEM, (i), (d).width * (d).height) ? __ldg(&(d).data[(i)]) : __int_as_float(0x7fc00000))
#else
#define SD_DEM_LD(d, i) __ldg(&(d).data[(i)])
#endif
SD_HD bool dem_sample(const DemView &d, double row_f, double col_f, float *h);

// returns false for Err(OutOfBounds); *h = NaN for voids.
SD_HD bool dem_elevation(const DemView &d, double lat_deg, double lon_deg, float *h) {
  double row_f, col_f;
  if (d.kind == SD_DEM_GEOGRAPHIC) {
    double lon_norm = lon_deg >= 180.0 ? lon_deg - 360.0 : lon_deg;
    row_f = (d.origin_y - lat_deg) / d.pixel_size;
    col_f = (lon_norm - d.origin_x) / d.pixel_size;
  } else {
    double x, y;
    utm_lonlat_to_xy(d.utm, lon_deg, lat_deg, &x, &y);
    row_f = (d.origin_y - y) / d.pixel_size;
    col_f = (x - d.origin_x) / d.pixel_size;
  }
  return dem_sample(d, row_f, col_f, h);
}

// Glo30Tile::elevation_at from fractional pixel coordinates (dem.rs:351-409).
SD_HD bool dem_sample(const DemView &d, double row_f, double col_f, float *h) {
  double max_row = (double)(d.height - 1);
  double max_col = (double)(d.width - 1);
  if (row_f < -0.5 || row_f > max_row + 0.5 || col_f < -0.5 || col_f > max_col + 0.5) return false;
  row_f = clampd(row_f, 0.0, max_row);
  col_f = clampd(col_f, 0.0, max_col);
  // bilinear_on_grid (dem.rs:385-409)
  uint64_t max_rc = d.height - 1;
  uint64_t r0 = f2u64(row_f);
  uint64_t rlim = max_rc == 0 ? 0 : max_rc - 1;
  if (r0 > rlim) r0 = rlim;
  uint64_t c0 = f2u64(col_f);
  uint64_t clim = d.width < 2 ? 0 : d.width - 2;
  if (c0 > clim) c0 = clim;
  uint64_t r1 = r0 + 1, c1 = c0 + 1;
  double dr = row_f - (double)r0;
  double dc = col_f - (double)c0;
#if defined(__CUDA_ARCH__)
  float v00 = SD_DEM_LD(d, r0 * d.width + c0), v01 = SD_DEM_LD(d, r0 * d.width + c1);
  float v10 = SD_DEM_LD(d, r1 * d.width + c0), v11 = SD_DEM_LD(d, r1 * d.width + c1);
#else
  float v00 = d.data[r0 * d.width + c0], v01 = d.data[r0 * d.width + c1];
  float v10 = d.data[r1 * d.width + c0], v11 = d.data[r1 * d.width + c1];
#endif
  if (v00 != v00 || v01 != v01 || v10 != v10 || v11 != v11) {
    *h = NAN;
    return true;
  }
  double v = (double)v00 * (1.0 - dr) * (1.0 - dc) + (double)v01 * (1.0 - dr) * dc +
             (double)v10 * dr * (1.0 - dc) + (double)v11 * dr * dc;
  *h = (float)v;
  return true;
}

// ── certified lookups ──────────────────────────────────────────────────────
// The device forms the DEM position of a UTM pixel by interpolation (the
// centre by a cubic Hermite between its row's anchors, the cardinal
// neighbours by a second-order local step) and fractional indices by
// multiplying with the reciprocal of the pixel size; the reference projects
// every lookup and divides.  The positions agree to ~9e-9 m (measured on a
// 250 km UTM row at 5,200 km northing, where the rounding of ~5e6 m northings
// dominates); kDemPosEps allows for northings up to 1e7 m.  A lookup is
// "decided" when the height the exact position gives is certain to be the
// same f32: no f32 rounding boundary lies within the bilinear value's
// uncertainty, and no cell edge, clamp or DEM margin lies within the
// position's.  An undecided lookup (~1e-4 of them) is redone exactly
// (dem_elevation).
constexpr double kDemPosEps = 3e-8;  // m

// 1 = decided (*inside = the lookup is inside the DEM; *h its height, NaN
// for a void), 0 = undecided.  eps_px: position uncertainty in pixels,
// to which the reciprocal's rounding is added here.
SD_HD int dem_sample_cert(const DemView &d, double row_f, double col_f, double eps_px, bool *inside, float *h) {
  const double max_row = (double)(d.height - 1);
  const double max_col = (double)(d.width - 1);
  // Within a pixel of the DEM's border the margin test (+-0.5 px,
  // dem.rs:351-371) and the clamps to [0, max] are near: left to the exact
  // lookup, as is anything non-finite.  Far outside is decided here.
  if (row_f < -1.0 || row_f > max_row + 1.0 || col_f < -1.0 || col_f > max_col + 1.0) {
    *inside = false;
    return 1;
  }
  if (!(row_f >= 1.0 && row_f <= max_row - 1.0 && col_f >= 1.0 && col_f <= max_col - 1.0)) return 0;
  const double eps = eps_px + 5e-16 * (row_f + col_f);
  *inside = true;
  uint64_t r0 = (uint64_t)row_f, c0 = (uint64_t)col_f;  // in [1, max - 1]: no clamp applies
  const double dr = row_f - (double)r0;
  const double dc = col_f - (double)c0;
  const uint64_t r1 = r0 + 1, c1 = c0 + 1;
#if defined(__CUDA_ARCH__)
#define SD_DEM_AT(R, C) SD_DEM_LD(d, (R) * d.width + (C))
#else
#define SD_DEM_AT(R, C) d.data[(R) * d.width + (C)]
#endif
  const float v00 = SD_DEM_AT(r0, c0), v01 = SD_DEM_AT(r0, c1);
  const float v10 = SD_DEM_AT(r1, c0), v11 = SD_DEM_AT(r1, c1);
  float lo4 = fminf(fminf(v00, v01), fminf(v10, v11)), hi4 = fmaxf(fmaxf(v00, v01), fmaxf(v10, v11));
  const bool nan4 = v00 != v00 || v01 != v01 || v10 != v10 || v11 != v11;
  // Within eps of a cell edge the exact position may fall in the next cell:
  // row er (r0 - 1 or r0 + 2) and column ec join the corners.  The bilinear
  // surface is continuous across the edge, so the value either cell gives
  // differs from this cell's by the corners' spread times eps plus rounding:
  // the spread is taken over the union.  (Output grids aligned with the DEM
  // put every lookup on a node, within rounding, so this is the common case.)
  const int64_t er = dr <= eps ? -1 : (dr >= 1.0 - eps ? 2 : 0);
  const int64_t ec = dc <= eps ? -1 : (dc >= 1.0 - eps ? 2 : 0);
  if (er | ec) {
    if (nan4) return 0;  // a void the other cell may not hold
    const uint64_t rr = (uint64_t)((int64_t)r0 + er), cc = (uint64_t)((int64_t)c0 + ec);
    float e0 = v00, e1 = v00, e2 = v00, e3 = v00, e4 = v00;
    if (er) e0 = SD_DEM_AT(rr, c0), e1 = SD_DEM_AT(rr, c1);
    if (ec) e2 = SD_DEM_AT(r0, cc), e3 = SD_DEM_AT(r1, cc);
    if (er && ec) e4 = SD_DEM_AT(rr, cc);
    if (e0 != e0 || e1 != e1 || e2 != e2 || e3 != e3 || e4 != e4) return 0;
    lo4 = fminf(lo4, fminf(fminf(e0, e1), fminf(fminf(e2, e3), e4)));
    hi4 = fmaxf(hi4, fmaxf(fmaxf(e0, e1), fmaxf(fmaxf(e2, e3), e4)));
  }
#undef SD_DEM_AT
  if (nan4) {
    *h = NAN;
    return 1;
  }
#if defined(__CUDA_ARCH__)
  // fused on the device: within a few ulps of the corner magnitudes of the
  // unfused sum, inside the 8e-15 allowance below
  const double wr = 1.0 - dr, wc = 1.0 - dc;
  const double v = fma((double)v11 * dr, dc, fma((double)v10 * dr, wc, fma((double)v01 * wr, dc, (double)v00 * wr * wc)));
#else
  const double v = (double)v00 * (1.0 - dr) * (1.0 - dc) + (double)v01 * (1.0 - dr) * dc +
                   (double)v10 * dr * (1.0 - dc) + (double)v11 * dr * dc;
#endif
  // the value's uncertainty: the corners' spread times the position's
  // uncertainty in both axes, plus the rounding of this sum and of the exact
  // position's (a few ulps of the corner magnitudes)
  const double dv = 2.0 * ((double)hi4 - (double)lo4) * eps + 8e-15 * fmax(fabs((double)lo4), fabs((double)hi4));
  const float lo = (float)(v - dv), hi = (float)(v + dv);
  if (lo != hi) return 0;
  *h = (float)v;
  return 1;
}

SD_HD bool dem_elevation(const DemView &d, double lat_deg, double lon_deg, float *h);
SD_HD_COLD bool dem_elevation_exact(const DemView &d, double lat_deg, double lon_deg, float *h) {
  return dem_elevation(d, lat_deg, lon_deg, h);
}

// Height at an interpolated projected position (x, y) of the geodetic point
// (lat, lon): decided from the position when possible, else the exact lookup.
SD_HD bool dem_at_xy_checked(const DemView &d, double x, double y, double lat_deg, double lon_deg, float *h) {
  bool inside = false;
  if (dem_sample_cert(d, (d.origin_y - y) * d.inv_ps, (x - d.origin_x) * d.inv_ps, kDemPosEps * d.inv_ps,
                      &inside, h))
    return inside;
  return dem_elevation_exact(d, lat_deg, lon_deg, h);
}
// Height at an exact lon/lat on a geographic DEM (only the reciprocal's
// rounding to allow for).
SD_HD bool dem_at_lonlat_checked(const DemView &d, double lon_deg, double lat_deg, float *h) {
  bool inside = false;
  const double lon_norm = lon_deg >= 180.0 ? lon_deg - 360.0 : lon_deg;
  if (dem_sample_cert(d, (d.origin_y - lat_deg) * d.inv_ps, (lon_norm - d.origin_x) * d.inv_ps, 0.0, &inside, h))
    return inside;
  return dem_elevation_exact(d, lat_deg, lon_deg, h);
}

// The same two lookups without the exact fallback: 1 = inside (*h the
// height, NaN on a void), 0 = outside the DEM, -1 = undecided (the caller
// defers the pixel to a pass that runs the checked form).
SD_HD int dem_at_xy_try(const DemView &d, double x, double y, float *h) {
  bool inside = false;
  if (!dem_sample_cert(d, (d.origin_y - y) * d.inv_ps, (x - d.origin_x) * d.inv_ps, kDemPosEps * d.inv_ps, &inside,
                       h))
    return -1;
  return inside ? 1 : 0;
}
SD_HD int dem_at_lonlat_try(const DemView &d, double lon_deg, double lat_deg, float *h) {
  bool inside = false;
  const double lon_norm = lon_deg >= 180.0 ? lon_deg - 360.0 : lon_deg;
  if (!dem_sample_cert(d, (d.origin_y - lat_deg) * d.inv_ps, (lon_norm - d.origin_x) * d.inv_ps, 0.0, &inside, h))
    return -1;
  return inside ? 1 : 0;
}

// The reference divides by the pixel size; the product with its reciprocal
// differs by at most an ulp of the fractional index (1e-16 px), far below
// anything the bilinear weights or the floor can resolve.
SD_HD bool dem_at_xy(const DemView &d, double x, double y, float *h) {
  return dem_sample(d, (d.origin_y - y) * d.inv_ps, (x - d.origin_x) * d.inv_ps, h);
}
SD_HD bool dem_at_lonlat(const DemView &d, double lon_deg, double lat_deg, float *h) {
  double lon_norm = lon_deg >= 180.0 ? lon_deg - 360.0 : lon_deg;
  return dem_sample(d, (d.origin_y - lat_deg) * d.inv_ps, (lon_norm - d.origin_x) * d.inv_ps, h);
}

// ── geoid (geoid.rs:220-251) ───────────────────────────────────────────────
SD_HD double geoid_undulation(const float *g, double lat_deg, double lon_deg) {
  if (g == nullptr) return 0.0;
  const uint64_t NLAT = 73, NLON = 144;
  // fmod(x, 360) is x itself for |x| < 360 (exactly, sign included)
  double lon = (lon_deg < 360.0 && lon_deg > -360.0) ? lon_deg : fmod(lon_deg, 360.0);
  if (lon < 0.0) lon += 360.0;
  double row_f = (90.0 - clampd(lat_deg, -90.0, 90.0)) / 2.5;
  double col_f = lon / 2.5;
  uint64_t r0 = f2u64(row_f);
  if (r0 > NLAT - 2) r0 = NLAT - 2;
  uint64_t r1 = r0 + 1;
  uint64_t c0 = f2u64(col_f) % NLON;
  uint64_t c1 = (c0 + 1) % NLON;
  double dr = row_f - (double)r0;
  double dc = col_f - (double)c0;
  double v00 = g[r0 * NLON + c0], v01 = g[r0 * NLON + c1];
  double v10 = g[r1 * NLON + c0], v11 = g[r1 * NLON + c1];
  dc = clampd(dc, 0.0, 1.0);
  return v00 * (1.0 - dr) * (1.0 - dc) + v01 * (1.0 - dr) * dc + v10 * dr * (1.0 - dc) + v11 * dr * dc;
}

// ── orbit: 8-point Lagrange position/velocity/acceleration (orbit.rs:498-596)
struct OrbitState {
  V3 pos, vel, acc;
};
enum { ORB_OK = 0, ORB_INSUFFICIENT = 1, ORB_OUTSIDE = 2 };

SD_HD int orbit_eval(const sd_state_vector *svs, uint64_t n, int64_t t, OrbitState *o) {
  if (n < 8) return ORB_INSUFFICIENT;
  if (t < svs[0].time_us || t > svs[n - 1].time_us) return ORB_OUTSIDE;
  const int64_t t_ref = svs[0].time_us;
  const double t_sec = (double)(t - t_ref) / 1e6;
  uint64_t lo = 0, hi = n;
  while (lo < hi) {
    uint64_t mid = (lo + hi) / 2;
    if (svs[mid].time_us <= t) lo = mid + 1; else hi = mid;
  }
  const uint64_t centre = lo - 1;
  const uint64_t start = centre < 4 ? 0 : (centre + 4 >= n ? n - 8 : centre - 3);
  double times[8];
#pragma unroll
  for (int i = 0; i < 8; ++i) times[i] = (double)(svs[start + i].time_us - t_ref) / 1e6;
  double rdiff[8];
  double total = 0.0;
#pragma unroll
  for (int j = 0; j < 8; ++j) {
    double diff = t_sec - times[j];
    rdiff[j] = 0.0;
    if (fabs(diff) > 1e-9) {
      rdiff[j] = 1.0 / diff;
      total += rdiff[j];
    }
  }
  double p0 = 0, p1 = 0, p2 = 0, v0 = 0, v1 = 0, v2 = 0, a0 = 0, a1 = 0, a2 = 0;
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    double basis = 1.0;
#pragma unroll
    for (int j = 0; j < 8; ++j)
      if (j != k) basis *= (t_sec - times[j]) / (times[k] - times[j]);
    double db = basis * (total - rdiff[k]);
    const sd_state_vector &sv = svs[start + k];
    p0 += basis * sv.position_m[0];
    p1 += basis * sv.position_m[1];
    p2 += basis * sv.position_m[2];
    v0 += basis * sv.velocity_m_s[0];
    v1 += basis * sv.velocity_m_s[1];
    v2 += basis * sv.velocity_m_s[2];
    a0 += db * sv.velocity_m_s[0];
    a1 += db * sv.velocity_m_s[1];
    a2 += db * sv.velocity_m_s[2];
  }
  o->pos = {p0, p1, p2};
  o->vel = {v0, v1, v2};
  o->acc = {a0, a1, a2};
  return ORB_OK;
}

// ── orbit as window polynomials ─────────────────────────────────────────────
// Inside one 8-point window (fixed by the "last state vector at or before t"
// rule, orbit.rs:530-535) the reference's position and velocity are degree-7
// polynomials in time (Lagrange interpolants of the window's positions and
// velocities) and its acceleration is the derivative of the velocity
// polynomial (orbit.rs:553-593: sum of L_k' v_k).  OrbPoly keeps their
// monomial coefficients about the window's fourth node, so a state is 60
// FMAs (Horner) instead of the Lagrange weights' divisions, and a scene's
// orbit is a few KB instead of a per-microsecond table.  The coefficients are
// formed in long double on the host; the states differ from the direct
// Lagrange sums by rounding only (~1e-9 m on 7e6 m).  At a time equal to a
// state-vector time the reference drops that node's 1/(t - t_j) term, which
// makes its acceleration differ from the derivative there; orbit_poly_eval
// then evaluates the reference formula directly.
struct OrbPoly {
  int64_t tc;       // time of the window's fourth node (us): x = (t - tc) / 1e6
  double c[9][8];   // pos xyz, vel xyz, acc xyz: coefficient of x^m at [.][m]
};

inline void orbit_poly_build(const sd_state_vector *svs, uint64_t n, OrbPoly *out) {
  for (uint64_t s = 0; s + 8 <= n; ++s) {
    OrbPoly &w = out[s];
    w.tc = svs[s + 3].time_us;
    long double x[8];
    for (int j = 0; j < 8; ++j) x[j] = (long double)(svs[s + j].time_us - w.tc) / 1e6L;
    long double cp[6][8] = {};
    for (int k = 0; k < 8; ++k) {
      long double poly[8] = {1.0L, 0, 0, 0, 0, 0, 0, 0};
      long double den = 1.0L;
      int deg = 0;
      for (int j = 0; j < 8; ++j) {
        if (j == k) continue;
        for (int m = deg + 1; m >= 1; --m) poly[m] = poly[m - 1] - x[j] * poly[m];
        poly[0] = -x[j] * poly[0];
        ++deg;
        den *= x[k] - x[j];
      }
      const sd_state_vector &sv = svs[s + k];
      for (int m = 0; m < 8; ++m) {
        const long double b = poly[m] / den;
        for (int d = 0; d < 3; ++d) {
          cp[d][m] += b * (long double)sv.position_m[d];
          cp[3 + d][m] += b * (long double)sv.velocity_m_s[d];
        }
      }
    }
    for (int d = 0; d < 6; ++d)
      for (int m = 0; m < 8; ++m) w.c[d][m] = (double)cp[d][m];
    for (int d = 0; d < 3; ++d) {
      for (int m = 0; m < 7; ++m) w.c[6 + d][m] = (double)((long double)(m + 1) * cp[3 + d][m + 1]);
      w.c[6 + d][7] = 0.0;
    }
  }
}

SD_HD double horner8(const double *c, double x) {
  double r = c[7];
  for (int m = 6; m >= 0; --m) r = fma(r, x, c[m]);
  return r;
}

// State at integer microsecond t from the window polynomials (orbit.rs:498-596
// semantics: window choice, refusal outside the state-vector span).
SD_HD int orbit_poly_eval(const sd_state_vector *svs, uint64_t n, const OrbPoly *win, int64_t t,
                          OrbitState *o) {
  if (n < 8) return ORB_INSUFFICIENT;
  if (t < svs[0].time_us || t > svs[n - 1].time_us) return ORB_OUTSIDE;
  uint64_t lo = 0, hi = n;
  while (lo < hi) {
    uint64_t mid = (lo + hi) / 2;
    if (svs[mid].time_us <= t) lo = mid + 1; else hi = mid;
  }
  const uint64_t centre = lo - 1;
  if (svs[centre].time_us == t) return orbit_eval(svs, n, t, o);
  const uint64_t start = centre < 4 ? 0 : (centre + 4 >= n ? n - 8 : centre - 3);
  const OrbPoly &w = win[start];
  const double x = (double)(t - w.tc) / 1e6;
  o->pos = {horner8(w.c[0], x), horner8(w.c[1], x), horner8(w.c[2], x)};
  o->vel = {horner8(w.c[3], x), horner8(w.c[4], x), horner8(w.c[5], x)};
  o->acc = {horner8(w.c[6], x), horner8(w.c[7], x), horner8(w.c[8], x)};
  return ORB_OK;
}

// One Newton step of solve_zero_doppler (terrain_correction.rs:1030-1067).
// Returns 0 = converged (|delta| < tol), 1 = step (t advanced), 2 = degenerate.
SD_HD int zd_step(V3 target, const OrbitState &s, double tol, double *delta_out) {
  V3 r = sub3(target, s.pos);
  double f = dot3(r, s.vel);
  double v_sq = dot3(s.vel, s.vel);
  double f_prime = -v_sq + dot3(r, s.acc);
  if (fabs(f_prime) < 1.0) return 2;
  double delta = -f / f_prime;
  *delta_out = delta;
  if (fabs(delta) < tol) return 0;
  return 1;
}

// ── resampling kernels (terrain_correction.rs:770-983) ─────────────────────
SD_HD double keys_weight(double t) {
  t = fabs(t);
  if (t < 1.0) return 1.5 * t * t * t - 2.5 * t * t + 1.0;
  if (t < 2.0) return -0.5 * t * t * t + 2.5 * t * t - 4.0 * t + 2.0;
  return 0.0;
}

SD_HD double lanczos_weight(double x) {
  double ax = fabs(x);
  if (ax < 1e-10) return 1.0;
  if (ax < 3.0) {
    double px = kPi * x;
    double pxa = kPi * x / 3.0;
    return sin(px) * sin(pxa) / (px * pxa);
  }
  return 0.0;
}

// ── terrain geometry (terrain_correction.rs:576-651) ───────────────────────
enum { GEOM_VALID = 0, GEOM_FORESHORTENING = 1, GEOM_LAYOVER = 2, GEOM_SHADOW = 3 };

SD_HD double flat_cell_area(double lat, double lon, double sp) {
  V3 fe = geodetic_to_ecef(lat, lon + sp, 0.0);
  V3 fw = geodetic_to_ecef(lat, lon - sp, 0.0);
  V3 fn = geodetic_to_ecef(lat + sp, lon, 0.0);
  V3 fs = geodetic_to_ecef(lat - sp, lon, 0.0);
  return norm3(cross3(sub3(fe, fw), sub3(fn, fs)));
}

SD_HD int terrain_geometry(double lat, double lon, double he, double hw, double hn, double hs,
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
  *cos_lia_out = clampd(local_proj / area, 0.0, 1.0);
  double w = local_proj / flat_area;
  *w_out = w;
  if (w < 0.05) return GEOM_FORESHORTENING;
  if (w > 2.0) return GEOM_LAYOVER;
  return GEOM_VALID;
}

}  // namespace sd
