// crmath.cuh — elementary functions written once for host and device, built
// from IEEE double additions, multiplications, divisions and square roots
// only, so the host compiler (gcc, no contraction) and the device compiler
// (nvcc --fmad=false) produce the same bits from the same inputs.  The one
// exception is sincos' fast path, which fuses its tail terms on the device:
// its results are correctly rounded on both sides, hence equal.
//
// * sincos: correctly rounded (round to nearest) sine and cosine for
//   |x| <= 1e5.  Method (Ziv's two-step strategy, as used by correctly
//   rounded libraries): Cody-Waite reduction x = k pi/2 + r with pi/2 split
//   into four parts (r as a double-double), r = j/256 + d with tabulated
//   sin(j/256), cos(j/256) as double-doubles, short Taylor series in d, and
//   the angle-addition formula evaluated in double-double arithmetic with
//   an error below 2^-66 of the result.  A result is returned only if it
//   rounds the same way at both ends of that error interval; otherwise
//   (about 1 call in 4000) a slow path evaluates the Taylor series of r in
//   double-double arithmetic (error ~2^-100) and tests again.  A result that
//   fails both tests (the exact value within ~2^-100 relative of a rounding
//   midpoint) is returned rounded from the slow path.  Larger |x|, NaN and
//   infinities go to the platform's sin/cos.
//   The terrain correction's target ECEF coordinates take their sines and
//   cosines from here: a libm that rounds correctly agrees with any other
//   such libm bit for bit, and the reference's own libm (glibc) disagrees
//   with correct rounding only in ~1.4e-3 of its sin/cos results.
// * tan, sinh, cosh, atanh and asinh (|x| <= 0.125), atan, atan2, hypot:
//   accurate to a few ulps, not correctly rounded; identical on host and
//   device.  They are the elementary functions of the UTM projection (a
//   restatement of the Krueger series, which the reference delegates to
//   proj4rs), so that the oracle and the device can evaluate that transform
//   with one arithmetic.
//
// All constants come from crmath_tab.h (generated by gen_crmath_tab.py in
// decimal arithmetic).
#pragma once

#include <cmath>
#include <cstdint>

#include "crmath_tab.h"

#if defined(__CUDACC__)
#define CRM_HD __host__ __device__ __forceinline__
#define CRM_HD_CALL __host__ __device__ inline
#define CRM_HD_COLD static __host__ __device__ __noinline__
#else
#define CRM_HD inline
#define CRM_HD_CALL inline
#define CRM_HD_COLD inline
#endif

namespace sd {
namespace crm {

#if defined(__CUDACC__)
__device__ const double d_sincos_tab[CRM_TAB_J * 4] = {CRM_SINCOS_TABLE};
__device__ const double d_invfact[64] = {CRM_INVFACT_TABLE};
__device__ const double d_invodd[32] = {CRM_INVODD_TABLE};
#endif
static const double h_sincos_tab[CRM_TAB_J * 4] = {CRM_SINCOS_TABLE};
static const double h_invfact[64] = {CRM_INVFACT_TABLE};
static const double h_invodd[32] = {CRM_INVODD_TABLE};

CRM_HD double sincos_tab(int i) {
#if defined(__CUDA_ARCH__)
  return __ldg(d_sincos_tab + i);
#else
  return h_sincos_tab[i];
#endif
}
CRM_HD double invfact(int i) {
#if defined(__CUDA_ARCH__)
  return __ldg(d_invfact + i);
#else
  return h_invfact[i];
#endif
}
CRM_HD double invodd(int i) {
#if defined(__CUDA_ARCH__)
  return __ldg(d_invodd + i);
#else
  return h_invodd[i];
#endif
}

// ── error-free transformations and double-double arithmetic ───────────────
CRM_HD void two_sum(double a, double b, double &s, double &e) {
  s = a + b;
  const double bb = s - a;
  e = (a - (s - bb)) + (b - bb);
}
CRM_HD void fast_two_sum(double a, double b, double &s, double &e) {  // |a| >= |b| or a == 0
  s = a + b;
  e = b - (s - a);
}
// p + e = a * b exactly: a fused multiply-add on the device; Dekker's
// product with Veltkamp's split on the host (the same exact e).
CRM_HD void two_prod(double a, double b, double &p, double &e) {
  p = a * b;
#if defined(__CUDA_ARCH__)
  e = fma(a, b, -p);
#else
  const double c = 134217729.0;  // 2^27 + 1
  double t = c * a;
  const double ah = t - (t - a), al = a - ah;
  t = c * b;
  const double bh = t - (t - b), bl = b - bh;
  e = ((ah * bh - p) + ah * bl + al * bh) + al * bl;
#endif
}
struct DD {
  double h, l;
};
CRM_HD DD dd_add(DD a, DD b) {
  double s, e;
  two_sum(a.h, b.h, s, e);
  e += a.l + b.l;
  DD r;
  fast_two_sum(s, e, r.h, r.l);
  return r;
}
CRM_HD DD dd_mul(DD a, DD b) {
  double p, e;
  two_prod(a.h, b.h, p, e);
  e += a.h * b.l + a.l * b.h;
  DD r;
  fast_two_sum(p, e, r.h, r.l);
  return r;
}

// Round-to-nearest test: the exact value lies within err of h + l, with
// h = RN(h + l).  True (and *out = the correctly rounded value) when both
// ends of the interval round to the same double.
CRM_HD bool round_ok(double h, double l, double err, double *out) {
  const double a = h + (l + err), b = h + (l - err);
  *out = a;
  return a == b;
}

// x = k pi/2 + r, r = rh + rl; returns k mod 4.  |k| < 2^20 keeps k * PIO2_1
// and k * PIO2_2 exact, and x - k * PIO2_1 is exact (Sterbenz).  The fast
// form leaves out PIO2_4 (k 2^-123 of absolute error).
CRM_HD int reduce_pio2(double x, bool with_p4, double &rh, double &rl) {
  const double kd = rint(x * CRM_TWO_OVER_PI);
  const double r1 = x - kd * CRM_PIO2_1;
  double s, e, p3, e3, s2, e2;
  two_sum(r1, -(kd * CRM_PIO2_2), s, e);
  two_prod(kd, CRM_PIO2_3, p3, e3);
  two_sum(s, -p3, s2, e2);
  double lo = (e + e2) - e3;
  if (with_p4) lo -= kd * CRM_PIO2_4;
  fast_two_sum(s2, lo, rh, rl);
  return (int)((int64_t)kd & 3);
}

// sin and cos of a = ah + al in [0, pi/4 + 2^-9], fast path (error below
// 2^-66 relative).  a = j/256 + d, d = dh + al, |dh| <= 2^-9.
//   sin(a) = S + C dh + [S_l + C_l dh + C dl + S pc + C dh ps - S dh dl]
//   cos(a) = C - S dh + [C_l - S_l dh - S dl + C pc - S dh ps - C dh dl]
// with S, C = sin, cos(j/256), pc = cos(dh) - 1, ps = sin(dh)/dh - 1 and
// every dropped term below 2^-72 of the result.
CRM_HD void sincos_fast(double ah, double al, DD *s, DD *c) {
  const int j = (int)rint(ah * (double)CRM_TAB_N);
  const double dh = ah - (double)j * (1.0 / CRM_TAB_N);  // exact
  const double dl = al;
  const double Sh = sincos_tab(4 * j), Sl = sincos_tab(4 * j + 1);
  const double Ch = sincos_tab(4 * j + 2), Cl = sincos_tab(4 * j + 3);
  const double d2 = dh * dh;
  double p, pe, m, me;
#if defined(__CUDA_ARCH__)
  // The same terms in the same order with fused multiply-adds: one rounding
  // per term instead of two, so the error bound holds a fortiori and a
  // result that passes the rounding test is the correctly rounded value,
  // equal to the host's.  (The FP64 pipe bounds the terrain kernels, and
  // this halves the multiply-add count of the tails.)
  const double pc = d2 * fma(d2, fma(-d2, 1.0 / 720.0, 1.0 / 24.0), -0.5);
  const double ps = d2 * fma(d2, fma(-d2, 1.0 / 5040.0, 1.0 / 120.0), -1.0 / 6.0);
  const double dps = dh * ps, ddl = dh * dl;
  two_prod(Ch, dh, p, pe);
  two_sum(Sh, p, m, me);
  double t = fma(-Sh, ddl, fma(Ch, dps, fma(Sh, pc, fma(Ch, dl, fma(Cl, dh, me + pe + Sl)))));
  fast_two_sum(m, t, s->h, s->l);
  two_prod(Sh, dh, p, pe);
  two_sum(Ch, -p, m, me);
  t = fma(-Ch, ddl, fma(-Sh, dps, fma(Ch, pc, fma(-Sh, dl, fma(-Sl, dh, me - pe + Cl)))));
  fast_two_sum(m, t, c->h, c->l);
#else
  const double pc = d2 * (-0.5 + d2 * ((1.0 / 24.0) - d2 * (1.0 / 720.0)));
  const double ps = d2 * ((-1.0 / 6.0) + d2 * ((1.0 / 120.0) - d2 * (1.0 / 5040.0)));
  const double dps = dh * ps, ddl = dh * dl;
  // sine
  two_prod(Ch, dh, p, pe);
  two_sum(Sh, p, m, me);
  double t = me + pe + Sl + Cl * dh + Ch * dl + Sh * pc + Ch * dps - Sh * ddl;
  fast_two_sum(m, t, s->h, s->l);
  // cosine
  two_prod(Sh, dh, p, pe);
  two_sum(Ch, -p, m, me);
  t = me - pe + Cl - Sl * dh - Sh * dl + Ch * pc - Sh * dps - Ch * ddl;
  fast_two_sum(m, t, c->h, c->l);
#endif
}

// sin and cos of r = (rh, rl), |r| <= pi/4 + 2^-9, by their Taylor series in
// double-double arithmetic (terms to r^29: error ~2^-100).
CRM_HD_COLD void sincos_slow(double rh, double rl, DD *s, DD *c) {
  const DD r{rh, rl};
  const DD r2 = dd_mul(r, r);
  DD ps{invfact(2 * 29), invfact(2 * 29 + 1)};
  DD pc{invfact(2 * 28), invfact(2 * 28 + 1)};
  for (int n = 27; n >= 1; n -= 2) {  // sin: sum (-1)^k r^(2k+1) / (2k+1)!
    const bool neg = (n >> 1) & 1;
    const DD cf{neg ? -invfact(2 * n) : invfact(2 * n), neg ? -invfact(2 * n + 1) : invfact(2 * n + 1)};
    ps = dd_add(dd_mul(ps, r2), cf);
  }
  for (int n = 26; n >= 0; n -= 2) {  // cos: sum (-1)^k r^(2k) / (2k)!
    const bool neg = (n >> 1) & 1;
    const DD cf{neg ? -invfact(2 * n) : invfact(2 * n), neg ? -invfact(2 * n + 1) : invfact(2 * n + 1)};
    pc = dd_add(dd_mul(pc, r2), cf);
  }
  *s = dd_mul(ps, r);
  *c = pc;
}

// Correctly rounded sin(x) and cos(x).  The slow path is not inlined at the
// call sites (it runs for ~1 call in 4000).
CRM_HD void sincos(double x, double *so, double *co) {
  if (!(fabs(x) <= 1e5)) {  // outside the reduction's range, NaN, infinities
    *so = ::sin(x);
    *co = ::cos(x);
    return;
  }
  double rh = x, rl = 0.0;
  // |x| < 0.78 < pi/4: k = 0, and every step of the reduction is exact, so it
  // would return (x, 0) itself.
  int q = fabs(x) < 0.78 ? 0 : reduce_pio2(x, false, rh, rl);
  const bool neg = rh < 0.0;
  DD s, c;
  sincos_fast(neg ? -rh : rh, neg ? -rl : rl, &s, &c);
  double sv, cv;
  bool ok = round_ok(s.h, s.l, fabs(s.h) * 0x1p-66 + 0x1p-100, &sv) &&
            round_ok(c.h, c.l, fabs(c.h) * 0x1p-66 + 0x1p-100, &cv);
  if (!ok) {
    q = reduce_pio2(x, true, rh, rl);
    sincos_slow(rh, rl, &s, &c);
    if (!round_ok(s.h, s.l, fabs(s.h) * 0x1p-98 + 0x1p-150, &sv)) sv = s.h + s.l;
    if (!round_ok(c.h, c.l, fabs(c.h) * 0x1p-98 + 0x1p-150, &cv)) cv = c.h + c.l;
  } else if (neg) {
    sv = -sv;
  }
  // x = k pi/2 + r
  switch (q) {
    case 0: *so = sv; *co = cv; break;
    case 1: *so = cv; *co = -sv; break;
    case 2: *so = -sv; *co = -cv; break;
    default: *so = -cv; *co = sv; break;
  }
}
CRM_HD double sin(double x) {
  double s, c;
  sincos(x, &s, &c);
  return s;
}
CRM_HD double cos(double x) {
  double s, c;
  sincos(x, &s, &c);
  return c;
}
CRM_HD double tan(double x) {
  double s, c;
  sincos(x, &s, &c);
  return s / c;
}

// ── functions of the UTM projection (a few ulps; identical on host and device)
// e^x - 1 for |x| <= 0.35: Taylor series to x^16 (truncation < 2^-68 relative).
CRM_HD_CALL double expm1_small(double x) {
  double p = invfact(2 * 16);
  for (int n = 15; n >= 1; --n) p = p * x + invfact(2 * n);
  return p * x;
}
CRM_HD double exp(double x) {
  if (!(fabs(x) <= 700.0)) return ::exp(x);
  const double kd = rint(x * CRM_INV_LN2);
  const double r = (x - kd * CRM_LN2_1) - kd * CRM_LN2_2;
  return ldexp(1.0 + expm1_small(r), (int)kd);
}
CRM_HD double sinh(double x) {
  const double ax = fabs(x);
  double v;
  if (ax < 0.35) {
    const double em = expm1_small(ax);
    v = 0.5 * (em + em / (em + 1.0));
  } else {
    const double e = exp(ax);
    v = 0.5 * (e - 1.0 / e);
  }
  return x < 0.0 ? -v : v;
}
CRM_HD double cosh(double x) {
  const double e = exp(fabs(x));
  return 0.5 * (e + 1.0 / e);
}
// atanh(x) = sum x^(2n+1) / (2n+1) for |x| <= 0.125 (terms to x^23:
// truncation < 2^-70 relative); the platform's atanh beyond (the UTM
// transform's arguments stay below the eccentricity, 0.082).
CRM_HD_CALL double atanh(double x) {
  if (!(fabs(x) <= 0.125)) return ::atanh(x);
  const double x2 = x * x;
  double p = invodd(11);
  for (int n = 10; n >= 0; --n) p = p * x2 + invodd(n);
  return p * x;
}
// asinh(x) = atanh(x / sqrt(1 + x^2)) for |x| <= 0.125 (the UTM transform's
// arguments stay below ~0.11 within a zone and its neighbours); the
// platform's asinh beyond.
CRM_HD double asinh(double x) {
  if (!(fabs(x) <= 0.125)) return ::asinh(x);
  return atanh(x / ::sqrt(1.0 + x * x));
}
// atan by two half-angle reductions, atan(x) = 2 atan(x / (1 + sqrt(1 + x^2))),
// to |x| <= tan(pi/16), then its Taylor series to x^29 (truncation < 2^-70
// relative); |x| > 1 through pi/2 - atan(1/x).
CRM_HD_CALL double atan(double x) {
  if (x != x) return x;
  const double ax = fabs(x);
  const bool inv = ax > 1.0;
  double y = inv ? 1.0 / ax : ax;
  y = y / (1.0 + ::sqrt(1.0 + y * y));
  y = y / (1.0 + ::sqrt(1.0 + y * y));
  const double y2 = y * y;
  double p = invodd(14);
  for (int n = 13; n >= 0; --n) p = p * y2 + ((n & 1) ? -invodd(n) : invodd(n));
  double v = 4.0 * (p * y);
  if (inv) v = (CRM_PIO2_1 - v) + (CRM_PIO2_2 + CRM_PIO2_3);
  return x < 0.0 ? -v : v;
}
CRM_HD double atan2(double y, double x) {
  if (x != x || y != y) return x + y;
  const double pi_h = 2.0 * CRM_PIO2_1, pi_l = 2.0 * (CRM_PIO2_2 + CRM_PIO2_3);
  if (x == 0.0) {
    if (y == 0.0) return std::signbit(x) ? (std::signbit(y) ? -(pi_h + pi_l) : pi_h + pi_l) : y;
    return y > 0.0 ? CRM_PIO2_1 + (CRM_PIO2_2 + CRM_PIO2_3) : -(CRM_PIO2_1 + (CRM_PIO2_2 + CRM_PIO2_3));
  }
  const double a = atan(fabs(y / x));
  double v = x > 0.0 ? a : (pi_h - a) + pi_l;
  return std::signbit(y) ? -v : v;
}
CRM_HD double hypot(double x, double y) {
  double a = fabs(x), b = fabs(y);
  if (a < b) {
    const double t = a;
    a = b;
    b = t;
  }
  if (a == 0.0 || b != b || a != a) return a + b;
  const double r = b / a;
  return a * ::sqrt(1.0 + r * r);
}

}  // namespace crm
}  // namespace sd
