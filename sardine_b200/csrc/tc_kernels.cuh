// tc_kernels.cuh — device code of the backward Range-Doppler terrain
// correction (terrain_correction.rs:1245-1836) and the host helpers that lay
// out work tables and launch its stages.  Included by tc.cu (one scene per
// call) and tc_tiles.cu (batches of tiles over resident scenes).
//
// The reference walks each output row column by column: the Newton
// zero-Doppler solve of column c starts from the converged azimuth time of
// the previous converged column (1443, 1580), moves in whole microseconds
// truncated toward zero (1067) and stops BEFORE applying a sub-tolerance
// step (1045-1065).  The converged time therefore depends on the seed, and a
// 1 us difference moves the sample by ~5e-4 azimuth line.  The stages
// reproduce that chain exactly while keeping the work data-parallel:
//
//  k_orbit_table   FP64 Lagrange state (pos, vel, acc, |v|^2) at every
//                  microsecond of the span a scene needs (80 B each), so a
//                  Newton iteration is one table read instead of an 8-point
//                  Lagrange evaluation with 56 divisions; outside the table
//                  the window polynomials (geo.cuh: OrbPoly) stand in.
//  k_orbit_taylor  the orbit's Taylor expansion about every 4th ms of the
//                  table's span, from which k_main's warps take their
//                  approximate states between table reads.
//  k_row_*         per-row set-up: UTM anchors (output_crs.rs:364-417),
//                  latitude seed, LUT guess, flat-cell area, and a coarse
//                  azimuth-time model (17 knots per row).
//  k_heights       per pixel: the DEM heights of the centre and of the four
//                  cardinal neighbours, decided as the exact projection
//                  would decide them (geo.cuh: dem_sample_cert).
//  k_main          per pixel: geoid, target ECEF; the reference iteration
//                  from the model time gives one converged time t*; the set
//                  F = {t : |delta(t)| < tol} of possible converged times (a
//                  pair {fb, fb+1}); and the outcome of the reference
//                  iteration from every member of the left neighbour's F (the
//                  only seeds the chain can hand it).  Decisions taken on an
//                  approximate orbit state near a threshold are re-taken on
//                  the reference's state.
//  k_scan          per row: a warp walks the columns composing the per-pixel
//                  outcome maps, selects each pixel's member of F, and runs
//                  the reference iteration in place for any seed outside the
//                  precomputed set.
//  k_cand          per pixel: the outputs (resampling, Small-2011 geometry,
//                  mask, NESZ) of the one selected converged time, final
//                  rasters, counters and Newton histogram; split precision
//                  defers what FP32 cannot settle to k_resample and k_redo.
#pragma once
#include <algorithm>
#include <cstdlib>
#include <limits>
#include <memory>

#include "tiles.cuh"

#ifndef SD_FACET_ABSOLUTE
#define SD_FACET_ABSOLUTE 0
#endif

#include "geo.cuh"
#include "runtime.cuh"

namespace sd {
namespace {

enum : uint8_t { ST_CONV = 0, ST_NONCONV = 1, ST_DEGEN = 2, ST_ORBIT = 3, ST_DEMMISS = 4 };
constexpr int KNOTS = 17;
constexpr int kCounters = 10;  // valid, dem, outside, nonconv, degen, flat, noise, spare, dB converted, dB masked
constexpr int kCntDb = 8;      // counters[kCntDb + cls] for db_value's class cls (0 converted, 1 noise-masked)

struct OrbTaylor;

struct OrbitDev {
  const sd_state_vector *svs;
  uint64_t n;
  const double2 *tab;   // 5 double2 per microsecond: pos, vel, acc, |v|^2
  int64_t tab_t0;
  int64_t tab_n;
  const OrbPoly *poly;  // n - 7 window polynomials for times outside the table
  const OrbTaylor *tay;  // expansions about tab_t0 + k * TAY_STEP, k < tay_n (k_orbit_taylor)
  int64_t tay_n;
};

// State at integer microsecond t: the table (the reference's Lagrange sums,
// evaluated once per microsecond) inside its span, the window polynomials
// outside it, the Lagrange sums directly when neither exists.  *exact: the
// state is the reference's Lagrange sums (not the polynomial form).
__device__ __forceinline__ int orbit_at(const OrbitDev &o, int64_t t, OrbitState *s, double *vsq,
                                        bool *exact = nullptr) {
  const int64_t i = t - o.tab_t0;
  if (exact) *exact = !(o.poly && !(i >= 0 && i < o.tab_n));
  if (i >= 0 && i < o.tab_n) {
    const double2 *e = o.tab + 5 * i;
    double2 a = __ldg(e), b = __ldg(e + 1), c = __ldg(e + 2), d = __ldg(e + 3), f = __ldg(e + 4);
    s->pos = {a.x, a.y, b.x};
    s->vel = {b.y, c.x, c.y};
    s->acc = {d.x, d.y, f.x};
    *vsq = f.y;
    return ORB_OK;
  }
  const int rc = o.poly ? orbit_poly_eval(o.svs, o.n, o.poly, t, s) : orbit_eval(o.svs, o.n, t, s);
  if (rc == ORB_OK) *vsq = dot3(s->vel, s->vel);
  return rc;
}

// The Lagrange sums out of line (taken rarely: times outside the table).
__device__ __noinline__ int orbit_eval_cold(const sd_state_vector *svs, uint64_t n, int64_t t, OrbitState *s) {
  return orbit_eval(svs, n, t, s);
}

// The reference's own state at t: the table inside its span, else the
// Lagrange sums (orbit_eval, the reference's formula).
__device__ __forceinline__ int orbit_exact(const OrbitDev &o, int64_t t, OrbitState *s, double *vsq) {
  const int64_t i = t - o.tab_t0;
  if (i >= 0 && i < o.tab_n) return orbit_at(o, t, s, vsq);
  const int rc = orbit_eval_cold(o.svs, o.n, t, s);
  if (rc == ORB_OK) *vsq = dot3(s->vel, s->vel);
  return rc;
}

// The reference's satellite position at t (the first 24 B of the table entry).
__device__ __forceinline__ bool orbit_pos_exact(const OrbitDev &o, int64_t t, V3 *S) {
  const int64_t i = t - o.tab_t0;
  if (i >= 0 && i < o.tab_n) {
    const double2 *e = o.tab + 5 * i;
    const double2 a = __ldg(e), b = __ldg(e + 1);
    *S = {a.x, a.y, b.x};
    return true;
  }
  OrbitState s;
  if (orbit_eval_cold(o.svs, o.n, t, &s) != ORB_OK) return false;
  *S = s.pos;
  return true;
}

// A Newton decision (the |delta| < tol test or the microsecond truncation of
// the step, 1045-1067) taken on an approximate state (the window polynomials,
// or a warp's Taylor expansion: within ~2e-8 m and ~2e-11 m/s of the
// reference's sums, which moves delta by <= ~3e-12 s) is re-taken on the
// reference's state when it lies within kZdEps of its threshold.
constexpr double kZdEps = 1e-11;  // s
__device__ __forceinline__ bool zd_marginal(double d, double tol) {
  const double ad = fabs(d);
  const double m = ad * 1e6, fr = m - floor(m);
  return fabs(ad - tol) <= kZdEps || fr <= kZdEps * 1e6 || fr >= 1.0 - kZdEps * 1e6;
}

struct ZdRes {
  uint8_t st;
  int64_t t;
  int it;
};

// solve_zero_doppler (terrain_correction.rs:1010-1073), bit-exact: a decision
// taken on a polynomial state near its threshold is re-taken on the
// reference's state.
__device__ ZdRes newton(const OrbitDev &o, V3 P, int64_t seed, int max_iter, double tol) {
  int64_t t = seed;
  for (int i = 0; i < max_iter; ++i) {
    OrbitState s;
    double vsq;
    bool exact;
    if (orbit_at(o, t, &s, &vsq, &exact) != ORB_OK) return {ST_ORBIT, t, i};
    V3 r = sub3(P, s.pos);
    double f = dot3(r, s.vel);
    double fp = -vsq + dot3(r, s.acc);
    if (fabs(fp) < 1.0) return {ST_DEGEN, t, i};
    double delta = -f / fp;
    if (!exact && zd_marginal(delta, tol) && orbit_exact(o, t, &s, &vsq) == ORB_OK) {
      r = sub3(P, s.pos);
      f = dot3(r, s.vel);
      fp = -vsq + dot3(r, s.acc);
      if (fabs(fp) < 1.0) return {ST_DEGEN, t, i};
      delta = -f / fp;
    }
    if (fabs(delta) < tol) return {ST_CONV, t, i + 1};
    t = t + f2i64(delta * 1e6);
  }
  return {ST_NONCONV, t, max_iter};
}

struct TcDev {
  // output grid
  uint64_t rows, cols;
  double lat_north, lon_west, sp, step_deg;
  int utm;
  Utm proj;
  // anchors (UTM)
  const double *ax;   // n_pts
  const double *alon; // rows * n_pts
  const double *alat;
  const UtmLocal *aloc; // rows * n_pts: DEM projection (UTM DEM) at every anchor, or null
  int n_anchors, n_pts;
  // LUT
  const double *lut_lat;
  const int64_t *lut_t;
  int lut_n;
  // rows
  int64_t *row_guess;
  double *row_flat;
  int64_t *knot_t;
  // scene
  OrbitDev orb;
  DemView dem;
  const float *geoid;
  const float *img;
  const float *nesz;
  uint64_t lines, samples;
  int64_t az_start;
  double ati, near_range, rps;
  int max_iter;
  double tol;
  int flatten, compute_lia, need_geom, resampling, nesz_mask;
  float nesz_factor;
  // per-pixel scratch
  int64_t *fb;
  uint32_t *cc;
  uint8_t *sel;
  // outputs
  float *out;
  float *cos_lia;
  uint8_t *mask;
  int64_t *az_time;  // optional: converged azimuth time per pixel (INT64_MIN if none)
  int *flags;
  unsigned long long *counters;
  unsigned long long *trange;  // [0] = min, [1] = max (biased by 2^63), or null
  uint64_t bpr;                // k_main row segments per row
  int seg_px;                  // pixels per k_main row segment (a segment is seg_px + 1 threads: the
  int seg_per_item;            // first is the left neighbour), and segments per k_main item
  int fast;                    // tolerance allows the fixed-point-pair scheme
  int split;                   // SD_PRECISION_SPLIT
  uint64_t row0;               // grid row of the job's first row (row bands)
  // per pixel, from k_heights (structure of arrays, npx apart): the target
  // ECEF x, y, z (x NaN: no DEM height) and, when the facet is needed, the
  // facet normal x, y, z and area (area NaN: a neighbour height missing)
  const double *tp;
  const double *fct;
  int db;                      // write sigma0/gamma0 in dB (to_db_inplace), below db_floor as NaN
  float db_floor;
  uint32_t *rs_cnt;            // split: per k_cand item (256 px), FP64 re-samples queued (may exceed RS_CAP)
  struct RsEnt *rs_ent;        // split: per k_cand item, RS_CAP queued re-samples
};

// ── work table ──────────────────────────────────────────────────────────────
// Every kernel below is one launch over a table of jobs (a whole scene, or
// many tiles of many scenes): for each stage, pre[stage][j] is the exclusive
// prefix sum of the stage's work items over jobs 0..j-1.  Kernels are
// persistent (grid sized to the device's resident CTAs) and stride over the
// items; a CUDA graph of the stages therefore does not depend on the batch.
enum { WK_ANCH = 0, WK_ROWS = 1, WK_KNOT = 2, WK_MAIN = 3, WK_SCAN = 4, WK_SEL = 5, WK_REDO = 6, kWk = 7 };
constexpr int SEL_THREADS = 256;
constexpr int REDO_CHUNK = SEL_THREADS * 32;  // pixels one k_redo block compacts

struct TcWork {
  int n_jobs;
  uint32_t hq_cap;      // capacity of hq
  const TcDev *jobs;
  const uint64_t *pre;  // kWk x (n_jobs + 1)
  // k_heights' deferred pixels (a DEM lookup undecided): job << 40 | pixel;
  // *hq_cnt counts every deferral, also those past hq_cap (done in place)
  unsigned long long *hq;
  unsigned int *hq_cnt;
};

__device__ __forceinline__ const uint64_t *stage_pre(const TcWork &w, int stage) {
  return w.pre + (size_t)stage * (size_t)(w.n_jobs + 1);
}

// last job j with pre[j] <= item (jobs without items in the stage are skipped)
__device__ __forceinline__ int find_job(const uint64_t *pre, int n_jobs, uint64_t item) {
  int lo = 0, hi = n_jobs;
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (__ldg(pre + mid) <= item) lo = mid;
    else hi = mid;
  }
  return lo;
}

// Copies a job record into shared memory with the calling threads.
__device__ __forceinline__ void load_job(unsigned char *dst, const TcDev *src, int lane, int nthreads) {
  static_assert(sizeof(TcDev) % 8 == 0, "TcDev size");
  const unsigned long long *s = reinterpret_cast<const unsigned long long *>(src);
  unsigned long long *d = reinterpret_cast<unsigned long long *>(dst);
  for (int k = lane; k < (int)(sizeof(TcDev) / 8); k += nthreads) d[k] = __ldg(s + k);
}

__device__ __forceinline__ double row_y(const TcDev &p, uint64_t r) {
  return p.lat_north - ((double)(r + p.row0) + 0.5) * p.sp;
}

// Output pixel centre in lon/lat: direct for WGS84, project_row anchors for
// UTM (output_crs.rs:383-415).
// Pixel centre as in pixel_lonlat, plus the anchor segment g and the
// position t in it (UTM grids only).
__device__ __forceinline__ void pixel_seg(const TcDev &p, uint64_t r, uint64_t c, double *lon, double *lat,
                                          int *gs, double *ts);

__device__ __forceinline__ void pixel_lonlat(const TcDev &p, uint64_t r, uint64_t c, double *lon, double *lat) {
  int g;
  double t;
  pixel_seg(p, r, c, lon, lat, &g, &t);
}

__device__ __forceinline__ void pixel_seg(const TcDev &p, uint64_t r, uint64_t c, double *lon, double *lat,
                                          int *gs, double *ts) {
  *gs = 0;
  *ts = 0.0;
  if (!p.utm) {
    *lon = p.lon_west + ((double)c + 0.5) * p.sp;
    *lat = row_y(p, r);
    return;
  }
  const double x_start = p.lon_west + 0.5 * p.sp;
  const double x = x_start + (double)c * p.sp;
  const int na = p.n_anchors;
  // segment: smallest s with s == na-1 or x <= ax[s+1]
  double anchor_dx = p.ax[1] - p.ax[0];
  int g = 0;
  if (anchor_dx > 0.0) {
    double q = floor((x - x_start) / anchor_dx);
    g = q < 0.0 ? 0 : (q > (double)(na - 1) ? na - 1 : (int)q);
  }
  while (g > 0 && x <= p.ax[g]) g--;
  while (g + 1 < na && x > p.ax[g + 1]) g++;
  const double x0 = p.ax[g], x1 = p.ax[g + 1];
  const double *lo = p.alon + r * p.n_pts, *la = p.alat + r * p.n_pts;
  double t = (x1 == x0) ? 0.0 : (x - x0) / (x1 - x0);
  *lon = lo[g] + t * (lo[g + 1] - lo[g]);
  *lat = la[g] + t * (la[g + 1] - la[g]);
  *gs = g;
  *ts = t;
}

// DEM-side projection of a pixel centre from its row's anchors (UTM grid on
// a UTM DEM).  The centre is the linear interpolation of anchors g, g+1 in
// lon/lat, so its projected position is a smooth function of t over the
// ~1 km segment: a cubic Hermite through the anchors' projected points and
// their derivatives along the segment (d/dt = dzeta/dw . (psi' dphi + i
// dlam)) reproduces the exact projection to ~1e-11 m.  The local-expansion
// terms used for the cardinal neighbours move by ~1e-4 relative over a
// segment and are interpolated linearly (effect ~3e-8 m on a 10 m step).
__device__ __forceinline__ void dem_local_from_anchors(const TcDev &p, uint64_t r, int g, double t, UtmLocal *o) {
  const UtmLocal &A = p.aloc[r * p.n_pts + g], &B = p.aloc[r * p.n_pts + g + 1];
  const double *lo = p.alon + r * p.n_pts, *la = p.alat + r * p.n_pts;
  const double k = kPi / 180.0;
  utm_local_hermite(A, B, (la[g + 1] - la[g]) * k, (lo[g + 1] - lo[g]) * k, p.dem.utm.k0A, t, o);
}

// guess_azimuth_time (terrain_correction.rs:1107-1137)
__device__ int64_t guess_time(const TcDev &p, double lat) {
  if (p.lut_n == 1) return p.lut_t[0];
  int lo = 0, hi = p.lut_n;
  while (lo < hi) {
    int mid = lo + (hi - lo) / 2;
    double v = p.lut_lat[mid];
    if (v < lat) lo = mid + 1;
    else if (v > lat) hi = mid;
    else return p.lut_t[mid];
  }
  if (lo == 0) return p.lut_t[0];
  if (lo >= p.lut_n) return p.lut_t[p.lut_n - 1];
  double frac = (lat - p.lut_lat[lo - 1]) / (p.lut_lat[lo] - p.lut_lat[lo - 1]);
  double dt_us = (double)(p.lut_t[lo] - p.lut_t[lo - 1]);
  return p.lut_t[lo - 1] + f2i64(frac * dt_us);
}

// ── K1 ─────────────────────────────────────────────────────────────────────

// ── K2 ─────────────────────────────────────────────────────────────────────
// ── orbit table ──────────────────────────────────────────────────────────────
__global__ void k_orbit_table(const sd_state_vector *svs, uint64_t n, int64_t t0, int64_t cnt,
                              double2 *tab) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= cnt) return;
  OrbitState s;
  orbit_eval(svs, n, t0 + i, &s);  // range is inside the state-vector window
  double2 *e = tab + 5 * i;
  e[0] = make_double2(s.pos.x, s.pos.y);
  e[1] = make_double2(s.pos.z, s.vel.x);
  e[2] = make_double2(s.vel.y, s.vel.z);
  e[3] = make_double2(s.acc.x, s.acc.y);
  e[4] = make_double2(s.acc.z, dot3(s.vel, s.vel));
}

#define SD_FOR_ITEMS(STAGE)                                                                  \
  const TcWork w = *wp;                                                                      \
  const uint64_t *pre = stage_pre(w, STAGE);                                                 \
  const uint64_t total = pre[w.n_jobs];                                                      \
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total;              \
       i += (uint64_t)gridDim.x * blockDim.x)

// Anchor li of job p: the exact inverse projection of its grid point and,
// for a UTM DEM, the forward projection's local expansion there.
__device__ __forceinline__ void anchor_item(const TcDev &p, uint64_t li) {
  const uint64_t r = li / p.n_pts, a = li % p.n_pts;
  double lon, lat;
  utm_xy_to_lonlat(p.proj, p.ax[a], row_y(p, r), &lon, &lat);
  ((double *)p.alon)[li] = lon;
  ((double *)p.alat)[li] = lat;
  if (p.aloc) {
    const Utm &u = p.dem.utm;
    utm_local(u, lat, utm_taup(u, lat), utm_lam(u, lon), (UtmLocal *)p.aloc + li);
  }
}

__global__ void k_row_anchors(const TcWork *__restrict__ wp) {
  SD_FOR_ITEMS(WK_ANCH) {
    const int j = find_job(pre, w.n_jobs, i);
    anchor_item(w.jobs[j], i - pre[j]);
  }
}

// Parameter form for one job: the projections' series coefficients sit in
// the parameter bank and enter the FP64 instructions as operands.
__global__ void k_row_anchors_param(TcDev p) {
  const uint64_t n = p.utm ? p.rows * (uint64_t)p.n_pts : 0;
  for (uint64_t li = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; li < n; li += (uint64_t)gridDim.x * blockDim.x)
    anchor_item(p, li);
}

__global__ void k_row_setup(const TcWork *__restrict__ wp) {
  SD_FOR_ITEMS(WK_ROWS) {
    const int j = find_job(pre, w.n_jobs, i);
    const TcDev &p = w.jobs[j];
    const uint64_t r = i - pre[j];
    if (r == 0) {  // the job's counters and flags start at zero
      for (int k = 0; k < kCounters + SD_NEWTON_ITER_HIST_SIZE; ++k) p.counters[k] = 0;
      for (int k = 0; k < 6; ++k) p.flags[k] = 0;
    }
    const double y = row_y(p, r);
    double lat_seed = y;
    if (p.utm) {
      double mid_x = p.lon_west + ((double)p.cols / 2.0) * p.sp;
      double lo;
      utm_xy_to_lonlat(p.proj, mid_x, y, &lo, &lat_seed);
    }
    p.row_guess[r] = guess_time(p, lat_seed);
    if (p.need_geom) {
      double ref_lon;
      if (p.utm) {
        double la;
        pixel_lonlat(p, r, p.cols / 2, &ref_lon, &la);
      } else {
        ref_lon = p.lon_west + ((double)p.cols / 2.0) * p.sp;
      }
      p.row_flat[r] = flat_cell_area(lat_seed, ref_lon, p.step_deg);
    }
  }
}

__device__ __forceinline__ uint64_t knot_col(const TcDev &p, int j) {
  return p.cols <= 1 ? 0 : (uint64_t)j * (p.cols - 1) / (KNOTS - 1);
}

// Coarse azimuth-time model: the reference iteration at KNOTS columns per
// row with the geoid surface (h = 0 orthometric).  Only a seed predictor.
__global__ void k_row_model(const TcWork *__restrict__ wp) {
  SD_FOR_ITEMS(WK_KNOT) {
    const int jb = find_job(pre, w.n_jobs, i);
    const TcDev &p = w.jobs[jb];
    const uint64_t li = i - pre[jb];
    const uint64_t r = li / KNOTS;
    const int j = (int)(li % KNOTS);
    const uint64_t c = knot_col(p, j);
    double lon, lat;
    pixel_lonlat(p, r, c, &lon, &lat);
    V3 P = geodetic_to_ecef(lat, lon, geoid_undulation(p.geoid, lat, lon));
    ZdRes z = newton(p.orb, P, p.row_guess[r], 40, 1e-6);
    if (z.st == ST_CONV) {
      p.knot_t[li] = z.t;
      if (p.trange) {
        unsigned long long b = (unsigned long long)z.t ^ 0x8000000000000000ull;
        atomicMin(&p.trange[0], b);
        atomicMax(&p.trange[1], b);
      }
    } else {
      p.knot_t[li] = INT64_MIN;
    }
  }
}

__device__ __forceinline__ int64_t predicted_time(const TcDev &p, uint64_t r, uint64_t c) {
  const int64_t *k = p.knot_t + r * KNOTS;
  if (p.cols <= 1) return k[0] != INT64_MIN ? k[0] : p.row_guess[r];
  int j = (int)((c * (KNOTS - 1)) / (p.cols - 1));
  if (j >= KNOTS - 1) j = KNOTS - 2;
  uint64_t c0 = knot_col(p, j), c1 = knot_col(p, j + 1);
  int64_t t0 = k[j], t1 = k[j + 1];
  if (t0 == INT64_MIN && t1 == INT64_MIN) return p.row_guess[r];
  if (t0 == INT64_MIN) return t1;
  if (t1 == INT64_MIN || c1 == c0) return t0;
  double f = (double)(c - c0) / (double)(c1 - c0);
  return t0 + (int64_t)llrint(f * (double)(t1 - t0));
}

// ── resampling (terrain_correction.rs:770-983) ───────────────────────────────
// One radar-image sample; n = lines x samples bounds it in SD_BOUNDS_CHECK builds.
__device__ __forceinline__ float ldf(const float *p, int64_t i, uint64_t n) {
  return SD_IN_BOUNDS(BS_IMAGE, i, n) ? __ldg(p + i) : __int_as_float(0x7fc00000);
}

__device__ float sample_bilinear(const float *d, uint64_t nl, uint64_t ns, double line, double sample) {
  int64_t max_line = nl == 0 ? 0 : (int64_t)nl - 1;
  int64_t max_sample = ns == 0 ? 0 : (int64_t)ns - 1;
  int64_t l0 = clampi(f2i64(floor(line)), 0, max_line);
  int64_t l1 = l0 + 1 < max_line ? l0 + 1 : max_line;
  int64_t s0 = clampi(f2i64(floor(sample)), 0, max_sample);
  int64_t s1 = s0 + 1 < max_sample ? s0 + 1 : max_sample;
  double dl = line - (double)l0;
  double ds = sample - (double)s0;
  float v00 = ldf(d, l0 * (int64_t)ns + s0, nl * ns), v01 = ldf(d, l0 * (int64_t)ns + s1, nl * ns);
  float v10 = ldf(d, l1 * (int64_t)ns + s0, nl * ns), v11 = ldf(d, l1 * (int64_t)ns + s1, nl * ns);
  if (v00 != v00 || v01 != v01 || v10 != v10 || v11 != v11) return NAN;
  double w00 = (1.0 - dl) * (1.0 - ds);
  double w01 = (1.0 - dl) * ds;
  double w10 = dl * (1.0 - ds);
  double w11 = dl * ds;
  return (float)((double)v00 * w00 + (double)v01 * w01 + (double)v10 * w10 + (double)v11 * w11);
}

__device__ float sample_bicubic(const float *d, uint64_t nl, uint64_t ns, double line, double sample) {
  int64_t max_l = (int64_t)nl - 1, max_s = (int64_t)ns - 1;
  int64_t lf = f2i64(floor(line)), sf = f2i64(floor(sample));
  double dl = line - (double)lf, ds = sample - (double)sf;
  double ws[4];
  int64_t cols[4];
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    ws[k] = keys_weight((double)(k - 1) - ds);
    cols[k] = clampi(sf + k - 1, 0, max_s);
  }
  double acc = 0.0;
#pragma unroll
  for (int li = -1; li <= 2; ++li) {
    int64_t row = clampi(lf + li, 0, max_l);
    double wl = keys_weight((double)li - dl);
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      float v = ldf(d, row * (int64_t)ns + cols[k], nl * ns);
      if (v != v) return NAN;
      acc += (double)v * wl * ws[k];
    }
  }
  return (float)acc;
}

// ── split precision (SD_PRECISION_SPLIT) ─────────────────────────────────────
// Everything that decides an integer outcome stays FP64: the orbit table,
// every Newton residual (so the microsecond chain, the converged times and
// the Newton histogram are those of the FP64 path), the target ECEF, the
// slant range, the image coordinates and the footprint test.  Resampling
// weights and sums, the NESZ sample, the facet normal (built from chords
// between the cardinal neighbours in a frame local to the pixel, never from
// absolute ECEF coordinates), cos(LIA) and the flattening weight run in FP32.
// A mask decision FP32 cannot settle (flattening weight within 1e-4
// relative of 0.05 or 2.0, local projection within 1e-4 of the facet area
// from zero, sigma0 within 1e-5 relative of the NESZ threshold) is redone
// with the FP64 candidate, so the mask equals the FP64 path's.
// The build compiles with --fmad=false (the FP64 path must not contract);
// the FP32 code contracts explicitly with fmaf.

// The fractional tap position f and its complement g = 1 - f, both formed in
// FP64 and then rounded, so each carries its own relative accuracy.  Weights
// that vanish as f -> 1 are proportional to g; a g formed in FP32 from the
// rounded f carries f's absolute error (2^-25) and loses its relative
// accuracy there, which the error bound below does not allow for.
struct FracF {
  float f, g;
};
__device__ __forceinline__ FracF frac_f(double x, int64_t base) {
  const double fd = x - (double)base;
  return {(float)fd, (float)(1.0 - fd)};
}

// keys_weight (a = -0.5) of the taps -1, 0, 1, 2 at offsets k - f, in
// factored form: 1.5u^3 - 2.5u^2 + 1 = (1 - u)(1 + u - 1.5u^2) on [0, 1) and
// -0.5u^3 + 2.5u^2 - 4u + 2 = -0.5(u - 1)(u - 2)^2 on [1, 2).  Expanded, the
// cubics cancel near their roots and a small weight loses its leading
// digits; factored, every weight keeps its relative accuracy.
__device__ __forceinline__ void keys4_f(FracF q, float w[4]) {
  const float f = q.f, g = q.g;
  w[0] = -0.5f * f * g * g;
  w[1] = g * fmaf(-1.5f * f, f, 1.f + f);
  w[2] = f * fmaf(-1.5f * g, g, 1.f + g);
  w[3] = -0.5f * g * f * f;
}

// Lanczos-3 weights (terrain_correction.rs:938-952) of the taps li = -2..3
// at x = f - li.  sin(pi x) = (-1)^li sin(pi f) and sin(pi x/3) =
// sin(pi f/3) cos(pi li/3) - cos(pi f/3) sin(pi li/3), so the six weights
// take two sinpi and one sincospi.  In FP32 every factor that vanishes as
// f -> 1 is taken from g = 1 - f (sin(pi f) = sin(pi g), x = f - 1 = -g).
template <typename T>
__device__ __forceinline__ void lanczos6(double fd, T w[6]);

template <>
__device__ __forceinline__ void lanczos6<float>(double fd, float w[6]) {
  const float f = (float)fd, g = (float)(1.0 - fd);
  const float s1 = sinpif(f <= 0.5f ? f : g);
  float s3, c3;
  sincospif(f * (1.f / 3.f), &s3, &c3);
  const float q = sinpif(g * (1.f / 3.f));
  const float h = 0.866025403784438647f;  // sin(pi/3)
  const float cl[6] = {-0.5f, 0.5f, 1.f, 0.5f, -0.5f, -1.f};
  const float sl[6] = {-h, -h, 0.f, h, h, 0.f};
  const float k = (float)(3.0 / (kPi * kPi));
#pragma unroll
  for (int j = 0; j < 6; ++j) {
    const int li = j - 2;
    const float x = li == 1 ? -g : f - (float)li;
    const float ax = fabsf(x);
    const float s = (li & 1) ? -s1 : s1;
    // taps li = -2 and 1: the angle-addition form cancels as f -> 1, so
    // their sines are taken directly, sin(pi(f+2)/3) = -sin(pi(f-1)/3) = q
    const float s3l = li == 1 ? -q : (li == -2 ? q : s3 * cl[j] - c3 * sl[j]);
    w[j] = ax < 1e-10f ? 1.f : (ax < 3.f ? k * s * s3l / (x * x) : 0.f);
  }
}

template <>
__device__ __forceinline__ void lanczos6<double>(double f, double w[6]) {
  const double s1 = sinpi(f);
  double s3, c3;
  sincospi(f * (1.0 / 3.0), &s3, &c3);
  const double q = sinpi((1.0 - f) * (1.0 / 3.0));
  const double h = 0.86602540378443864676;
  const double cl[6] = {-0.5, 0.5, 1.0, 0.5, -0.5, -1.0};
  const double sl[6] = {-h, -h, 0.0, h, h, 0.0};
  const double k = 3.0 / (kPi * kPi);
#pragma unroll
  for (int j = 0; j < 6; ++j) {
    const int li = j - 2;
    const double x = f - (double)li;
    const double ax = fabs(x);
    const double s = (li & 1) ? -s1 : s1;
    const double s3l = li == 1 ? -q : (li == -2 ? q : s3 * cl[j] - c3 * sl[j]);
    w[j] = ax < 1e-10 ? 1.0 : (ax < 3.0 ? k * s * s3l / (x * x) : 0.0);
  }
}

// The FP32 samplers also return the magnitude sum A = sum |v w|.  Their
// error is at most kSampErr * A: two nested fma chains of <= 6 terms
// (12 u of A) plus the FP32 weights' own rounding (a few ulps each, 2e-6 for
// a weight product).  That needs every weight to keep its relative accuracy,
// so the weights are formed from f and g = 1 - f each rounded from FP64
// (frac_f): a weight proportional to g is then exact to a few ulps also as
// f -> 1.  The bound travels with the value (CandPre::serr) to
// the mask decisions, so an inexact sum (negative lobes cancelling) costs an
// FP64 re-sample only where it can change the output: a valid pixel whose
// bound exceeds kSampRel of its value, or a noise-floor test within it.
constexpr float kSampErr = 4e-6f;
constexpr float kSampRel = 5e-5f;

// cand_post_f outcomes: settled; the whole candidate again in FP64 (a mask
// decision within its FP32 margin: k_redo); only the value in FP64 (the
// image coordinates and flattening weight are queued for k_resample).
enum { RD_NONE = 0, RD_FULL = 1, RD_SAMPLE = 2 };
struct RsEnt {
  double line, sample;  // FP64 image coordinates of the candidate
  float wdiv;           // flattening weight the value is divided by (1: none)
  uint32_t thread;      // pixel within the k_cand item (0..255)
};
constexpr int RS_CAP = 64;  // queued re-samples per k_cand item (beyond: k_redo)

__device__ float sample_bilinear_f(const float *d, uint64_t nl, uint64_t ns, double line, double sample,
                                   float *amag) {
  int64_t max_line = nl == 0 ? 0 : (int64_t)nl - 1;
  int64_t max_sample = ns == 0 ? 0 : (int64_t)ns - 1;
  int64_t l0 = clampi(f2i64(floor(line)), 0, max_line);
  int64_t l1 = l0 + 1 < max_line ? l0 + 1 : max_line;
  int64_t s0 = clampi(f2i64(floor(sample)), 0, max_sample);
  int64_t s1 = s0 + 1 < max_sample ? s0 + 1 : max_sample;
  // dl may be negative (line in [-0.5, 0)) or beyond 1 at the far edge
  const FracF ql = frac_f(line, l0), qs = frac_f(sample, s0);
  const float dl = ql.f, ds = qs.f;
  float v00 = ldf(d, l0 * (int64_t)ns + s0, nl * ns), v01 = ldf(d, l0 * (int64_t)ns + s1, nl * ns);
  float v10 = ldf(d, l1 * (int64_t)ns + s0, nl * ns), v11 = ldf(d, l1 * (int64_t)ns + s1, nl * ns);
  if (v00 != v00 || v01 != v01 || v10 != v10 || v11 != v11) return NAN;
  // explicit weights, as the reference forms them: with non-negative
  // weights and samples every term is non-negative and the sum keeps its
  // relative accuracy even near zero (the lerp form a + t(b - a) does not)
  const float w00 = ql.g * qs.g, w01 = ql.g * ds;
  const float w10 = dl * qs.g, w11 = dl * ds;
  const float r = fmaf(v00, w00, fmaf(v01, w01, fmaf(v10, w10, v11 * w11)));
  const float a = fmaf(fabsf(v00), fabsf(w00), fmaf(fabsf(v01), fabsf(w01),
                       fmaf(fabsf(v10), fabsf(w10), fabsf(v11) * fabsf(w11))));
  *amag = a;
  return r;
}

__device__ float sample_bicubic_f(const float *d, uint64_t nl, uint64_t ns, double line, double sample,
                                  float *amag) {
  int64_t max_l = (int64_t)nl - 1, max_s = (int64_t)ns - 1;
  int64_t lf = f2i64(floor(line)), sf = f2i64(floor(sample));
  float ws[4], wls[4];
  keys4_f(frac_f(sample, sf), ws);
  keys4_f(frac_f(line, lf), wls);
  int64_t cols[4];
#pragma unroll
  for (int k = 0; k < 4; ++k) cols[k] = clampi(sf + k - 1, 0, max_s);
  float acc = 0.f, aacc = 0.f;
#pragma unroll
  for (int li = -1; li <= 2; ++li) {
    int64_t row = clampi(lf + li, 0, max_l);
    const float wl = wls[li + 1];
    float racc = 0.f, rabs = 0.f;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      float v = ldf(d, row * (int64_t)ns + cols[k], nl * ns);
      if (v != v) return NAN;
      racc = fmaf(v, ws[k], racc);
      rabs = fmaf(fabsf(v), fabsf(ws[k]), rabs);
    }
    acc = fmaf(racc, wl, acc);
    aacc = fmaf(rabs, fabsf(wl), aacc);
  }
  *amag = aacc;
  return acc;
}

template <typename T>
__device__ float sample_lanczos_t(const float *d, uint64_t nl, uint64_t ns, double line, double sample,
                                  float *amag) {
  int64_t max_l = (int64_t)nl - 1, max_s = (int64_t)ns - 1;
  int64_t lf = f2i64(floor(line)), sf = f2i64(floor(sample));
  T wl[6], ws[6];
  lanczos6<T>(line - (double)lf, wl);
  lanczos6<T>(sample - (double)sf, ws);
  int64_t cols[6];
#pragma unroll
  for (int k = 0; k < 6; ++k) cols[k] = clampi(sf + k - 2, 0, max_s);
  T acc = 0, aacc = 0;
#pragma unroll
  for (int j = 0; j < 6; ++j) {
    int64_t row = clampi(lf + j - 2, 0, max_l);
    T racc = 0, rabs = 0;
#pragma unroll
    for (int k = 0; k < 6; ++k) {
      float v = ldf(d, row * (int64_t)ns + cols[k], nl * ns);
      if (v != v) return NAN;
      racc += (T)v * ws[k];
      if (amag) rabs += fabs((T)v * ws[k]);
    }
    acc += racc * wl[j];
    if (amag) aacc += rabs * fabs(wl[j]);
  }
  if (amag) *amag = (float)aacc;
  return (float)acc;
}

// KDYN: the resampling kernel is read from the job record (batches whose
// tiles mix kernels); 0..2 fix it at compile time.
constexpr int KDYN = 3;

template <int KERNEL>
__device__ __forceinline__ float resample_f(const TcDev &p, double line, double sample, float *amag) {
  if (KERNEL == KDYN) {
    switch (p.resampling) {
      case SD_RESAMPLE_BICUBIC: return sample_bicubic_f(p.img, p.lines, p.samples, line, sample, amag);
      case SD_RESAMPLE_LANCZOS3: return sample_lanczos_t<float>(p.img, p.lines, p.samples, line, sample, amag);
      default: return sample_bilinear_f(p.img, p.lines, p.samples, line, sample, amag);
    }
  }
  return KERNEL == SD_RESAMPLE_BICUBIC    ? sample_bicubic_f(p.img, p.lines, p.samples, line, sample, amag)
         : KERNEL == SD_RESAMPLE_LANCZOS3 ? sample_lanczos_t<float>(p.img, p.lines, p.samples, line, sample, amag)
                                          : sample_bilinear_f(p.img, p.lines, p.samples, line, sample, amag);
}

template <int KERNEL>
__device__ __forceinline__ float resample(const TcDev &p, double line, double sample) {
  if (KERNEL == KDYN) {
    switch (p.resampling) {
      case SD_RESAMPLE_BICUBIC: return sample_bicubic(p.img, p.lines, p.samples, line, sample);
      case SD_RESAMPLE_LANCZOS3: return sample_lanczos_t<double>(p.img, p.lines, p.samples, line, sample, nullptr);
      default: return sample_bilinear(p.img, p.lines, p.samples, line, sample);
    }
  }
  return KERNEL == SD_RESAMPLE_BICUBIC    ? sample_bicubic(p.img, p.lines, p.samples, line, sample)
         : KERNEL == SD_RESAMPLE_LANCZOS3 ? sample_lanczos_t<double>(p.img, p.lines, p.samples, line, sample, nullptr)
                                          : sample_bilinear(p.img, p.lines, p.samples, line, sample);
}

// ── per-pixel geometry ───────────────────────────────────────────────────────
// Centre of output pixel (r, c): lat/lon, DEM height and target ECEF.  The
// sines/cosines and projection terms are kept for the neighbour lookups.
struct PixGeo {
  double lat, lon;
  double la, lo;              // radians as geodesy.rs:39-40 converts them
  double sla, cla, slo, clo;  // their sines and cosines
  UtmLocal loc;               // UTM DEM: projection of the centre and its local expansion
  V3 P;
};

// DEM lookup of the centre (1529-1536), geoid (1545) and target ECEF (1546).
// Returns false when the DEM has no finite height there.
// Centre of the pixel: lon/lat, the UTM local expansion for a projected DEM,
// and the DEM height; false when there is no finite height.
__device__ __forceinline__ bool pixel_height(const TcDev &p, uint64_t r, uint64_t c, PixGeo *g, float *hf) {
  int seg;
  double t;
  pixel_seg(p, r, c, &g->lon, &g->lat, &seg, &t);
  bool ok;
  if (p.dem.kind == SD_DEM_PROJECTED_UTM) {
    const Utm &u = p.dem.utm;
    if (p.aloc) dem_local_from_anchors(p, r, seg, t, &g->loc);
    else utm_local(u, g->lat, utm_taup(u, g->lat), utm_lam(u, g->lon), &g->loc);
    ok = dem_at_xy_checked(p.dem, g->loc.x, g->loc.y, g->lat, g->lon, hf);
  } else {
    ok = dem_at_lonlat_checked(p.dem, g->lon, g->lat, hf);
  }
  return ok && isfinite(*hf);
}

// Geoid, sines and cosines and the target ECEF from the centre height.
__device__ __forceinline__ void pixel_ecef(const TcDev &p, PixGeo *g, float hf) {
  double h_ell = (double)hf + geoid_undulation(p.geoid, g->lat, g->lon);
  g->la = deg2rad_ecef(g->lat);
  g->lo = deg2rad_ecef(g->lon);
  crm::sincos(g->la, &g->sla, &g->cla);  // correctly rounded (crmath.cuh)
  crm::sincos(g->lo, &g->slo, &g->clo);
  g->P = ecef_sc(g->sla, g->cla, g->slo, g->clo, h_ell);
}

// pixel_height with decided lookups only: 1 = a finite height, 0 = none
// (outside the DEM or a void), -1 = the lookup is undecided.
__device__ __forceinline__ int pixel_height_try(const TcDev &p, uint64_t r, uint64_t c, PixGeo *g, float *hf) {
  int seg;
  double t;
  pixel_seg(p, r, c, &g->lon, &g->lat, &seg, &t);
  int st;
  if (p.dem.kind == SD_DEM_PROJECTED_UTM) {
    const Utm &u = p.dem.utm;
    if (p.aloc) dem_local_from_anchors(p, r, seg, t, &g->loc);
    else utm_local(u, g->lat, utm_taup(u, g->lat), utm_lam(u, g->lon), &g->loc);
    st = dem_at_xy_try(p.dem, g->loc.x, g->loc.y, hf);
  } else {
    st = dem_at_lonlat_try(p.dem, g->lon, g->lat, hf);
  }
  if (st < 0) return -1;
  return st > 0 && isfinite(*hf) ? 1 : 0;
}

__device__ bool pixel_geo(const TcDev &p, uint64_t r, uint64_t c, PixGeo *g) {
  float hf;
  if (!pixel_height(p, r, c, g, &hf)) return false;
  pixel_ecef(p, g, hf);
  return true;
}

// Facet of the four cardinal DEM neighbours (1642-1675): normal and area.
// The neighbours sit step_deg from the centre, so their projected
// coordinates come from the centre's local expansion and their sines and
// cosines from angle addition over the exact argument differences.
struct Facet {
  bool ok;
  V3 normal;
  double area;
};

// Heights of the east, west, north and south neighbours (1642-1675: DEM
// heights without the geoid); false when any lies outside the DEM or on a void.
__device__ __forceinline__ bool facet_heights(const TcDev &p, const PixGeo &g, float h[4]) {
  const double sd = p.step_deg;
  const double lon_e = g.lon + sd, lon_w = g.lon - sd, lat_n = g.lat + sd, lat_s = g.lat - sd;
  float he, hw, hn, hs;
  bool ok;
  if (p.dem.kind == SD_DEM_PROJECTED_UTM) {
    const Utm &u = p.dem.utm;
    const double k = kPi / 180.0;
    double x, y;
    utm_local_step(u, g.loc, 0.0, (lon_e - g.lon) * k, &x, &y);
    ok = dem_at_xy_checked(p.dem, x, y, g.lat, lon_e, &he);
    utm_local_step(u, g.loc, 0.0, (lon_w - g.lon) * k, &x, &y);
    ok = dem_at_xy_checked(p.dem, x, y, g.lat, lon_w, &hw) && ok;
    utm_local_step(u, g.loc, (lat_n - g.lat) * k, 0.0, &x, &y);
    ok = dem_at_xy_checked(p.dem, x, y, lat_n, g.lon, &hn) && ok;
    utm_local_step(u, g.loc, (lat_s - g.lat) * k, 0.0, &x, &y);
    ok = dem_at_xy_checked(p.dem, x, y, lat_s, g.lon, &hs) && ok;
  } else {
    ok = dem_at_lonlat_checked(p.dem, lon_e, g.lat, &he);
    ok = dem_at_lonlat_checked(p.dem, lon_w, g.lat, &hw) && ok;
    ok = dem_at_lonlat_checked(p.dem, g.lon, lat_n, &hn) && ok;
    ok = dem_at_lonlat_checked(p.dem, g.lon, lat_s, &hs) && ok;
  }
  h[0] = he, h[1] = hw, h[2] = hn, h[3] = hs;
  return ok && isfinite(he) && isfinite(hw) && isfinite(hn) && isfinite(hs);
}

// facet_heights with decided lookups only: 1 = four finite heights, 0 = a
// neighbour outside the DEM or on a void, -1 = a lookup is undecided.
__device__ __forceinline__ int facet_heights_try(const TcDev &p, const PixGeo &g, float h[4]) {
  const double sd = p.step_deg;
  const double lon_e = g.lon + sd, lon_w = g.lon - sd, lat_n = g.lat + sd, lat_s = g.lat - sd;
  int s[4];
  if (p.dem.kind == SD_DEM_PROJECTED_UTM) {
    const Utm &u = p.dem.utm;
    const double k = kPi / 180.0;
    double x, y;
    utm_local_step(u, g.loc, 0.0, (lon_e - g.lon) * k, &x, &y);
    s[0] = dem_at_xy_try(p.dem, x, y, &h[0]);
    utm_local_step(u, g.loc, 0.0, (lon_w - g.lon) * k, &x, &y);
    s[1] = dem_at_xy_try(p.dem, x, y, &h[1]);
    utm_local_step(u, g.loc, (lat_n - g.lat) * k, 0.0, &x, &y);
    s[2] = dem_at_xy_try(p.dem, x, y, &h[2]);
    utm_local_step(u, g.loc, (lat_s - g.lat) * k, 0.0, &x, &y);
    s[3] = dem_at_xy_try(p.dem, x, y, &h[3]);
  } else {
    s[0] = dem_at_lonlat_try(p.dem, lon_e, g.lat, &h[0]);
    s[1] = dem_at_lonlat_try(p.dem, lon_w, g.lat, &h[1]);
    s[2] = dem_at_lonlat_try(p.dem, g.lon, lat_n, &h[2]);
    s[3] = dem_at_lonlat_try(p.dem, g.lon, lat_s, &h[3]);
  }
  if (s[0] < 0 || s[1] < 0 || s[2] < 0 || s[3] < 0) return -1;
  return s[0] > 0 && s[1] > 0 && s[2] > 0 && s[3] > 0 && isfinite(h[0]) && isfinite(h[1]) && isfinite(h[2]) &&
                 isfinite(h[3])
             ? 1
             : 0;
}

// Normal and area of the facet from the four neighbour heights.
__device__ Facet facet_from(const TcDev &p, const PixGeo &g, const float h[4]) {
  Facet f{};
  f.ok = true;
  const float he = h[0], hw = h[1], hn = h[2], hs = h[3];
  const double sd = p.step_deg;
  const double lon_e = g.lon + sd, lon_w = g.lon - sd, lat_n = g.lat + sd, lat_s = g.lat - sd;
#if SD_FACET_ABSOLUTE
  // the reference's form: four absolute ECEF points, then their differences
  double se, ce, sw, cw, sn, cn, ss, cs;
  sincos_add(g.slo, g.clo, deg2rad_ecef(lon_e) - g.lo, &se, &ce);
  sincos_add(g.slo, g.clo, deg2rad_ecef(lon_w) - g.lo, &sw, &cw);
  sincos_add(g.sla, g.cla, deg2rad_ecef(lat_n) - g.la, &sn, &cn);
  sincos_add(g.sla, g.cla, deg2rad_ecef(lat_s) - g.la, &ss, &cs);
  V3 pe = ecef_sc(g.sla, g.cla, se, ce, (double)he);
  V3 pw = ecef_sc(g.sla, g.cla, sw, cw, (double)hw);
  V3 pn = ecef_sc(sn, cn, g.slo, g.clo, (double)hn);
  V3 ps = ecef_sc(ss, cs, g.slo, g.clo, (double)hs);
  f.normal = cross3(sub3(pe, pw), sub3(pn, ps));
#else
  // The same two chords pe - pw and pn - ps, expanded about the centre in
  // the angular steps a, b (east, west) and c, d (north, south), ~1.6e-6
  // rad, through second order (the third-order terms are ~1e-11 m on ~20 m
  // chords).  The reference subtracts absolute ECEF coordinates of ~6.4e6 m,
  // which already costs it ~3e-11 of relative precision, so the two forms
  // agree to the reference's own rounding; this one needs no square root or
  // division per neighbour.
  const double a = deg2rad_ecef(lon_e) - g.lo, b = g.lo - deg2rad_ecef(lon_w);
  const double c = deg2rad_ecef(lat_n) - g.la, d = g.la - deg2rad_ecef(lat_s);
  const double sp = g.sla, cp = g.cla, sl = g.slo, cl = g.clo;
  const double den = 1.0 - WGS84_E2 * sp * sp;
  const double N = WGS84_A / sqrt(den);
  const double dN = N * WGS84_E2 * sp * cp / den;
  const double B = N * (1.0 - WGS84_E2), dB = dN * (1.0 - WGS84_E2);
  const double Hn = (double)hn, Hs = (double)hs, He = (double)he, Hw = (double)hw;
  // east-west: (N + h) cos(phi) (cos, sin)(lam +- step), (B + h) sin(phi)
  const double dh = He - Hw;
  const double q = (N + He) * a + (N + Hw) * b;
  const double r2 = 0.5 * ((N + He) * a * a - (N + Hw) * b * b);
  const V3 e = {cp * (cl * dh - sl * q - cl * r2), cp * (sl * dh + cl * q - sl * r2), sp * dh};
  // north-south: G(phi) = N cos(phi), Z(phi) = B sin(phi) and the heights
  const double dv = Hn - Hs, h2 = 0.5 * (Hn * c * c - Hs * d * d);
  const double An = cp * (dv + dN * (c + d)) - sp * ((N + Hn) * c + (N + Hs) * d) - cp * h2;
  const double Zn = sp * (dv + dB * (c + d)) + cp * ((B + Hn) * c + (B + Hs) * d) - sp * h2;
  f.normal = cross3(e, V3{cl * An, sl * An, Zn});
#endif
  f.area = norm3(f.normal);
  return f;
}

__device__ Facet pixel_facet(const TcDev &p, const PixGeo &g) {
  float h[4];
  if (!facet_heights(p, g, h)) return Facet{};
  return facet_from(p, g, h);
}

// Output of one pixel for one converged azimuth time (1585-1739): sigma0 /
// gamma0, cos(LIA), mask code and counter class (0 valid, 2 outside
// footprint, 5 flat-masked, 6 noise-masked).
struct CandOut {
  float data, cos;
  uint8_t mask, cls;
};

struct CandPre {  // steps 4-6 of the reference loop for one candidate
  double line, sample;
  float sigma0;
  float serr;  // bound on |sigma0 - FP64 value| (0 when sampled in FP64)
  bool inside;
};

// Slant range, image coordinates and the footprint test (745-760).
__device__ __forceinline__ CandPre cand_geom(const TcDev &p, V3 P, V3 S, int64_t t) {
  CandPre c;
  double slant = norm3(sub3(P, S));
  double dt = (double)(t - p.az_start) / 1e6;
  c.line = dt / p.ati;
  c.sample = (slant - p.near_range) / p.rps;
  c.inside = !(c.line < -0.5 || c.line > ((double)p.lines - 0.5) || c.sample < -0.5 ||
               c.sample > ((double)p.samples - 0.5));
  c.sigma0 = NAN;
  c.serr = 0.f;
  return c;
}

template <int KERNEL, bool SPLIT>
__device__ CandPre cand_pre(const TcDev &p, V3 P, V3 S, int64_t t) {
  CandPre c = cand_geom(p, P, S, t);
  if (c.inside) {
    if (SPLIT) {
      float amag = 0.f;
      c.sigma0 = resample_f<KERNEL>(p, c.line, c.sample, &amag);
      c.serr = kSampErr * amag;
    } else {
      c.sigma0 = resample<KERNEL>(p, c.line, c.sample);
    }
  } else {
    c.sigma0 = NAN;
  }
  if (c.sigma0 != c.sigma0) c.inside = false;
  return c;
}

__device__ CandOut cand_post(const TcDev &p, const CandPre &c, V3 P, V3 S, const Facet &f, double flat_area) {
  CandOut o{NAN, NAN, SD_MASK_OUTSIDE_FOOTPRINT, 2};
  if (!c.inside) return o;
  float sigma0 = c.sigma0;
  uint8_t m = SD_MASK_OUTSIDE_FOOTPRINT;
  float cosv = NAN;
  if (p.need_geom) {
    if (!f.ok) {
      m = SD_MASK_DEM_NEIGHBOUR_MISSING;
      if (p.flatten) return {NAN, cosv, m, 5};
    } else {
      V3 look = normalize3(sub3(S, P));
      double local_proj = dot3(f.normal, look);
      if (local_proj <= 0.0 || f.area == 0.0) {
        m = SD_MASK_SHADOW;
        if (p.flatten) return {NAN, cosv, m, 5};
      } else {
        double cl = clampd(local_proj / f.area, 0.0, 1.0);
        double w = local_proj / flat_area;
        cosv = (float)cl;
        if (w < 0.05 || w > 2.0) {
          m = w > 2.0 ? SD_MASK_LAYOVER : SD_MASK_FORESHORTENING;
          if (p.flatten) return {NAN, cosv, m, 5};
        } else if (p.flatten) {
          sigma0 /= (float)w;
        }
      }
    }
  }
  if (p.nesz_mask) {
    float nz = sample_bilinear(p.nesz, p.lines, p.samples, c.line, c.sample);
    if (nz == nz) {
      float thr = nz * p.nesz_factor;
      if (sigma0 <= thr) return {NAN, cosv, (uint8_t)SD_MASK_NOISE_MASKED, 6};
    }
  }
  return {sigma0, cosv, (uint8_t)SD_MASK_VALID, 0};
}

// Facet in FP32: the east-west and north-south chords between the cardinal
// neighbours, expanded about the centre (latitude phi, longitude lam,
// prime-vertical radius N(phi)) to first order in the angular steps a, b, c,
// d (~1.6e-6 rad); the dropped terms are below 1e-7 m on chords of ~20 m.
//   E-W: cos(phi) (cos(lam) dh - sin(lam) q, sin(lam) dh + cos(lam) q),
//        sin(phi) dh,  dh = he - hw, q = (N + he) a + (N + hw) b
//   N-S: (cos(lam) An, sin(lam) An, Zn) with
//        An = cos(phi) (hn - hs + N'(c + d)) - sin(phi) ((N + hn) c + (N + hs) d)
//        Zn = sin(phi) (hn - hs + B'(c + d)) + cos(phi) ((B + hn) c + (B + hs) d)
//        B = N (1 - e^2), N' = dN/dphi = N e^2 sin cos / (1 - e^2 sin^2).
// en = |E-W chord| x |N-S chord| scales the normal's rounding error: every
// component of the FP32 cross product is within ~10 u en of the exact one
// (u = 2^-24), so the local projection lp = n . look is within
// kLpErr * en + kLpRel * |lp| of its FP64 value.
struct FacetF {
  bool ok;
  float nx, ny, nz, area, en;
};
constexpr float kLpErr = 1e-6f;   // ~16 u, plus the chord expansion's ~1e-8
constexpr float kLpRel = 4e-7f;   // look vector and its rsqrt
constexpr float kWRelFull = 2e-5f;  // beyond: the flattening weight itself is redone in FP64

__device__ FacetF facetf_from(const TcDev &p, const PixGeo &g, const float h[4]) {
  FacetF f{};
  f.ok = true;
  const float he = h[0], hw = h[1], hn = h[2], hs = h[3];
  const double sd = p.step_deg;
  const double lon_e = g.lon + sd, lon_w = g.lon - sd, lat_n = g.lat + sd, lat_s = g.lat - sd;
  const float a = (float)(deg2rad_ecef(lon_e) - g.lo), b = (float)(g.lo - deg2rad_ecef(lon_w));
  const float c = (float)(deg2rad_ecef(lat_n) - g.la), d = (float)(g.la - deg2rad_ecef(lat_s));
  const float sp = (float)g.sla, cp = (float)g.cla, sl = (float)g.slo, cl = (float)g.clo;
  const float e2 = (float)WGS84_E2;
  const float den = 1.f - e2 * sp * sp;
  const float N = (float)WGS84_A * rsqrtf(den);
  const float dN = N * e2 * sp * cp / den;
  const float B = N * (1.f - e2), dB = dN * (1.f - e2);
  const float dh = he - hw;
  const float q = fmaf(N + he, a, (N + hw) * b);
  const float ex = cp * (cl * dh - sl * q), ey = cp * (sl * dh + cl * q), ez = sp * dh;
  const float dv = hn - hs;
  const float An = cp * fmaf(dN, c + d, dv) - sp * fmaf(N + hn, c, (N + hs) * d);
  const float nx = cl * An, ny = sl * An;
  const float nz = sp * fmaf(dB, c + d, dv) + cp * fmaf(B + hn, c, (B + hs) * d);
  f.nx = ey * nz - ez * ny;
  f.ny = ez * nx - ex * nz;
  f.nz = ex * ny - ey * nx;
  f.area = sqrtf(f.nx * f.nx + f.ny * f.ny + f.nz * f.nz);
  f.en = sqrtf((ex * ex + ey * ey + ez * ez) * (nx * nx + ny * ny + nz * nz));
  return f;
}

__device__ FacetF pixel_facet_f(const TcDev &p, const PixGeo &g) {
  float h[4];
  if (!facet_heights(p, g, h)) return FacetF{};
  return facetf_from(p, g, h);
}

// cand_post in split precision; *redo is set when a mask decision falls
// inside the FP32 error margin and the FP64 candidate must decide.
__device__ CandOut cand_post_f(const TcDev &p, const CandPre &c, V3 P, V3 S, const FacetF &f,
                               float flat_area, int *redo, float *wdiv) {
  CandOut o{NAN, NAN, SD_MASK_OUTSIDE_FOOTPRINT, 2};
  *redo = RD_NONE;
  if (!c.inside) return o;
  float sigma0 = c.sigma0, serr = c.serr, wd = 1.f;
  float cosv = NAN;
  if (p.need_geom) {
    if (!f.ok) {
      if (p.flatten) return {NAN, cosv, (uint8_t)SD_MASK_DEM_NEIGHBOUR_MISSING, 5};
    } else {
      const float lx = (float)(S.x - P.x), ly = (float)(S.y - P.y), lz = (float)(S.z - P.z);
      const float il = rsqrtf(lx * lx + ly * ly + lz * lz);
      const float lp = (f.nx * lx + f.ny * ly + f.nz * lz) * il;
      const float dlp = kLpErr * f.en + kLpRel * fabsf(lp);  // bound on |lp - lp_fp64|
      if (fabsf(lp) <= fmaxf(1e-4f * f.area, 8.f * dlp)) { *redo = RD_FULL; return o; }
      if (lp <= 0.f || f.area == 0.f) {
        if (p.flatten) return {NAN, cosv, (uint8_t)SD_MASK_SHADOW, 5};
      } else {
        const float w = lp / flat_area;
        // relative error of w: that of lp, the division and flat_area's rounding
        const float ew = dlp / lp + 2.4e-7f;
        if (fabsf(w - 0.05f) <= 0.05f * fmaxf(1e-4f, 4.f * ew) ||
            fabsf(w - 2.0f) <= 2.0f * fmaxf(1e-4f, 4.f * ew)) {
          *redo = RD_FULL;
          return o;
        }
        cosv = fminf(fmaxf(lp / f.area, 0.f), 1.f);
        if (w < 0.05f || w > 2.0f) {
          if (p.flatten) return {NAN, cosv, (uint8_t)(w > 2.0f ? SD_MASK_LAYOVER : SD_MASK_FORESHORTENING), 5};
        } else if (p.flatten) {
          sigma0 /= w;
          // gamma0 = sigma0 / w: the sampling bound scales by 1 / w and the
          // weight's own relative error adds; a weight too inexact to be
          // reused by the FP64 re-sample sends the candidate to k_redo
          serr = serr / w + fabsf(sigma0) * ew;
          wd = w;
          if (ew > kWRelFull && serr > kSampRel * fabsf(sigma0)) { *redo = RD_FULL; return o; }
        }
      }
    }
  }
  const bool sample_ok = serr <= kSampRel * fabsf(sigma0);
  if (p.nesz_mask) {
    // NESZ is non-negative, so its bilinear sum is accurate to a few ulps
    float nz_mag;
    float nz = sample_bilinear_f(p.nesz, p.lines, p.samples, c.line, c.sample, &nz_mag);
    if (nz == nz) {
      float thr = nz * p.nesz_factor;
      if (fabsf(sigma0 - thr) > serr + 1e-5f * (fabsf(thr) + nz_mag * fabsf(p.nesz_factor))) {
        if (sigma0 <= thr) return {NAN, cosv, (uint8_t)SD_MASK_NOISE_MASKED, 6};
      } else if (sample_ok) {
        *redo = RD_FULL;  // the threshold test itself is marginal
        return o;
      }
    }
  }
  if (!sample_ok) {  // geometry settled; the value (and a NESZ test) wait for the FP64 re-sample
    *redo = RD_SAMPLE;
    *wdiv = wd;
    o.cos = cosv;
    return o;
  }
  return {sigma0, cosv, (uint8_t)SD_MASK_VALID, 0};
}

// One candidate's output from scratch (exact-path pixels, and split-precision
// candidates whose mask FP32 cannot settle).
// h4: the neighbour heights when already known (NaN when the facet is
// missing), else null to look them up.
__device__ __forceinline__ bool heights_ok(const float *h4) {
  return isfinite(h4[0]) && isfinite(h4[1]) && isfinite(h4[2]) && isfinite(h4[3]);
}

// One candidate's output in FP64 from the stored target and facet.
template <int KERNEL>
__device__ CandOut cand_fp64_tf(const TcDev &p, V3 P, const Facet &f, V3 S, int64_t t, double flat_area) {
  CandPre pre = cand_pre<KERNEL, false>(p, P, S, t);
  return cand_post(p, pre, P, S, f, flat_area);
}

template <int KERNEL>
__device__ CandOut cand_fp64(const TcDev &p, const PixGeo &g, V3 S, int64_t t, double flat_area,
                             const float *h4) {
  CandPre pre = cand_pre<KERNEL, false>(p, g.P, S, t);
  Facet f{};
  if (pre.inside && p.need_geom) f = h4 ? (heights_ok(h4) ? facet_from(p, g, h4) : Facet{}) : pixel_facet(p, g);
  return cand_post(p, pre, g.P, S, f, flat_area);
}

// ── per-pixel stores ─────────────────────────────────────────────────────────
// fb: the base of the fixed-point pair F = {fb, fb+1} (k_main), or the
// converged time of an exact-path pixel (k_scan).  cc: codes (outcome of the
// reference iteration seeded at each member of the left neighbour's F), F
// membership and flags.
enum : uint32_t { CF_DEMMISS = 1u << 18, CF_HASF = 1u << 19, CF_CODES = 1u << 20 /* F and codes recorded */,
                  CF_REDO = 1u << 21 /* split: outputs to be redone in FP64 (k_redo) */ };
// sel byte written by the scan: low 3 bits = outcome, high 4 bits = iterations
enum : uint8_t { SEL_M0 = 0, SEL_M1 = 1, SEL_DONE = 2, SEL_NONCONV = 3, SEL_DEGEN = 4, SEL_DEMMISS = 5,
                 SEL_ORBIT = 6 };

struct Ent {  // one orbit-table record
  double px, py, pz, vx, vy, vz, ax, ay, az, vsq;
};

__device__ __forceinline__ int ent_at(const OrbitDev &o, int64_t t, Ent *e, bool *exact = nullptr) {
  OrbitState s;
  double vsq;
  int rc = orbit_at(o, t, &s, &vsq, exact);
  if (rc != ORB_OK) return rc;
  *e = {s.pos.x, s.pos.y, s.pos.z, s.vel.x, s.vel.y, s.vel.z, s.acc.x, s.acc.y, s.acc.z, vsq};
  return ORB_OK;
}
__device__ __forceinline__ int ent_exact(const OrbitDev &o, int64_t t, Ent *e) {
  OrbitState s;
  double vsq;
  int rc = orbit_exact(o, t, &s, &vsq);
  if (rc != ORB_OK) return rc;
  *e = {s.pos.x, s.pos.y, s.pos.z, s.vel.x, s.vel.y, s.vel.z, s.acc.x, s.acc.y, s.acc.z, vsq};
  return ORB_OK;
}

// One evaluation of the Newton step at a tabulated state (1030-1053).
// Returns 0 = converged (|delta| < tol), 1 = step, 2 = degenerate.
__device__ __forceinline__ int zd_eval(V3 P, const Ent &e, double tol, double *delta) {
  V3 r = {P.x - e.px, P.y - e.py, P.z - e.pz};
  double f = r.x * e.vx + r.y * e.vy + r.z * e.vz;
  double fp = -e.vsq + (r.x * e.ax + r.y * e.ay + r.z * e.az);
  if (fabs(fp) < 1.0) return 2;
  double d = -f / fp;
  *delta = d;
  return fabs(d) < tol ? 0 : 1;
}

// zd_eval on *e, re-evaluated on the reference's state at t (which replaces
// *e; *exact becomes true) when e is approximate and the decision marginal.
__device__ __forceinline__ int zd_step(const OrbitDev &o, V3 P, Ent *e, bool *exact, int64_t t, double tol,
                                       double *delta) {
  int st = zd_eval(P, *e, tol, delta);
  if (!*exact && st != 2 && zd_marginal(*delta, tol) && ent_exact(o, t, e) == ORB_OK) {
    *exact = true;
    st = zd_eval(P, *e, tol, delta);
  }
  return st;
}

struct Slot {  // shared-memory record exchanged with the right-hand neighbour
  int64_t fb;
  int32_t fmask;
  int32_t exact;  // bit k: e[k] is the reference's state
  Ent e[2];
};

#ifndef SD_MAIN_THREADS
#define SD_MAIN_THREADS 256  // 255 pixels + the left neighbour per block
#endif
#ifndef SD_MAIN_MINB
#define SD_MAIN_MINB 2  // blocks per SM the register budget is cut for (128 regs)
#endif
constexpr int MAIN_THREADS = SD_MAIN_THREADS;
constexpr int MAIN_PIX = MAIN_THREADS - 1;  // widest segment: thread 0 is the left halo pixel

// k_main's segment length for a row of `cols` pixels: 255, 127 or 63 pixels
// (one item holds 1, 2 or 4 segments), the one that leaves the fewest
// threads idle; a shorter segment must gain more than 2 % of utilisation
// (each segment spends a thread on its left neighbour).
inline void set_main_segments(TcDev *p) {
  int best = MAIN_PIX;
  double best_u = 0.0;
  for (int seg = MAIN_PIX; seg >= (MAIN_THREADS / 4) - 1; seg = (seg + 1) / 2 - 1) {
    const uint64_t spr = (p->cols + seg - 1) / seg;
    const double u = spr ? (double)p->cols / (double)(spr * (uint64_t)(seg + 1)) : 0.0;
    if (u > best_u + 0.02) best = seg, best_u = u;
  }
  p->seg_px = best;
  p->seg_per_item = MAIN_THREADS / (best + 1);
  p->bpr = (p->cols + best - 1) / best;
}
inline uint64_t main_items(const TcDev &p) {
  return (p.rows * p.bpr + p.seg_per_item - 1) / p.seg_per_item;
}
static_assert(MAIN_THREADS <= 256, "RsEnt::meta holds the k_main thread in 8 bits");

// ── K3: per-pixel solve, candidate outcomes and candidate outputs ───────────
// ── k_heights: the geometry of every pixel ahead of k_main ─────────────────
// Per pixel: the centre height (DEM lookup of 1529-1536), geoid and target
// ECEF (1545-1546), and, where the facet is needed, the four neighbour
// heights and the facet normal and area (1642-1675).  None of it depends on
// the azimuth time, so k_main reads the target (24 B) and k_cand the target
// and facet (56 B) instead of recomputing them.
#ifndef SD_HEIGHTS_MINB
#define SD_HEIGHTS_MINB 4
#endif

// Target and facet of pixel i once its heights are known (ok: the centre
// height hf is finite; fs: the four neighbour heights h are).
__device__ __forceinline__ void heights_store(const TcDev &p, uint64_t i, PixGeo &g, bool ok, float hf, bool fs,
                                              const float h[4]) {
  const uint64_t npx = p.rows * p.cols;
  double *tp = (double *)p.tp;
  if (!ok) {
    tp[i] = NAN;
    if (p.fct) ((double *)p.fct)[3 * npx + i] = NAN;
    return;
  }
  pixel_ecef(p, &g, hf);
  tp[i] = g.P.x;
  tp[npx + i] = g.P.y;
  tp[2 * npx + i] = g.P.z;
  if (p.fct) {
    double *f = (double *)p.fct;
    if (fs) {
      const Facet fc = facet_from(p, g, h);
      f[i] = fc.normal.x;
      f[npx + i] = fc.normal.y;
      f[2 * npx + i] = fc.normal.z;
      f[3 * npx + i] = fc.area;
    } else {
      f[3 * npx + i] = NAN;
    }
  }
}

// Pixel i with the checked lookups (an undecided lookup is redone exactly).
__device__ __noinline__ void heights_exact(const TcDev &p, uint64_t i) {
  const uint64_t r = i / p.cols, c = i % p.cols;
  PixGeo g;
  float hf, h[4];
  const bool ok = pixel_height(p, r, c, &g, &hf);
  const bool fs = ok && p.fct && facet_heights(p, g, h);
  heights_store(p, i, g, ok, hf, fs, h);
}

// The exact lookup behind an undecided one costs a full UTM projection;
// taken inline by ~1 pixel in 200 it stalls the other 31 lanes of the warp
// and the instruction cache.  Such pixels are queued instead and k_heights_fix
// runs them 32 to a warp.
// One k_heights item: SEL_THREADS pixels of job jb from local item li.
// Every thread of the block calls it (the deferral ballot needs all lanes);
// wp's deferral queue is read only when a lane defers.
__device__ __forceinline__ void heights_item(const TcDev &p, int jb, uint64_t li, const TcWork *__restrict__ wp) {
  if (p.rs_cnt && threadIdx.x == 0) p.rs_cnt[li] = 0;  // k_cand's queue of this item
  const uint64_t i = li * SEL_THREADS + threadIdx.x;
  bool defer = false;
  if (i < p.rows * p.cols) {
    const uint64_t r = i / p.cols, c = i % p.cols;
    PixGeo g;
    float hf, h[4];
    const int st = pixel_height_try(p, r, c, &g, &hf);
    const int fs = st > 0 && p.fct ? facet_heights_try(p, g, h) : 0;
    if (st >= 0 && fs >= 0) heights_store(p, i, g, st > 0, hf, fs > 0, h);
    else defer = true;
  }
  // queue the deferred lanes, one atomic per warp
  const unsigned m = __ballot_sync(0xffffffffu, defer);
  if (m) {
    const int lane = threadIdx.x & 31;
    unsigned base = 0;
    if (lane == 0) base = atomicAdd(wp->hq_cnt, (unsigned)__popc(m));
    base = __shfl_sync(0xffffffffu, base, 0);
    if (defer) {
      const unsigned slot = base + __popc(m & ((1u << lane) - 1u));
      if (slot < wp->hq_cap) wp->hq[slot] = ((unsigned long long)jb << 40) | i;
      ((double *)p.tp)[i] = -INFINITY;  // the mark k_heights_fix scans for when the queue overflowed
    }
  }
}

// Persistent form over the work table: the current job's record in shared
// memory (restaged when the block's item stride crosses into the next job).
__global__ void __launch_bounds__(SEL_THREADS, SD_HEIGHTS_MINB) k_heights(const TcWork *__restrict__ wp) {
  __shared__ __align__(16) unsigned char s_job[sizeof(TcDev)];
  const uint64_t *pre = stage_pre(*wp, WK_SEL);
  const int n_jobs = wp->n_jobs;
  const uint64_t total = pre[n_jobs];
  const TcDev &p = *reinterpret_cast<const TcDev *>(s_job);
  int cur = -1;
  for (uint64_t item = blockIdx.x; item < total; item += gridDim.x) {
    const int jb = find_job(pre, n_jobs, item);  // uniform over the block
    if (jb != cur) {
      __syncthreads();  // every thread is done with the previous record
      load_job(s_job, wp->jobs + jb, threadIdx.x, SEL_THREADS);
      __syncthreads();
      cur = jb;
    }
    heights_item(p, jb, item - pre[jb], wp);
  }
}

// Parameter form: one job (work-table index jb), one block per item.  The
// record sits in the kernel's parameter bank, so its fields are instruction
// operands rather than loads into registers.
__global__ void __launch_bounds__(SEL_THREADS, SD_HEIGHTS_MINB) k_heights_param(TcDev p, int jb,
                                                                              const TcWork *__restrict__ wp) {
  heights_item(p, jb, blockIdx.x, wp);
}

// The deferred pixels of k_heights, with the checked lookups: the queue, or
// after an overflow every pixel k_heights marked.
__global__ void __launch_bounds__(128) k_heights_fix(const TcWork *__restrict__ wp) {
  const TcWork w = *wp;
  const unsigned cnt = *w.hq_cnt;
  if (cnt <= w.hq_cap) {
    for (unsigned k = blockIdx.x * blockDim.x + threadIdx.x; k < cnt; k += gridDim.x * blockDim.x) {
      const unsigned long long e = w.hq[k];
      const int jb = (int)(e >> 40);
      const uint64_t i = e & ((1ull << 40) - 1);
      if (jb < w.n_jobs && i < w.jobs[jb].rows * w.jobs[jb].cols) heights_exact(w.jobs[jb], i);
    }
    return;
  }
  const uint64_t *pre = stage_pre(w, WK_SEL);
  const uint64_t total = pre[w.n_jobs] * SEL_THREADS;
  for (uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; k < total; k += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t item = k / SEL_THREADS;
    const int jb = find_job(pre, w.n_jobs, item);
    const TcDev &p = w.jobs[jb];
    const uint64_t i = (item - pre[jb]) * SEL_THREADS + k % SEL_THREADS;
    if (i < p.rows * p.cols && p.tp[i] == -INFINITY) heights_exact(p, i);
  }
}

// ── the orbit around a warp's shared time ────────────────────────────────────
// A warp's 32 pixels converge within ~±5 ms of its shared time uw.  Inside
// one Lagrange window the reference's position and velocity are degree-7
// polynomials in time, so their Taylor expansions about uw reproduce them;
// to third order the remainder is < 1e-14 m and 1e-17 m/s over 20 ms.  The
// expansion starts from the table entry at uw (the reference's own sums) and
// takes its higher derivatives from the window polynomials, so a lane's
// states cost ~30 FMAs from shared memory instead of 80 B orbit-table reads
// at scattered microseconds (the table entries of neighbouring pixels lie
// ~250 us apart).  Times outside uw's window, at a state-vector time (where
// the reference's acceleration drops a term) or more than 20 ms from uw read
// the table.
struct OrbTaylor {
  double p0[3], v0[3], a0[3];  // table state at uw
  double dp[3], p2[3], p3[3];  // position: d/dt, d2/dt2 / 2, d3/dt3 / 6
  double v2[3], v3[3];         // velocity: d2/dt2 / 2, d3/dt3 / 6
  int64_t uw, lo, hi;          // valid for lo < t < hi (uw's window), |t - uw| <= 20 ms
  int ok, pad;
};

// Lanes 0-2 of the warp fill coordinate `lane` of T; lane 0 the bounds.
__device__ __forceinline__ void orb_taylor_build(const OrbitDev &o, int64_t uw, const Ent &ew, bool ew_ok,
                                                 int lane, OrbTaylor *T) {
  if (lane > 2) return;
  bool ok = ew_ok && o.poly && o.n >= 8;
  uint64_t centre = 0;
  if (ok) {
    uint64_t lo = 0, hi = o.n;
    while (lo < hi) {
      const uint64_t mid = (lo + hi) / 2;
      if (o.svs[mid].time_us <= uw) lo = mid + 1; else hi = mid;
    }
    centre = lo - 1;
    ok = centre + 1 < o.n && o.svs[centre].time_us != uw;
  }
  if (lane == 0) {
    T->ok = ok;
    T->uw = uw;
    T->lo = ok ? o.svs[centre].time_us : 0;
    T->hi = ok ? o.svs[centre + 1].time_us : 0;
  }
  if (!ok) return;
  const uint64_t start = centre < 4 ? 0 : (centre + 4 >= o.n ? o.n - 8 : centre - 3);
  const OrbPoly &w = o.poly[start];
  const double x = (double)(uw - w.tc) / 1e6;
  const int d = lane;
  double b[8], v[8];
#pragma unroll
  for (int m = 0; m < 8; ++m) {
    b[m] = w.c[d][m];
    v[m] = w.c[3 + d][m];
  }
  // Taylor shift by repeated synthetic division: after pass k, b[k] = p^(k)(x)/k!
#pragma unroll
  for (int k = 0; k < 4; ++k)
#pragma unroll
    for (int j = 6; j >= k; --j) {
      b[j] = fma(x, b[j + 1], b[j]);
      v[j] = fma(x, v[j + 1], v[j]);
    }
  const double pe[3] = {ew.px, ew.py, ew.pz}, ve[3] = {ew.vx, ew.vy, ew.vz}, ae[3] = {ew.ax, ew.ay, ew.az};
  T->p0[d] = pe[d];
  T->v0[d] = ve[d];
  T->a0[d] = ae[d];
  T->dp[d] = b[1];
  T->p2[d] = b[2];
  T->p3[d] = b[3];
  T->v2[d] = v[2];
  T->v3[d] = v[3];
}

// Expansions about every TAY_STEP-th microsecond of the orbit table's span,
// built once per table: a warp copies the one nearest its shared time
// (|uw - centre| <= 2 ms, so its lanes' times stay well inside the 20 ms
// bound) instead of searching the state vectors and shifting the window
// polynomial on the way to its first Newton step.
constexpr int64_t TAY_STEP = 4000;
constexpr int TAY_WORDS = (int)(sizeof(OrbTaylor) / 8);
static_assert(sizeof(OrbTaylor) % 8 == 0 && TAY_WORDS <= 32, "one 8-byte word of OrbTaylor per lane");

inline int64_t tay_count(int64_t tab_n) { return tab_n > 0 ? (tab_n - 1) / TAY_STEP + 1 : 0; }

// Thread 3k + d fills coordinate d of expansion k (o.tab must be built).
__global__ void k_orbit_taylor(OrbitDev o, int64_t n, OrbTaylor *out) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= 3 * n) return;
  const int64_t k = i / 3;
  const int64_t u = o.tab_t0 + k * TAY_STEP;
  Ent e;
  const bool ok = ent_at(o, u, &e) == ORB_OK;
  orb_taylor_build(o, u, e, ok, (int)(i % 3), out + k);
}

// Every lane of the warp calls it with the warp's shared time uw.
__device__ __forceinline__ void orb_taylor_fetch(const OrbitDev &o, int64_t uw, const Ent &ew, bool ew_ok,
                                                 int lane, OrbTaylor *T) {
  const int64_t q = uw - o.tab_t0 + TAY_STEP / 2;
  if (o.tay && q >= 0 && q / TAY_STEP < o.tay_n) {
    if (lane < TAY_WORDS)
      reinterpret_cast<uint64_t *>(T)[lane] = __ldg(reinterpret_cast<const uint64_t *>(o.tay + q / TAY_STEP) + lane);
  } else {
    orb_taylor_build(o, uw, ew, ew_ok, lane, T);
  }
}

// Expansions over orb's table into d_out (tay_count(orb->tab_n) entries);
// sets orb->tay.
inline int launch_orbit_taylor(sd_ctx *ctx, OrbitDev *orb, OrbTaylor *d_out) {
  const int64_t n = tay_count(orb->tab_n);
  orb->tay = nullptr;
  orb->tay_n = 0;
  if (n == 0) return SD_OK;
  OrbitDev o = *orb;
  SD_TIMED_BEGIN(ctx, "k_orbit_taylor");
  k_orbit_taylor<<<grid_for((size_t)(3 * n), 128), 128, 0, ctx->stream>>>(o, n, d_out);
  SD_LAUNCHED(ctx);
  orb->tay = d_out;
  orb->tay_n = n;
  return SD_OK;
}

// State at t from the warp's expansion (*exact = false), or from the table.
__device__ __forceinline__ int ent_lane(const OrbitDev &o, const OrbTaylor &T, int64_t t, Ent *e, bool *exact) {
  const int64_t dt = t - T.uw;
  if (T.ok && t > T.lo && t < T.hi && dt <= 20000 && dt >= -20000) {
    const double h = (double)dt * 1e-6;
    double P[3], V[3], A[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      P[d] = fma(h, fma(h, fma(h, T.p3[d], T.p2[d]), T.dp[d]), T.p0[d]);
      V[d] = fma(h, fma(h, fma(h, T.v3[d], T.v2[d]), T.a0[d]), T.v0[d]);
      A[d] = fma(h, fma(h, 3.0 * T.v3[d], 2.0 * T.v2[d]), T.a0[d]);
    }
    *e = {P[0], P[1], P[2], V[0], V[1], V[2], A[0], A[1], A[2], V[0] * V[0] + V[1] * V[1] + V[2] * V[2]};
    *exact = false;
    return ORB_OK;
  }
  return ent_at(o, t, e, exact);
}

// One k_main work item: seg_per_item consecutive row segments of seg_px
// pixels (the first thread of each segment holds the segment's left
// neighbour).  Narrow rows use shorter segments, so a 256-pixel row is not
// one full item and one nearly empty one.  Every thread of the block calls
// it.  It records F and the codes only: the outputs of the one member the
// row walk selects are computed after the walk (k_cand), so this kernel
// holds no resampling or facet state.
__device__ __forceinline__ void main_item(const TcDev &p, uint64_t item, Slot *slot, OrbTaylor *tw) {
  const int tid = threadIdx.x;
  const int fast = p.fast;
  const int segw = p.seg_px + 1, pos = tid % segw;
  const uint64_t sg = item * (uint64_t)p.seg_per_item + (uint64_t)(tid / segw);  // the thread's segment
  const bool seg_ok = sg < p.rows * p.bpr;
  const uint64_t r = seg_ok ? sg / p.bpr : p.rows;  // r == rows: no pixel
  const int64_t c = (int64_t)(seg_ok ? sg % p.bpr : 0) * p.seg_px + pos - 1;
  const bool in_row = seg_ok && c >= 0 && c < (int64_t)p.cols;
  const uint64_t i = r * p.cols + (uint64_t)(c < 0 ? 0 : c);
  PixGeo g;
  bool geo_ok = false;
  int fmask = 0;
  int64_t fb = 0;
  // The pair's orbit states go to this thread's slot as soon as they are
  // known, so they do not stay live in registers across the block barrier.
  Slot &my = slot[tid];
  int exm = 0;  // bit k: my.e[k] is the reference's state
  // The warp's 32 pixels lie within ~10 ms of azimuth time: all lanes take
  // their first Newton step from one shared state (one broadcast read), the
  // landing point is within a few ns of each lane's own root.
  const uint64_t rr = r < p.rows ? r : p.rows - 1;
  const uint64_t cq = c < 0 ? 0 : ((uint64_t)c < p.cols ? (uint64_t)c : p.cols - 1);
  // the target from k_heights (every job has it), loaded ahead of the warp's
  // orbit expansion, which does not depend on it
  const bool px_in = in_row && r < p.rows;
  if (px_in) {
    const uint64_t npx = p.rows * p.cols;
    g.P.x = __ldg(p.tp + i);
    g.P.y = __ldg(p.tp + npx + i);
    g.P.z = __ldg(p.tp + 2 * npx + i);
  }
  const int64_t uw = __shfl_sync(0xffffffffu, predicted_time(p, rr, cq), 16);
  Ent ew;
  bool ew_exact = false;
  const bool ew_ok = fast && ent_at(p.orb, uw, &ew, &ew_exact) == ORB_OK;
  OrbTaylor &T = tw[tid >> 5];
  orb_taylor_fetch(p.orb, uw, ew, ew_ok, tid & 31, &T);
  __syncwarp();
  if (px_in) {
    geo_ok = isfinite(g.P.x);
    if (geo_ok && fast) {
      // reference iteration from the shared state: one converged t*
      int64_t t = ew_ok ? uw : predicted_time(p, r, (uint64_t)c);
      Ent e;
      bool ex = false;
      double d = 0.0;
      int st = 1;
      for (int it = 0; it < 40 && st == 1; ++it) {
        if (it == 0 && ew_ok) {
          e = ew;
          ex = ew_exact;
        } else if (ent_lane(p.orb, T, t, &e, &ex) != ORB_OK) {
          st = 3;
          break;
        }
        st = zd_step(p.orb, g.P, &e, &ex, t, p.tol, &d);
        if (st == 1) t = t + f2i64(d * 1e6);
      }
      if (st == 0) {
        // F = {t : |delta(t)| < tol} lies in {t*-1, t*, t*+1}.  The root sits
        // at t* + d; delta carries ~1e-13 s of rounding noise (the dot
        // product cancels terms of ~6e9) and the states' approximation up to
        // ~3e-12 s, so for |d| >= 1e-11 s only t* + sign(d) can join t*,
        // while for smaller |d| both neighbours are evaluated.  A
        // three-member F is left to the exact path.
        const int64_t ta = d > 0.0 ? t + 1 : t - 1;  // the likely member
        const int kt = ta > t ? 0 : 1;                // position of t* in the pair {ta, t*}
        my.e[kt] = e;
        int ex_t = ex ? 1 : 0;
        bool ma;
        {
          Ent ea;
          bool exa = false;
          double da = 0.0;
          ma = ent_lane(p.orb, T, ta, &ea, &exa) == ORB_OK && zd_step(p.orb, g.P, &ea, &exa, ta, p.tol, &da) == 0;
          my.e[1 - kt] = ea;
          exm = (ex_t << kt) | ((exa ? 1 : 0) << (1 - kt));
        }
        bool mb = false;
        if (fabs(d) < 1e-11) {
          const int64_t tb = d > 0.0 ? t - 1 : t + 1;
          Ent eb;
          bool exb = false;
          double db = 0.0;
          mb = ent_lane(p.orb, T, tb, &eb, &exb) == ORB_OK && zd_step(p.orb, g.P, &eb, &exb, tb, p.tol, &db) == 0;
          if (mb && !ma) {  // the pair {t*, tb}: t* moves to the other position
            my.e[1 - kt] = my.e[kt];
            my.e[kt] = eb;
            exm = (ex_t << (1 - kt)) | ((exb ? 1 : 0) << kt);
          }
        }
        if (!(ma && mb)) {
          if (mb) {  // {t*, tb}, tb on the other side of t* than ta
            fb = kt == 0 ? t - 1 : t;
            fmask = 3;
          } else {   // {t*, ta}
            fb = kt == 0 ? t : ta;
            fmask = (1 << kt) | (ma ? 1 << (1 - kt) : 0);
          }
        }
      }
    }
  }
  my.fb = fb;
  my.fmask = fmask;
  my.exact = exm;
  __syncthreads();
  if (pos == 0 || !in_row || r >= p.rows) return;

  uint32_t cc = 0xFFFFu;
  if (!geo_ok) {
    cc |= CF_DEMMISS;
  } else if (fmask) {
    cc |= CF_HASF | CF_CODES | ((uint32_t)fmask << 16);
    // outcome of the reference iteration seeded at each member of the left
    // neighbour's F (the only seeds the row walk can hand this pixel)
    const Slot &L = slot[tid - 1];
    if (c > 0 && L.fmask) {
      for (int k = 0; k < 2; ++k) {
        if (!((L.fmask >> k) & 1)) continue;
        int64_t t = L.fb + k;
        uint32_t code = 0xFF;
        for (int it = 0; it < p.max_iter; ++it) {
          // a member of this pixel's F converges by definition (|delta| < tol
          // was evaluated there with the same state and arithmetic)
          const int64_t mf = t - fb;
          if ((mf == 0 || mf == 1) && ((fmask >> mf) & 1)) {
            code = (uint32_t)mf | ((uint32_t)min(it + 1, 15) << 4);
            break;
          }
          Ent e;
          bool exact = false;
          bool have = true;
          if (t == L.fb + k) {
            e = L.e[k];
            exact = (L.exact >> k) & 1;
          } else {
            have = ent_lane(p.orb, T, t, &e, &exact) == ORB_OK;
          }
          if (!have) break;  // orbit error: the walk redoes it
          double d;
          int st = zd_step(p.orb, g.P, &e, &exact, t, p.tol, &d);
          if (st == 0) {
            int64_t m = t - fb;
            if ((m == 0 || m == 1) && ((fmask >> m) & 1)) code = (uint32_t)m | ((uint32_t)min(it + 1, 15) << 4);
            break;
          }
          if (st == 2) {
            code = 3u | (2u << 2) | ((uint32_t)min(it, 15) << 4);
            break;
          }
          t = t + f2i64(d * 1e6);
          if (it + 1 == p.max_iter) code = 3u | (1u << 2) | ((uint32_t)min(p.max_iter, 15) << 4);
        }
        cc = (cc & ~(0xFFu << (8 * k))) | (code << (8 * k));
      }
    }
  }
  p.fb[i] = fb;
  p.cc[i] = cc;
}

// Single job: the job record is a kernel parameter (constant-bank operands)
// and the grid covers its rows x bpr items.
__global__ void __launch_bounds__(MAIN_THREADS, SD_MAIN_MINB) k_main(TcDev p) {
  __shared__ Slot slot[MAIN_THREADS];
  __shared__ OrbTaylor tw[MAIN_THREADS / 32];
  main_item(p, blockIdx.x, slot, tw);
}

// Tile batches: persistent CTAs over the work table; the current job's
// record is staged in shared memory.
__global__ void __launch_bounds__(MAIN_THREADS, SD_MAIN_MINB) k_main_batch(const TcWork *__restrict__ wp) {
  __shared__ Slot slot[MAIN_THREADS];
  __shared__ __align__(16) unsigned char s_job[sizeof(TcDev)];
  __shared__ OrbTaylor tw[MAIN_THREADS / 32];
  __shared__ int s_j;
  const TcWork w = *wp;
  const uint64_t *pre = stage_pre(w, WK_MAIN);
  const uint64_t total = pre[w.n_jobs];
  const TcDev &p = *reinterpret_cast<const TcDev *>(s_job);
  const int tid = threadIdx.x;
  int cur = -1;
  for (uint64_t item = blockIdx.x; item < total; item += gridDim.x) {
    __syncthreads();  // the previous item is done with slot[] and the job record
    if (tid == 0) s_j = find_job(pre, w.n_jobs, item);
    __syncthreads();
    const int jb = s_j;
    if (jb != cur) {
      load_job(s_job, w.jobs + jb, tid, MAIN_THREADS);
      __syncthreads();
      cur = jb;
    }
    const uint64_t li = item - pre[jb];
    main_item(p, li, slot, tw);
  }
}

// ── K4: the row walk ──────────────────────────────────────────────────────
// The walk's state between two pixels is either an index into the recorded
// F of the previous pixel (kind 0) or an explicit seed time (kind 1, after a
// DEM void, a non-converged solve or an exact-path pixel); kind 2 marks an
// entry that cannot occur.
struct WState {
  int kind;
  int64_t v;
};

// The reference solve of pixel (r, c) from seed s, for pixels the
// precomputed records do not cover.  A converged time that is not a member
// of the pixel's F is selected as SEL_DONE and, with `write`, stored in fb
// (nothing reads that pixel's F afterwards: the walk leaves it with an
// explicit seed).
__device__ WState exact_pixel(const TcDev &p, uint64_t r, uint64_t c, int64_t s, uint32_t cc, int64_t fb,
                              bool write, uint8_t *sel) {
  const uint64_t i = r * p.cols + c;
  PixGeo g;
  if (!pixel_geo(p, r, c, &g)) {
    *sel = SEL_DEMMISS;
    return {1, s};
  }
  ZdRes z = newton(p.orb, g.P, s, p.max_iter, p.tol);
  if (z.st == ST_ORBIT) {
    if (write) atomicOr(&p.flags[0], 1);
    *sel = SEL_ORBIT;
    return {1, s};
  }
  if (z.st == ST_NONCONV || z.st == ST_DEGEN) {
    *sel = z.st == ST_NONCONV ? SEL_NONCONV : SEL_DEGEN;
    return {1, s};
  }
  const int it = z.it > 15 ? 15 : z.it;
  if (cc & CF_CODES) {
    const uint32_t fm = (cc >> 16) & 3u;
    const int64_t m = z.t - fb;
    if ((m == 0 || m == 1) && ((fm >> m) & 1)) {
      *sel = (uint8_t)(m | (it << 4));
      return {0, m};
    }
  }
  *sel = (uint8_t)(SEL_DONE | (it << 4));
  if (write) {
    atomicAdd(&p.flags[1], 1);
    p.fb[i] = z.t;
  }
  return {1, z.t};
}

// Walk columns [b, e) of row r from state st (terrain_correction.rs:
// 1443-1580), any pixel kind.  fb is read only where a seed value is needed.
__device__ WState walk_seg(const TcDev &p, uint64_t r, uint64_t b, uint64_t e, WState st, bool write) {
  const uint64_t base = r * p.cols;
  uint32_t prev_cc = b > 0 ? p.cc[base + b - 1] : CF_DEMMISS;
  if (st.kind == 0 && !((prev_cc & CF_HASF) && ((prev_cc >> (16 + st.v)) & 1u))) return {2, 0};
  for (uint64_t c = b; c < e; ++c) {
    const uint32_t cc = p.cc[base + c];
    uint8_t sel;
    if (cc & CF_DEMMISS) {
      if (st.kind == 0) st = {1, p.fb[base + c - 1] + st.v};  // the seed passes through the void
      sel = SEL_DEMMISS;
    } else {
      uint32_t code = 0xFF;
      if (st.kind == 0 && (prev_cc & CF_HASF) && (cc & CF_CODES)) code = (cc >> (8 * st.v)) & 0xFFu;
      if (code != 0xFF && (code & 3u) != 3u) {
        st = {0, (int64_t)(code & 3u)};
        sel = (uint8_t)((code & 3u) | (code & 0xF0u));
      } else if (code != 0xFF) {
        st = {1, p.fb[base + c - 1] + st.v};  // not converged: seed unchanged
        sel = (uint8_t)((((code >> 2) & 3u) == 1u ? SEL_NONCONV : SEL_DEGEN) | (code & 0xF0u));
      } else {
        const int64_t s = st.kind == 0 ? p.fb[base + c - 1] + st.v : st.v;
        st = exact_pixel(p, r, c, s, cc, p.fb[base + c], write, &sel);
      }
    }
    if (write) p.sel[base + c] = sel;
    prev_cc = cc;
  }
  return st;
}

// One warp per row.  Lane 0 resolves the row's first valid pixel from the
// LUT guess; the remaining columns are cut into 32 segments, each lane maps
// the two possible entry states (which member of the left F the seed is)
// through its segment, the maps are composed in lane order (a lane whose
// entry is an explicit seed walks its segment at that point), and each lane
// writes its segment from its actual entry.  In the regular case the
// segments are streamed 32 columns at a time through shared memory with
// coalesced transposed loads and stores; a segment with any other pixel
// kind is (re)done by walk_seg.
constexpr int SCAN_WARPS = 4;

__global__ void __launch_bounds__(SCAN_WARPS * 32) k_scan(const TcWork *__restrict__ wp) {
  __shared__ uint32_t sbuf[SCAN_WARPS][32][33];
  __shared__ __align__(16) unsigned char s_job[SCAN_WARPS][sizeof(TcDev)];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  uint32_t(*buf)[33] = sbuf[wid];
  const TcWork w = *wp;
  const uint64_t *pre = stage_pre(w, WK_SCAN);
  const uint64_t total = pre[w.n_jobs];
  const TcDev &p = *reinterpret_cast<const TcDev *>(s_job[wid]);
  const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  int cur = -1;
  for (uint64_t item = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; item < total;
       item += nwarps) {  // one output row per warp and item
  const int jb = find_job(pre, w.n_jobs, item);
  __syncwarp();
  if (jb != cur) {
    load_job(s_job[wid], w.jobs + jb, lane, 32);
    __syncwarp();
    cur = jb;
  }
  const uint64_t r = item - pre[jb];
  const uint64_t n = p.cols, base = r * n;
  const uint32_t *ccr = p.cc + base;
  uint64_t c0 = n;
  WState st0{1, 0};
  if (lane == 0) {
    uint64_t c = 0;
    while (c < n && (ccr[c] & CF_DEMMISS)) {
      p.sel[base + c] = SEL_DEMMISS;
      ++c;
    }
    if (c < n) {
      st0 = walk_seg(p, r, c, c + 1, WState{1, p.row_guess[r]}, true);
      c0 = c + 1;
    }
  }
  c0 = __shfl_sync(0xffffffffu, c0, 0);
  st0.kind = __shfl_sync(0xffffffffu, st0.kind, 0);
  st0.v = __shfl_sync(0xffffffffu, st0.v, 0);
  if (c0 >= n) continue;
  const uint64_t seg = (n - c0 + 31) / 32;
  const uint64_t b = c0 + (uint64_t)lane * seg;
  const uint64_t e = min(n, b + seg);
  const int nchunks = (int)((seg + 31) / 32);

  // phase 1: both entry states through the segment (regular pixels only)
  int s0 = 0, s1 = 1, bad = 0;
  if (b < e) {
    const uint32_t prev = ccr[b - 1];
    if (!((prev & CF_HASF) && ((prev >> 16) & 1u))) bad |= 1;
    if (!((prev & CF_HASF) && ((prev >> 17) & 1u))) bad |= 2;
  }
  for (int k = 0; k < nchunks; ++k) {
    for (int j = 0; j < 32; ++j) {
      const uint64_t bj = c0 + (uint64_t)j * seg, ej = min(n, bj + seg);
      const uint64_t idx = bj + 32 * (uint64_t)k + lane;
      buf[j][lane] = idx < ej ? __ldg(ccr + idx) : 0u;
    }
    __syncwarp();
    const int cnt = b + 32 * (uint64_t)k < e ? (int)min((uint64_t)32, e - b - 32 * (uint64_t)k) : 0;
    for (int t = 0; t < cnt; ++t) {
      const uint32_t w = buf[lane][t];
      if ((w & (CF_DEMMISS | CF_CODES)) != CF_CODES) bad = 3;
      const uint32_t x0 = (w >> (8 * s0)) & 0xFFu, x1 = (w >> (8 * s1)) & 0xFFu;
      if (x0 == 0xFFu || (x0 & 3u) == 3u) bad |= 1;
      if (x1 == 0xFFu || (x1 & 3u) == 3u) bad |= 2;
      s0 = (int)(x0 & 1u);
      s1 = (int)(x1 & 1u);
    }
    __syncwarp();
  }
  WState ex0 = {0, 0}, ex1 = {0, 1};
  if (b < e) {
    ex0 = (bad & 1) ? walk_seg(p, r, b, e, WState{0, 0}, false) : WState{0, s0};
    ex1 = (bad & 2) ? walk_seg(p, r, b, e, WState{0, 1}, false) : WState{0, s1};
  }
  // phase 2: compose the lanes' maps in order
  WState st = st0, entry{2, 0};
  for (int j = 0; j < 32; ++j) {
    WState nx = st;
    if (lane == j) {
      entry = st;
      if (b < e) {
        if (st.kind == 0) nx = st.v == 0 ? ex0 : ex1;
        else nx = walk_seg(p, r, b, e, st, false);
      }
    }
    st.kind = __shfl_sync(0xffffffffu, nx.kind, j);
    st.v = __shfl_sync(0xffffffffu, nx.v, j);
  }
  // phase 3: write the segments
  const bool regular = b < e && entry.kind == 0 && !((bad >> entry.v) & 1);
  int s = regular ? (int)entry.v : 0;
  uint8_t *selr = p.sel + base;
  for (int k = 0; k < nchunks; ++k) {
    for (int j = 0; j < 32; ++j) {
      const uint64_t bj = c0 + (uint64_t)j * seg, ej = min(n, bj + seg);
      const uint64_t idx = bj + 32 * (uint64_t)k + lane;
      buf[j][lane] = idx < ej ? __ldg(ccr + idx) : 0u;
    }
    __syncwarp();
    if (regular) {
      const int cnt = b + 32 * (uint64_t)k < e ? (int)min((uint64_t)32, e - b - 32 * (uint64_t)k) : 0;
      for (int t = 0; t < cnt; ++t) {
        const uint32_t code = (buf[lane][t] >> (8 * s)) & 0xFFu;
        s = (int)(code & 3u);
        buf[lane][t] = (uint32_t)(s | (code & 0xF0u));
      }
    }
    __syncwarp();
    for (int j = 0; j < 32; ++j) {
      const uint64_t bj = c0 + (uint64_t)j * seg, ej = min(n, bj + seg);
      const uint64_t idx = bj + 32 * (uint64_t)k + lane;
      const bool reg_j = __shfl_sync(0xffffffffu, regular, j);
      if (reg_j && idx < ej) selr[idx] = (uint8_t)buf[j][lane];
    }
    __syncwarp();
  }
  if (b < e && !regular) walk_seg(p, r, b, e, entry, true);
  }
}

// ── K5: outputs of the selected member, rasters, counters, histogram ───────
// After the walk every pixel with a converged time has exactly one: fb +
// member (SEL_M0/SEL_M1) or fb itself (an exact-path pixel).  One thread per
// pixel recomputes the pixel's geometry (lon/lat, the DEM heights k_heights
// left, geoid, target ECEF), reads the satellite position at that time from
// the orbit table (the reference's own sums, so the slant range and image
// coordinates are the reference's) and forms the reference's outputs (1585-1739:
// resampling, facet, flattening, masks, NESZ).  Split precision: a candidate
// FP32 cannot settle is queued for an FP64 re-sample (RD_SAMPLE, k_resample)
// or flagged for the FP64 candidate (RD_FULL, k_redo), which write and count
// it instead.
#ifndef SD_CAND_MINB
#define SD_CAND_MINB 4  // blocks of 256 per SM the register budget is cut for (latency-bound: warps over spills)
#endif

// The pixel's target and facet as k_heights left them (every job has them).
// A pixel's k_heights planes, loaded together (one memory round trip: no
// load waits on another's value).
struct PixPlanes {
  double t[3], f[4];
};
__device__ __forceinline__ PixPlanes load_planes(const TcDev &p, uint64_t i) {
  const uint64_t npx = p.rows * p.cols;
  PixPlanes q;
#pragma unroll
  for (int k = 0; k < 3; ++k) q.t[k] = __ldg(p.tp + k * npx + i);
#pragma unroll
  for (int k = 0; k < 4; ++k) q.f[k] = p.fct ? __ldg(p.fct + k * npx + i) : NAN;
  return q;
}
// target_facet from preloaded planes
__device__ __forceinline__ bool target_facet_of(const TcDev &p, const PixPlanes &q, V3 *P, Facet *f) {
  P->x = q.t[0];
  if (!isfinite(P->x)) return false;
  P->y = q.t[1];
  P->z = q.t[2];
  f->ok = false;
  if (p.fct && isfinite(q.f[3])) {
    f->ok = true;
    f->normal = {q.f[0], q.f[1], q.f[2]};
    f->area = q.f[3];
  }
  return true;
}

__device__ __forceinline__ bool target_facet(const TcDev &p, uint64_t i, V3 *P, Facet *f) {
  const uint64_t npx = p.rows * p.cols;
  P->x = __ldg(p.tp + i);
  if (!isfinite(P->x)) return false;
  P->y = __ldg(p.tp + npx + i);
  P->z = __ldg(p.tp + 2 * npx + i);
  f->ok = false;
  if (p.fct) {
    const double area = __ldg(p.fct + 3 * npx + i);
    if (isfinite(area)) {
      f->ok = true;
      f->normal = {__ldg(p.fct + i), __ldg(p.fct + npx + i), __ldg(p.fct + 2 * npx + i)};
      f->area = area;
    }
  }
  return true;
}

// One k_cand item: the outputs of SEL_THREADS pixels of job p from local
// item li; counts go to the block's s_cnt.
template <int KERNEL, bool SPLIT>
__device__ __forceinline__ void cand_item(const TcDev &p, uint64_t li, unsigned int *s_cnt) {
  const int tid = threadIdx.x;
  const uint64_t npx = p.rows * p.cols;
  const uint64_t i = li * SEL_THREADS + tid;
  // the pixel's walk outcome, base time and geometry in one round trip
  uint8_t sel = (uint8_t)SEL_ORBIT;
  int64_t fbv = 0;
  PixPlanes pl;
  if (i < npx) {
    sel = p.sel[i];
    fbv = p.fb[i];
    pl = load_planes(p, i);
  }
  const int code = sel & 7, it = sel >> 4;
  const bool has_t = code == SEL_M0 || code == SEL_M1 || code == SEL_DONE;
  const int64_t t = has_t ? fbv + (code == SEL_M1 ? 1 : 0) : 0;
  int counter = -1;
  if (has_t) {
    atomicAdd(&s_cnt[kCounters + it], 1u);
    const uint64_t r = i / p.cols;
    V3 P;
    Facet fc;
    const bool ok = target_facet_of(p, pl, &P, &fc);
    V3 S;
    const bool orb_ok = ok && orbit_pos_exact(p.orb, t, &S);
    if (!orb_ok) atomicOr(&p.flags[ok ? 0 : 5], 1);  // cannot happen for a converged time
    CandOut o{NAN, NAN, SD_MASK_OUTSIDE_FOOTPRINT, 2};
    bool deferred = false;
    if (orb_ok) {
      const double flat_area = p.need_geom ? p.row_flat[r] : 0.0;
      if constexpr (SPLIT) {
        const CandPre cp = cand_pre<KERNEL, true>(p, P, S, t);
        // the FP64 facet rounded to FP32: within 2^-24 |n| per component,
        // inside the bound cand_post_f allows (kLpErr en, en = area)
        FacetF f{};
        if (fc.ok) {
          f.ok = true;
          f.nx = (float)fc.normal.x, f.ny = (float)fc.normal.y, f.nz = (float)fc.normal.z;
          f.area = (float)fc.area;
          f.en = f.area;
        }
        int redo;
        float wd = 1.f;
        o = cand_post_f(p, cp, P, S, f, (float)flat_area, &redo, &wd);
        if (redo == RD_SAMPLE) {  // queue the FP64 re-sample in this item's slots
          const uint32_t q = atomicAdd(p.rs_cnt + li, 1u);
          if (q < (uint32_t)RS_CAP) {
            p.rs_ent[li * RS_CAP + q] = RsEnt{cp.line, cp.sample, wd, (uint32_t)tid};
            if (p.compute_lia) p.cos_lia[i] = o.cos;
            deferred = true;
          } else {
            redo = RD_FULL;
          }
        }
        if (redo == RD_FULL) {
          p.cc[i] |= CF_REDO;
          atomicAdd(&p.flags[3], 1);
          deferred = true;
        }
      } else {
        const CandPre cp = cand_pre<KERNEL, false>(p, P, S, t);
        o = cand_post(p, cp, P, S, fc, flat_area);
      }
    }
    if (!deferred) {
      float v = o.data;
      if (p.db) {
        int dc;
        v = db_value(v, p.db_floor, &dc);
        if (dc >= 0) atomicAdd(&s_cnt[kCntDb + dc], 1u);
      }
      p.out[i] = v;
      if (p.compute_lia) {
        p.cos_lia[i] = o.cos;
        p.mask[i] = o.mask;
      }
      counter = o.cls;
    }
    if (p.az_time) p.az_time[i] = t;
  } else if (i < npx && code != SEL_ORBIT) {
    const uint8_t m = code == SEL_NONCONV ? SD_MASK_NON_CONVERGED
                      : code == SEL_DEGEN ? SD_MASK_DEGENERATE_GEOMETRY
                                          : SD_MASK_DEM_MISSING;
    counter = code == SEL_NONCONV ? 3 : (code == SEL_DEGEN ? 4 : 1);
    if (p.az_time) p.az_time[i] = INT64_MIN;
    p.out[i] = NAN;
    if (p.compute_lia) {
      p.cos_lia[i] = NAN;
      p.mask[i] = m;
    }
  }
  if (counter >= 0) atomicAdd(&s_cnt[counter], 1u);
}

template <int KERNEL, bool SPLIT>
__global__ void __launch_bounds__(SEL_THREADS, SD_CAND_MINB) k_cand(const TcWork *__restrict__ wp) {
  __shared__ unsigned int s_cnt[kCounters + SD_NEWTON_ITER_HIST_SIZE];
  __shared__ __align__(16) unsigned char s_job[sizeof(TcDev)];
  const TcWork w = *wp;
  const uint64_t *pre = stage_pre(w, WK_SEL);
  const uint64_t total = pre[w.n_jobs];
  const int tid = threadIdx.x;
  // counters accumulate in shared memory over the block's items of one job
  // and go to the job's counters when the job changes or the block ends;
  // the job's record is staged in shared memory at the same change
  for (int k = tid; k < kCounters + SD_NEWTON_ITER_HIST_SIZE; k += blockDim.x) s_cnt[k] = 0;
  const TcDev &p = *reinterpret_cast<const TcDev *>(s_job);
  int cur = -1;
  for (uint64_t item = blockIdx.x; item < total; item += gridDim.x) {
    const int jb = find_job(pre, w.n_jobs, item);
    if (jb != cur) {  // block-uniform
      __syncthreads();
      if (cur >= 0)
        for (int k = tid; k < kCounters + SD_NEWTON_ITER_HIST_SIZE; k += blockDim.x)
          if (s_cnt[k]) {
            atomicAdd(&w.jobs[cur].counters[k], (unsigned long long)s_cnt[k]);
            s_cnt[k] = 0;
          }
      load_job(s_job, w.jobs + jb, tid, blockDim.x);
      __syncthreads();
      cur = jb;
    }
    cand_item<KERNEL, SPLIT>(p, item - pre[jb], s_cnt);
  }
  __syncthreads();
  if (cur >= 0)
    for (int k = tid; k < kCounters + SD_NEWTON_ITER_HIST_SIZE; k += blockDim.x)
      if (s_cnt[k]) atomicAdd(&w.jobs[cur].counters[k], (unsigned long long)s_cnt[k]);
}

// Parameter form for one job (the record in the parameter bank), persistent
// over the job's items.
template <int KERNEL, bool SPLIT>
__global__ void __launch_bounds__(SEL_THREADS, SD_CAND_MINB) k_cand_param(TcDev p) {
  __shared__ unsigned int s_cnt[kCounters + SD_NEWTON_ITER_HIST_SIZE];
  const int tid = threadIdx.x;
  for (int k = tid; k < kCounters + SD_NEWTON_ITER_HIST_SIZE; k += blockDim.x) s_cnt[k] = 0;
  __syncthreads();
  const uint64_t items = (p.rows * p.cols + SEL_THREADS - 1) / SEL_THREADS;
  for (uint64_t li = blockIdx.x; li < items; li += gridDim.x) cand_item<KERNEL, SPLIT>(p, li, s_cnt);
  __syncthreads();
  for (int k = tid; k < kCounters + SD_NEWTON_ITER_HIST_SIZE; k += blockDim.x)
    if (s_cnt[k]) atomicAdd(&p.counters[k], (unsigned long long)s_cnt[k]);
}

// ── k_resample (split precision): FP64 values of the queued candidates ────────
// k_cand queues a candidate (RD_SAMPLE) whose geometry, masks and flattening
// weight FP32 settled but whose resampling sum cancelled past its error
// bound.  One warp per k_cand item, one lane per queued candidate: the FP64
// sampler, the flattening division and the NESZ test of cand_post; a NESZ
// test within its margin sends the pixel to k_redo instead.  Counters are
// added per warp.
template <int KERNEL>
__global__ void __launch_bounds__(SEL_THREADS) k_resample(const TcWork *__restrict__ wp) {
  const TcWork w = *wp;
  const uint64_t *pre = stage_pre(w, WK_SEL);
  const uint64_t total = pre[w.n_jobs];
  const int lane = threadIdx.x & 31;
  const uint64_t nwarps = (uint64_t)gridDim.x * (SEL_THREADS / 32);
  for (uint64_t item = (uint64_t)blockIdx.x * (SEL_THREADS / 32) + (threadIdx.x >> 5); item < total;
       item += nwarps) {
    const int jb = find_job(pre, w.n_jobs, item);
    const TcDev &p = w.jobs[jb];
    if (!p.rs_cnt) continue;
    const uint64_t li = item - pre[jb];
    const uint32_t n = min(p.rs_cnt[li], (uint32_t)RS_CAP);
    if (n == 0) continue;
    for (uint32_t q0 = 0; q0 < n; q0 += 32) {  // warp-uniform: the ballots below
      const uint32_t q = q0 + lane;
      int cls = -1, dbc = -1;
      if (q < n) {
        const RsEnt e = p.rs_ent[li * RS_CAP + q];
        const uint64_t i = li * SEL_THREADS + e.thread;
        float sigma0 = resample<KERNEL>(p, e.line, e.sample);
        uint8_t m = SD_MASK_VALID;
        cls = 0;
        if (sigma0 != sigma0) {
          m = SD_MASK_OUTSIDE_FOOTPRINT;
          cls = 2;
          if (p.compute_lia) p.cos_lia[i] = NAN;
        } else {
          sigma0 /= e.wdiv;
          if (p.nesz_mask) {
            const float nz = sample_bilinear(p.nesz, p.lines, p.samples, e.line, e.sample);
            if (nz == nz) {
              const float thr = nz * p.nesz_factor;
              if (fabsf(sigma0 - thr) <= 1e-5f * fabsf(thr)) {
                atomicOr(p.cc + i, (uint32_t)CF_REDO);
                atomicAdd(&p.flags[3], 1);
                cls = -1;
              } else if (sigma0 <= thr) {
                sigma0 = NAN;
                m = SD_MASK_NOISE_MASKED;
                cls = 6;
              }
            }
          }
        }
        if (cls >= 0) {
          if (p.db) sigma0 = db_value(sigma0, p.db_floor, &dbc);
          p.out[i] = sigma0;
          if (p.compute_lia) p.mask[i] = m;
        }
      }
      const int n0 = __popc(__ballot_sync(0xffffffffu, cls == 0));
      const int n2 = __popc(__ballot_sync(0xffffffffu, cls == 2));
      const int n6 = __popc(__ballot_sync(0xffffffffu, cls == 6));
      const int d0 = __popc(__ballot_sync(0xffffffffu, dbc == 0));  // dB converted / noise-masked
      const int d1 = __popc(__ballot_sync(0xffffffffu, dbc == 1));
      if (lane == 0) {
        if (n0) atomicAdd(&p.counters[0], (unsigned long long)n0);
        if (n2) atomicAdd(&p.counters[2], (unsigned long long)n2);
        if (n6) atomicAdd(&p.counters[6], (unsigned long long)n6);
        if (d0) atomicAdd(&p.counters[kCntDb], (unsigned long long)d0);
        if (d1) atomicAdd(&p.counters[kCntDb + 1], (unsigned long long)d1);
      }
    }
    if (lane == 0) atomicAdd(&p.flags[4], (int)n);
  }
}

// ── k_redo (split precision): FP64 outputs for the flagged pixels ──────────
// Pixels with a mask decision inside its FP32 margin (or more queued
// re-samples than their item holds) get the FP64 candidate of their
// selected member here, outside k_cand's warps; flags[2] counts them.
template <int KERNEL>
__global__ void __launch_bounds__(SEL_THREADS) k_redo(const TcWork *__restrict__ wp) {
  // flagged pixels are sparse: each block first compacts the flagged pixels
  // of a REDO_CHUNK into shared memory, then runs them densely
  __shared__ uint16_t list[REDO_CHUNK];
  __shared__ int n_list;
  const TcWork w = *wp;
  const uint64_t *pre = stage_pre(w, WK_REDO);
  const uint64_t total = pre[w.n_jobs];
  for (uint64_t item = blockIdx.x; item < total; item += gridDim.x) {
    const int jb = find_job(pre, w.n_jobs, item);
    const TcDev &p = w.jobs[jb];
    if (p.flags[3] == 0) continue;  // nothing flagged in this job (uniform over the block)
    const uint64_t npx = p.rows * p.cols;
    const uint64_t base = (item - pre[jb]) * REDO_CHUNK;
    __syncthreads();  // the previous item is done with the list
    if (threadIdx.x == 0) n_list = 0;
    __syncthreads();
    for (int k = 0; k < REDO_CHUNK / SEL_THREADS; ++k) {
      const uint64_t i = base + (uint64_t)k * SEL_THREADS + threadIdx.x;
      if (i < npx && (p.cc[i] & CF_REDO)) list[atomicAdd(&n_list, 1)] = (uint16_t)(i - base);
    }
    __syncthreads();
    const int n = n_list;
    if (n > 0 && threadIdx.x == 0) atomicAdd(&p.flags[2], n);
    for (int q = threadIdx.x; q < n; q += SEL_THREADS) {
      const uint64_t i = base + list[q];
      const uint64_t r = i / p.cols;
      const int code = p.sel[i] & 7;
      const int64_t t = p.fb[i] + (code == SEL_M1 ? 1 : 0);
      V3 P;
      Facet fc;
      const bool ok = target_facet(p, i, &P, &fc);
      OrbitState os;
      double vsq;
      if (!ok || orbit_exact(p.orb, t, &os, &vsq) != ORB_OK) {
        atomicOr(&p.flags[ok ? 0 : 5], 1);
        continue;
      }
      const CandOut o = cand_fp64_tf<KERNEL>(p, P, fc, os.pos, t, p.need_geom ? p.row_flat[r] : 0.0);
      float v = o.data;
      if (p.db) {
        int dc;
        v = db_value(v, p.db_floor, &dc);
        if (dc >= 0) atomicAdd(&p.counters[kCntDb + dc], 1ull);
      }
      p.out[i] = v;
      if (p.compute_lia) {
        p.cos_lia[i] = o.cos;
        p.mask[i] = o.mask;
      }
      atomicAdd(&p.counters[o.cls], 1ull);
    }
  }
}

}  // namespace
}  // namespace sd

namespace sd {
namespace {

// ── work tables and stage launches (host) ───────────────────────────────────
struct TcWorkHost {
  uint64_t totals[kWk];
  TcDev *d_jobs;  // device address of the job records
};

size_t al16(size_t x) { return (x + 15) & ~(size_t)15; }

size_t work_bytes(int n) {
  return al16(sizeof(TcWork)) + al16((size_t)n * sizeof(TcDev)) + (size_t)kWk * (size_t)(n + 1) * 8;
}

uint64_t stage_items(int stage, const TcDev &p) {
  switch (stage) {
    case WK_ANCH: return p.utm ? p.rows * (uint64_t)p.n_pts : 0;
    case WK_ROWS: return p.rows;
    case WK_KNOT: return p.rows * KNOTS;
    case WK_MAIN: return main_items(p);
    case WK_SCAN: return p.rows;
    case WK_REDO: return (p.rows * p.cols + REDO_CHUNK - 1) / REDO_CHUNK;
    default: return (p.rows * p.cols + SEL_THREADS - 1) / SEL_THREADS;
  }
}

// Lays out the table for `n` jobs in host memory `h`, addressed for the
// device copy at `d`: TcWork | TcDev[n] | pre[kWk][n + 1].
void work_layout(const TcDev *jobs, int n, unsigned char *h, unsigned char *d, TcWorkHost *wk) {
  const size_t o_jobs = al16(sizeof(TcWork));
  const size_t o_pre = o_jobs + al16((size_t)n * sizeof(TcDev));
  TcWork w{};
  w.n_jobs = n;
  w.jobs = reinterpret_cast<const TcDev *>(d + o_jobs);
  w.pre = reinterpret_cast<const uint64_t *>(d + o_pre);
  std::memcpy(h, &w, sizeof w);
  std::memcpy(h + o_jobs, jobs, (size_t)n * sizeof(TcDev));
  uint64_t *pre = reinterpret_cast<uint64_t *>(h + o_pre);
  for (int st = 0; st < kWk; ++st) {
    uint64_t acc = 0;
    for (int j = 0; j < n; ++j) {
      pre[st * (n + 1) + j] = acc;
      acc += stage_items(st, jobs[j]);
    }
    pre[st * (n + 1) + n] = acc;
    wk->totals[st] = acc;
  }
  wk->d_jobs = reinterpret_cast<TcDev *>(d + o_jobs);
}

// k_heights' deferral queue for `px` pixels: 1 entry per 64 pixels plus
// 4096 (deferrals are rare; an overflow falls back to a scan), after a
// 16-byte count.
uint64_t heights_queue_cap(uint64_t px) { return std::min<uint64_t>(px / 64 + 4096, 0x7FFFFFFFull); }
size_t heights_queue_bytes(uint64_t px) { return 16 + heights_queue_cap(px) * 8; }

int work_upload(sd_ctx *ctx, const char *name, const TcDev *jobs, int n, TcWorkHost *wk, TcWork **d_work) {
  const size_t bytes = work_bytes(n);
  void *d = nullptr;
  SD_TRY(scratch(ctx, name, bytes, &d));
  std::vector<unsigned char> h(bytes);
  work_layout(jobs, n, h.data(), (unsigned char *)d, wk);
  // k_heights' queue (heights_queue_bytes), its count zeroed ahead of the stages
  const uint64_t px = wk->totals[WK_SEL] * SEL_THREADS;
  const uint64_t cap = heights_queue_cap(px);
  unsigned char *q = nullptr;
  SD_TRY(scratch_t(ctx, (std::string(name) + ".hq").c_str(), heights_queue_bytes(px), &q));
  TcWork *hw = reinterpret_cast<TcWork *>(h.data());
  hw->hq_cnt = reinterpret_cast<unsigned int *>(q);
  hw->hq = reinterpret_cast<unsigned long long *>(q + 16);
  hw->hq_cap = (uint32_t)cap;
  SD_CUDA(ctx, cudaMemsetAsync(q, 0, 4, ctx->stream));
  // pageable source: the copy is staged before the call returns
  SD_CUDA(ctx, cudaMemcpyAsync(d, h.data(), bytes, cudaMemcpyHostToDevice, ctx->stream));
  *d_work = (TcWork *)d;
  return SD_OK;
}

// work blocks of `items` items, `per` per block (~0 = a full resident grid)
uint64_t blocks_for(uint64_t items, unsigned per) { return items == ~0ull ? ~0ull : grid_for(items, per); }

// SARDINE_B200_HEIGHTS_PARAM=0 keeps k_heights in its persistent
// work-table form where the parameter form would run.
inline bool heights_param_enabled() {
  static const bool on = [] {
    const char *e = std::getenv("SARDINE_B200_HEIGHTS_PARAM");
    return !(e && e[0] == '0');
  }();
  return on;
}

// SARDINE_B200_ANCHORS_PARAM=0 keeps k_row_anchors in its persistent
// work-table form where the parameter form would run.
inline bool anchors_param_enabled() {
  static const bool on = [] {
    const char *e = std::getenv("SARDINE_B200_ANCHORS_PARAM");
    return !(e && e[0] == '0');
  }();
  return on;
}

// k_row_anchors in its parameter form for one job on st.
inline int launch_anchors_param(sd_ctx *ctx, const TcDev &job, cudaStream_t st) {
  const uint64_t items = stage_items(WK_ANCH, job);
  if (items == 0) return SD_OK;
  k_row_anchors_param<<<persistent_grid(k_row_anchors_param, 128, 0, blocks_for(items, 128)), 128, 0, st>>>(job);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return set_error(ctx, SD_ERR_CUDA, "kernel launch failed: %s", cudaGetErrorString(e));
  ctx->launches++;
  return SD_OK;
}

// k_heights in its parameter form for job `job` (work-table index jb) on st.
inline int launch_heights_param(sd_ctx *ctx, const TcDev &job, int jb, const TcWork *d_work, cudaStream_t st) {
  const uint64_t items = stage_items(WK_SEL, job);
  if (items == 0) return SD_OK;
  k_heights_param<<<(unsigned)items, SEL_THREADS, 0, st>>>(job, jb, d_work);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return set_error(ctx, SD_ERR_CUDA, "kernel launch failed: %s", cudaGetErrorString(e));
  ctx->launches++;
  return SD_OK;
}

// The pixels k_heights deferred (their count is known on the device only).
int launch_heights_fix(sd_ctx *ctx, const TcWork *d_work, const uint64_t *totals) {
  SD_TIMED_BEGIN(ctx, "k_heights_fix");
  k_heights_fix<<<persistent_grid(k_heights_fix, 128, 0, blocks_for(totals[WK_SEL] == ~0ull ? ~0ull : totals[WK_SEL] * 4, 128)), 128, 0, ctx->stream>>>(
      d_work);
  SD_LAUNCHED(ctx);
  return SD_OK;
}

// Row stages, then k_heights and k_heights_fix unless `heights` is false
// (the caller launches them itself).  single: the one job's record, for the
// parameter form of k_heights.
int launch_rows(sd_ctx *ctx, const TcWork *d_work, const uint64_t *totals, const TcDev *single = nullptr,
                bool heights = true, bool anchors = true) {
  cudaStream_t st = ctx->stream;
  if (anchors && totals[WK_ANCH]) {
    SD_TIMED_BEGIN(ctx, "k_row_anchors");
    if (single && anchors_param_enabled())
      k_row_anchors_param<<<persistent_grid(k_row_anchors_param, 128, 0, blocks_for(totals[WK_ANCH], 128)), 128, 0,
                            st>>>(*single);
    else
      k_row_anchors<<<persistent_grid(k_row_anchors, 128, 0, blocks_for(totals[WK_ANCH], 128)), 128, 0, st>>>(d_work);
    SD_LAUNCHED(ctx);
  }
  SD_TIMED_BEGIN(ctx, "k_row_setup");
  k_row_setup<<<persistent_grid(k_row_setup, 128, 0, blocks_for(totals[WK_ROWS], 128)), 128, 0, st>>>(d_work);
  SD_LAUNCHED(ctx);
  SD_TIMED_BEGIN(ctx, "k_row_model");
  k_row_model<<<persistent_grid(k_row_model, 128, 0, blocks_for(totals[WK_KNOT], 128)), 128, 0, st>>>(d_work);
  SD_LAUNCHED(ctx);
  if (!heights) return SD_OK;
  SD_TIMED_BEGIN(ctx, "k_heights");
  if (single && heights_param_enabled()) {
    SD_TRY(launch_heights_param(ctx, *single, 0, d_work, st));
    ::sd::timing_end(ctx);
  } else {
    k_heights<<<persistent_grid(k_heights, SEL_THREADS, 0, totals[WK_SEL]), SEL_THREADS, 0, st>>>(d_work);
    SD_LAUNCHED(ctx);
  }
  return launch_heights_fix(ctx, d_work, totals);
}

// Stages of launch_pixels_t.
enum : unsigned { PX_MAIN = 1, PX_SCAN = 2, PX_CAND = 4, PX_POST = 8, PX_ALL = 15 };

// SARDINE_B200_CAND_PARAM=0 keeps k_cand in its persistent work-table form
// where the parameter form would run.
inline bool cand_param_enabled() {
  static const bool on = [] {
    const char *e = std::getenv("SARDINE_B200_CAND_PARAM");
    return !(e && e[0] == '0');
  }();
  return on;
}

// k_cand in its parameter form for one job on st, specialised on the job's
// own resampling kernel.
template <bool S>
int launch_cand_param(sd_ctx *ctx, const TcDev &job, cudaStream_t st) {
  const uint64_t items = stage_items(WK_SEL, job);
  if (items == 0) return SD_OK;
  switch (job.resampling) {
    case SD_RESAMPLE_BICUBIC:
      k_cand_param<SD_RESAMPLE_BICUBIC, S>
          <<<persistent_grid(k_cand_param<SD_RESAMPLE_BICUBIC, S>, SEL_THREADS, 0, items), SEL_THREADS, 0, st>>>(job);
      break;
    case SD_RESAMPLE_LANCZOS3:
      k_cand_param<SD_RESAMPLE_LANCZOS3, S>
          <<<persistent_grid(k_cand_param<SD_RESAMPLE_LANCZOS3, S>, SEL_THREADS, 0, items), SEL_THREADS, 0, st>>>(job);
      break;
    default:
      k_cand_param<SD_RESAMPLE_BILINEAR, S>
          <<<persistent_grid(k_cand_param<SD_RESAMPLE_BILINEAR, S>, SEL_THREADS, 0, items), SEL_THREADS, 0, st>>>(job);
  }
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return set_error(ctx, SD_ERR_CUDA, "kernel launch failed: %s", cudaGetErrorString(e));
  ctx->launches++;
  return SD_OK;
}

// job: the single job's record (parameter form of k_main), or null for the
// persistent work-table form.  Stages: k_main (F and codes), k_scan (the row
// walk), k_cand (outputs of the selected members), and in split precision
// k_resample and k_redo (the candidates FP32 could not settle).
template <int K, bool S>
int launch_pixels_t(sd_ctx *ctx, const TcWork *d_work, const uint64_t *totals, const TcDev *job,
                    unsigned stages = PX_ALL) {
  cudaStream_t st = ctx->stream;
  if (stages & PX_MAIN) {
    if (job) {
      if (totals[WK_MAIN] > 0x7FFFFFFFull)
        return set_error(ctx, SD_ERR_INVALID_ARGUMENT, "output grid too large");
      SD_TIMED_BEGIN(ctx, "k_main");
      k_main<<<(unsigned)std::max<uint64_t>(totals[WK_MAIN], 1), MAIN_THREADS, 0, st>>>(*job);
    } else {
      unsigned g = persistent_grid(k_main_batch, MAIN_THREADS, 0, totals[WK_MAIN]);
      if (ctx->main_cps > 0) {
        int dev = 0, sms = 1;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        g = std::min<unsigned>(g, (unsigned)(ctx->main_cps * sms));
      }
      SD_TIMED_BEGIN(ctx, "k_main_batch");
      k_main_batch<<<g, MAIN_THREADS, 0, st>>>(d_work);
    }
    SD_LAUNCHED(ctx);
  }
  if (stages & PX_SCAN) {
    SD_TIMED_BEGIN(ctx, "k_scan");
    k_scan<<<persistent_grid(k_scan, SCAN_WARPS * 32, 0, blocks_for(totals[WK_SCAN], SCAN_WARPS)),
             SCAN_WARPS * 32, 0, st>>>(d_work);
    SD_LAUNCHED(ctx);
  }
  if (stages & PX_CAND) {
    SD_TIMED_BEGIN(ctx, S ? "k_cand<SPLIT>" : "k_cand");
    if (job && K != KDYN && cand_param_enabled())
      k_cand_param<K == KDYN ? 0 : K, S>
          <<<persistent_grid(k_cand_param<K == KDYN ? 0 : K, S>, SEL_THREADS, 0, totals[WK_SEL]), SEL_THREADS, 0, st>>>(
              *job);
    else
      k_cand<K, S><<<persistent_grid(k_cand<K, S>, SEL_THREADS, 0, totals[WK_SEL]), SEL_THREADS, 0, st>>>(d_work);
    SD_LAUNCHED(ctx);
  }
  if (S && (stages & PX_POST)) {
    SD_TIMED_BEGIN(ctx, "k_resample");
    k_resample<K><<<persistent_grid(k_resample<K>, SEL_THREADS, 0, blocks_for(totals[WK_SEL], SEL_THREADS / 32)),
                    SEL_THREADS, 0, st>>>(d_work);
    SD_LAUNCHED(ctx);
    SD_TIMED_BEGIN(ctx, "k_redo");
    k_redo<K><<<persistent_grid(k_redo<K>, SEL_THREADS, 0, totals[WK_REDO]), SEL_THREADS, 0, st>>>(d_work);
    SD_LAUNCHED(ctx);
  }
  return SD_OK;
}

// FP64 Lagrange state at every microsecond of [t0, t1] into scratch `name`
// (capped at 96 M entries, 7.7 GB, centred on [tmin, tmax]), and the orbit
// expansions over it into scratch `tay_name`.
int build_orbit_table(sd_ctx *ctx, const char *name, const char *tay_name, const sd_state_vector *d_svs,
                      uint64_t nsv, int64_t t0, int64_t t1, int64_t tmin, int64_t tmax, OrbitDev *orb) {
  const int64_t max_entries = 96ll * 1000 * 1000;
  if (t1 - t0 + 1 > max_entries) {
    const int64_t mid = (tmin / 2 + tmax / 2);
    t0 = std::max(t0, mid - max_entries / 2);
    t1 = std::min(t1, t0 + max_entries - 1);
  }
  if (t1 < t0) return SD_OK;
  double2 *d_tab;
  SD_TRY(scratch_t(ctx, name, (size_t)(t1 - t0 + 1) * 5, &d_tab));
  SD_TIMED_BEGIN(ctx, "k_orbit_table");
  k_orbit_table<<<grid_for((size_t)(t1 - t0 + 1), 128), 128, 0, ctx->stream>>>(d_svs, nsv, t0, t1 - t0 + 1, d_tab);
  SD_LAUNCHED(ctx);
  orb->tab = d_tab;
  orb->tab_t0 = t0;
  orb->tab_n = t1 - t0 + 1;
  OrbTaylor *d_tay;
  SD_TRY(scratch_t(ctx, tay_name, (size_t)tay_count(orb->tab_n), &d_tay));
  return launch_orbit_taylor(ctx, orb, d_tay);
}

// Window polynomials of the orbit (orbit_poly_build) in scratch `name`.
int upload_orbit_poly(sd_ctx *ctx, const char *name, const sd_state_vector *svs, uint64_t nsv,
                      OrbitDev *orb) {
  if (nsv < 8) return SD_OK;  // the solve reports the reference's orbit error
  std::vector<OrbPoly> w(nsv - 7);
  orbit_poly_build(svs, nsv, w.data());
  OrbPoly *d = nullptr;
  SD_TRY(scratch_t(ctx, name, w.size(), &d));
  SD_CUDA(ctx, cudaMemcpyAsync(d, w.data(), w.size() * sizeof(OrbPoly), cudaMemcpyHostToDevice, ctx->stream));
  orb->poly = d;
  return SD_OK;
}

}  // namespace
}  // namespace sd
