// InSAR after deramping: co-registration resampling of the secondary
// (resample_secondary, insar/coreg.rs:230-264) and interferogram formation
// with coherence (form_interferogram, insar/interferogram.rs:165-398).
//
// k_coreg_resample: one thread per reference pixel; the degree-2 offset
//   polynomials in f64 and the f32 bilinear gather of coreg.rs:428-456.
// k_igram: one thread per pixel; the flat-earth point by the 3x3 Newton
//   solve of ecef_from_slant_range_doppler (coreg.rs:280-362) from the
//   line's reference state, the secondary range, the f32 flat-earth phase,
//   its FP64 sincos and the cross-product.  It writes {Re, Im, |ref|^2,
//   |sec|^2} as one float4 a pixel; the satellite states per line come from
//   the host (orbit_eval, the reference's Lagrange interpolation).
// k_coherence: the boxcar sums in f64, each output in the reference's
//   order (window rows ascending, columns ascending within a row), so the
//   sums equal a sequential evaluation bit for bit.  A thread owns R
//   outputs of one column on consecutive rows; every window pixel it loads
//   is added to each of its outputs whose window holds that row, which
//   keeps each output's order and shares the load.  A window row feeding
//   outputs 0..k or k..R-1 (every row, once the half window is at least
//   (R - 1) / 2) runs an add loop compiled for that range, so no add is
//   issued under a false predicate.  The block's window rows and columns
//   are staged in shared memory when they fit in 96 KB (otherwise the loads
//   go through L1).
#include <cmath>
#include <vector>

#include "geo.cuh"
#include "runtime.cuh"

namespace sd {
namespace {

constexpr double kC = 299792458.0;
constexpr double kA = 6378137.0, kB = 6356752.314245;  // WGS84 (interferogram.rs / coreg.rs)
constexpr int kCohThreads = 128;
constexpr int kCohRows = 8;

__device__ __forceinline__ double poly6(const double *p, double l, double c) {
  return p[0] + p[1] * l + p[2] * c + p[3] * l * l + p[4] * l * c + p[5] * c * c;
}

struct Poly12 {
  double az[6], rg[6];
};

__global__ void k_coreg_resample(const float2 *__restrict__ sec, uint64_t sl, uint64_t ss, uint64_t lines,
                                 uint32_t samples, Poly12 p, float2 *__restrict__ out) {
  const uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= samples) return;
  const double cf = (double)c;
  for (uint64_t l = blockIdx.y; l < lines; l += gridDim.y) {
    const double lf = (double)l;
    const double ls = lf + poly6(p.az, lf, cf), cs = cf + poly6(p.rg, lf, cf);
    float2 o = make_float2(0.0f, 0.0f);
    if (!(ls < 0.0 || cs < 0.0)) {
      const double lfl = floor(ls), cfl = floor(cs);
      // `as usize`: NaN -> 0; indices at or past the end only need to fail the bounds test
      const uint64_t l0 = lfl == lfl ? (lfl < (double)sl ? (uint64_t)lfl : sl) : 0;
      const uint64_t c0 = cfl == cfl ? (cfl < (double)ss ? (uint64_t)cfl : ss) : 0;
      if (l0 + 1 < sl && c0 + 1 < ss) {
        const float wl = (float)(ls - (double)l0), wc = (float)(cs - (double)c0);
        const float2 p00 = __ldg(sec + l0 * ss + c0), p01 = __ldg(sec + l0 * ss + c0 + 1);
        const float2 p10 = __ldg(sec + (l0 + 1) * ss + c0), p11 = __ldg(sec + (l0 + 1) * ss + c0 + 1);
        const float i0 = p00.x + (p01.x - p00.x) * wc, i1 = p10.x + (p11.x - p10.x) * wc;
        const float q0 = p00.y + (p01.y - p00.y) * wc, q1 = p10.y + (p11.y - p10.y) * wc;
        o = make_float2(i0 + (i1 - i0) * wl, q0 + (q1 - q0) * wl);
      }
    }
    out[l * samples + c] = o;
  }
}

// ecef_from_slant_range_doppler (coreg.rs:280-362).
__device__ bool flat_point(const double *sp, const double *sv, double r, double *t, int max_iter = 10,
                           double tol_m = 1.0) {
  const double px = sp[0], py = sp[1], pz = sp[2], vx = sv[0], vy = sv[1], vz = sv[2];
  const double a = kA, b = kB;
  const double sat_r = sqrt(px * px + py * py + pz * pz);
  const double scale = a / sat_r;
  double tx = px * scale, ty = py * scale, tz = pz * scale * (b / a);
  for (int it = 0; it < max_iter; ++it) {
    const double dx = tx - px, dy = ty - py, dz = tz - pz;
    const double f1 = dx * vx + dy * vy + dz * vz;
    const double f2 = dx * dx + dy * dy + dz * dz - r * r;
    const double f3 = tx * tx / (a * a) + ty * ty / (a * a) + tz * tz / (b * b) - 1.0;
    const double j00 = vx, j01 = vy, j02 = vz;
    const double j10 = 2.0 * dx, j11 = 2.0 * dy, j12 = 2.0 * dz;
    const double j20 = 2.0 * tx / (a * a), j21 = 2.0 * ty / (a * a), j22 = 2.0 * tz / (b * b);
    const double det = j00 * (j11 * j22 - j12 * j21) - j01 * (j10 * j22 - j12 * j20) + j02 * (j10 * j21 - j11 * j20);
    if (fabs(det) < 1e-20) return false;
    const double dxt = (f1 * (j11 * j22 - j12 * j21) - j01 * (f2 * j22 - j12 * f3) + j02 * (f2 * j21 - j11 * f3)) / det;
    const double dyt = (j00 * (f2 * j22 - j12 * f3) - f1 * (j10 * j22 - j12 * j20) + j02 * (j10 * f3 - f2 * j20)) / det;
    const double dzt = (j00 * (j11 * f3 - f2 * j21) - j01 * (j10 * f3 - f2 * j20) + f1 * (j10 * j21 - j11 * j20)) / det;
    tx -= dxt;
    ty -= dyt;
    tz -= dzt;
    if (sqrt(dxt * dxt + dyt * dyt + dzt * dzt) < tol_m) {
      t[0] = tx, t[1] = ty, t[2] = tz;
      return true;
    }
  }
  return false;
}


constexpr int kGridAz = 20, kGridRg = 50;  // GRID_AZ, GRID_RG (coreg.rs:54-56)

struct CoregGeom {
  const sd_state_vector *ro, *so;
  uint64_t nr, ns;
  int64_t ref_first, sec_first;
  double ref_ati, ref_tau0, ref_dtau, ref_off, sec_ati, sec_tau0, sec_dtau, sec_off, az_step, rg_step;
};

// One sparse grid point of compute_coreg_offsets (coreg.rs:159-207): forward
// geocoding of the reference pixel (20 iterations, 1 mm), solve_zero_doppler
// on the secondary orbit from its first line (20 iterations, 1e-9 s;
// terrain_correction.rs:1010-1073) and secondary_sar_coords (coreg.rs:371-414).
__global__ void k_coreg_grid(CoregGeom g, double4 *pts, int *ok) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= kGridAz * kGridRg) return;
  ok[i] = 0;
  const int gi = i / kGridRg, gj = i - gi * kGridRg;
  const double l = (double)(gi + 1) * g.az_step, c = (double)(gj + 1) * g.rg_step;
  const int64_t t_ref = g.ref_first + f2i64(l * g.ref_ati * 1e6);
  const double range_m = (g.ref_tau0 + (c + g.ref_off) * g.ref_dtau) * kC / 2.0;
  OrbitState s;
  if (orbit_eval(g.ro, g.nr, t_ref, &s) != ORB_OK) return;
  const double sp[3] = {s.pos.x, s.pos.y, s.pos.z}, sv[3] = {s.vel.x, s.vel.y, s.vel.z};
  double P[3];
  if (!flat_point(sp, sv, range_m, P, 20, 1e-3)) return;
  int64_t t = g.sec_first;
  bool conv = false;
  OrbitState q;
  for (int it = 0; it < 20; ++it) {
    if (orbit_eval(g.so, g.ns, t, &q) != ORB_OK) return;
    const double rx = P[0] - q.pos.x, ry = P[1] - q.pos.y, rz = P[2] - q.pos.z;
    const double f = rx * q.vel.x + ry * q.vel.y + rz * q.vel.z;
    const double vsq = q.vel.x * q.vel.x + q.vel.y * q.vel.y + q.vel.z * q.vel.z;
    const double fp = -vsq + (rx * q.acc.x + ry * q.acc.y + rz * q.acc.z);
    if (fabs(fp) < 1.0) return;
    const double delta = -f / fp;
    if (fabs(delta) < 1e-9) {
      conv = true;
      break;
    }
    t = t + f2i64(delta * 1e6);
  }
  if (!conv) return;
  const double l_sec = (double)(t - g.sec_first) / (g.sec_ati * 1e6);
  const double dx = P[0] - q.pos.x, dy = P[1] - q.pos.y, dz = P[2] - q.pos.z;
  const double rng = sqrt(dx * dx + dy * dy + dz * dz);
  const double c_sec = (2.0 * rng / kC - g.sec_tau0) / g.sec_dtau - g.sec_off;
  pts[i] = make_double4(l, c, l_sec - l, c_sec - c);
  ok[i] = 1;
}

__global__ void __launch_bounds__(128, 7) k_igram(const float2 *__restrict__ ref, const float2 *__restrict__ sec,
                        const double *__restrict__ st, uint64_t lines, uint32_t samples, double srt, double dtau,
                        double col_off, double k, float4 *__restrict__ out) {
  const uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= samples) return;
  const double tau = srt + ((double)c + col_off) * dtau;
  const double r_ref = tau * kC / 2.0;
  for (uint64_t l = blockIdx.y; l < lines; l += gridDim.y) {
    double s[9];  // reference position, velocity; secondary position
#pragma unroll
    for (int j = 0; j < 9; ++j) s[j] = __ldg(st + 9 * l + j);
    double p[3];
    float fe = 0.0f;  // a point that does not converge keeps a zero flat-earth phase
    if (flat_point(s, s + 3, r_ref, p)) {
      const double dx = s[6] - p[0], dy = s[7] - p[1], dz = s[8] - p[2];
      const double r_sec = sqrt(dx * dx + dy * dy + dz * dz);
      fe = (float)(k * 2.0 * (r_ref - r_sec));
    }
    const uint64_t i = l * samples + c;
    const float2 rv = __ldg(ref + i), sv = __ldg(sec + i);
    double sn, cs;
    sincos((double)fe, &sn, &cs);
    const double re = (double)sv.x * cs + (double)sv.y * sn;
    const double im = (double)sv.x * sn - (double)sv.y * cs;
    out[i] = make_float4((float)((double)rv.x * re - (double)rv.y * im), (float)((double)rv.x * im + (double)rv.y * re),
                         rv.x * rv.x + rv.y * rv.y, sv.x * sv.x + sv.y * sv.y);
  }
}

// window pixels of one window row added to outputs LO..HI of the thread;
// `row` is the tile row (its columns start at xo) or the image row (xo 0)
template <int R, int LO, int HI, bool SMEM>
__device__ __forceinline__ void coh_row(double (&acc)[R][4], const float4 *row, int64_t c0, int64_t c1,
                                        int64_t xo) {
  for (int64_t x = c0; x < c1; ++x) {
    const float4 v = SMEM ? row[x - xo] : __ldg(row + x);
    const double d0 = v.x, d1 = v.y, d2 = v.z, d3 = v.w;
#pragma unroll
    for (int r = LO; r <= HI; ++r) {
      acc[r][0] += d0;
      acc[r][1] += d1;
      acc[r][2] += d2;
      acc[r][3] += d3;
    }
  }
}

// window pixels of one window row added to outputs lo..hi (runtime range, predicated adds)
template <int R, bool SMEM>
__device__ __forceinline__ void coh_row_any(int lo, int hi, double (&acc)[R][4], const float4 *row, int64_t c0,
                                            int64_t c1, int64_t xo) {
  for (int64_t x = c0; x < c1; ++x) {
    const float4 v = SMEM ? row[x - xo] : __ldg(row + x);
    const double d0 = v.x, d1 = v.y, d2 = v.z, d3 = v.w;
#pragma unroll
    for (int r = 0; r < R; ++r)
      if (r >= lo && r <= hi) {
        acc[r][0] += d0;
        acc[r][1] += d1;
        acc[r][2] += d2;
        acc[r][3] += d3;
      }
  }
}

// outputs 0..hi: coh_row<0, K> for K == hi
template <int R, bool SMEM, int K = 0>
__device__ __forceinline__ void coh_prefix(int hi, double (&acc)[R][4], const float4 *row, int64_t c0, int64_t c1,
                                           int64_t xo) {
  if (hi == K) return coh_row<R, 0, K, SMEM>(acc, row, c0, c1, xo);
  if constexpr (K + 1 < R) coh_prefix<R, SMEM, K + 1>(hi, acc, row, c0, c1, xo);
}

// outputs lo..R-1: coh_row<K, R - 1> for K == lo
template <int R, bool SMEM, int K = 1>
__device__ __forceinline__ void coh_suffix(int lo, double (&acc)[R][4], const float4 *row, int64_t c0, int64_t c1,
                                           int64_t xo) {
  if (lo == K) return coh_row<R, K, R - 1, SMEM>(acc, row, c0, c1, xo);
  if constexpr (K + 1 < R) coh_suffix<R, SMEM, K + 1>(lo, acc, row, c0, c1, xo);
}

// the window row's outputs [lo, hi] (0 <= lo <= hi < R).  When the half
// window is at least (R - 1) / 2 every range holds output 0 or output R - 1,
// and those ranges have loops of their own (2R - 1 of them); ranges inside
// (small windows only) take the predicated loop.
template <int R, bool SMEM>
__device__ __forceinline__ void coh_dispatch(int lo, int hi, double (&acc)[R][4], const float4 *row, int64_t c0,
                                             int64_t c1, int64_t xo) {
  if (lo == 0)
    coh_prefix<R, SMEM>(hi, acc, row, c0, c1, xo);
  else if (hi == R - 1)
    coh_suffix<R, SMEM>(lo, acc, row, c0, c1, xo);
  else
    coh_row_any<R, SMEM>(lo, hi, acc, row, c0, c1, xo);
}

template <int R, bool SMEM>
__global__ void __launch_bounds__(kCohThreads) k_coherence(const float4 *__restrict__ ig, int64_t lines,
                                                           int64_t samples, int64_t ah, int64_t rh,
                                                           float *__restrict__ coh, float *__restrict__ phase) {
  extern __shared__ float4 tile[];  // trows x tcols window pixels {Re, Im, |ref|^2, |sec|^2}
  const int64_t cb = (int64_t)blockIdx.x * kCohThreads;
  const int64_t c = cb + threadIdx.x;
  const int64_t tcols = kCohThreads + 2 * rh, trows = R + 2 * ah, ps = trows * tcols;
  for (int64_t lb = (int64_t)blockIdx.y * R; lb < lines; lb += (int64_t)gridDim.y * R) {
    if (SMEM) {
      __syncthreads();  // the previous group's reads are done
      for (int64_t e = threadIdx.x; e < ps; e += kCohThreads) {
        const int64_t tr = e / tcols, tc = e - tr * tcols;
        const int64_t gl = lb - ah + tr, gc = cb - rh + tc;
        tile[e] = (gl >= 0 && gl < lines && gc >= 0 && gc < samples) ? __ldg(ig + gl * samples + gc)
                                                                       : make_float4(0.f, 0.f, 0.f, 0.f);
      }
      __syncthreads();
    }
    if (c >= samples) continue;
    const int64_t c0 = c > rh ? c - rh : 0, c1 = c + rh + 1 < samples ? c + rh + 1 : samples;
    const int64_t wlo = lb > ah ? lb - ah : 0;
    const int64_t whi = lb + R + ah < lines ? lb + R + ah : lines;
    double acc[R][4];
#pragma unroll
    for (int r = 0; r < R; ++r) acc[r][0] = acc[r][1] = acc[r][2] = acc[r][3] = 0.0;
    for (int64_t wl = wlo; wl < whi; ++wl) {
      // outputs lb + r whose window holds row wl: |wl - (lb + r)| <= ah, a range [lo, hi] with lo <= hi
      const int64_t d = wl - lb;
      const int lo = (int)(d - ah > 0 ? d - ah : 0), hi = (int)(d + ah < R - 1 ? d + ah : R - 1);
      // in the tile the window row's columns start at cb - rh
      coh_dispatch<R, SMEM>(lo, hi, acc, SMEM ? tile + (d + ah) * tcols : ig + wl * samples, c0, c1,
                            SMEM ? cb - rh : 0);
    }
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const int64_t l = lb + r;
      if (l >= lines) break;
      const double den = sqrt(acc[r][2] * acc[r][3]);
      coh[l * samples + c] =
          den > 0.0 ? (float)fmin(sqrt(acc[r][0] * acc[r][0] + acc[r][1] * acc[r][1]) / den, 1.0) : 0.0f;
      if (phase) phase[l * samples + c] = (float)atan2(acc[r][1], acc[r][0]);
    }
  }
}

}  // namespace
}  // namespace sd

using namespace sd;

extern "C" int sd_resample_secondary(sd_ctx *ctx, const float *sec, uint64_t sec_lines, uint64_t sec_samples,
                                     uint64_t lines, uint64_t samples, const double *az_poly, const double *rg_poly,
                                     float *out) {
  SD_STAGE("resample_secondary");
  if (!ctx) return SD_ERR_INVALID_ARGUMENT;
  if (!az_poly || !rg_poly) return set_error(ctx, SD_ERR_INVALID_ARGUMENT, "null polynomial");
  if (samples > 0xffffffffull) return set_error(ctx, SD_ERR_INVALID_ARGUMENT, "too many samples per line");
  if (lines == 0 || samples == 0) return SD_OK;
  if (!out || (!sec && sec_lines * sec_samples)) return set_error(ctx, SD_ERR_INVALID_ARGUMENT, "null buffer");
  SD_CUDA(ctx, cudaSetDevice(ctx->device));
  Poly12 p;
  for (int j = 0; j < 6; ++j) p.az[j] = az_poly[j], p.rg[j] = rg_poly[j];
  const void *din = nullptr;
  void *dout;
  if (sec_lines * sec_samples) SD_TRY(stage_in(ctx, "co.sec", sec, sec_lines * sec_samples * 8, &din));
  SD_TRY(stage_out(ctx, "co.out", out, lines * samples * 8, &dout));
  const dim3 grid((unsigned)((samples + 255) / 256), (unsigned)(lines < 65535 ? lines : 65535));
  SD_TIMED_BEGIN(ctx, "k_coreg_resample");
  k_coreg_resample<<<grid, 256, 0, ctx->stream>>>((const float2 *)din, sec_lines, sec_samples, lines,
                                                  (uint32_t)samples, p, (float2 *)dout);
  SD_LAUNCHED(ctx);
  SD_TRY(finish_out(ctx, out, dout, lines * samples * 8));
  return sync(ctx);
}

extern "C" int sd_form_interferogram(sd_ctx *ctx, const float *ref, const float *sec, uint64_t lines,
                                     uint64_t samples, uint64_t valid_sample_offset, double slant_range_time_s,
                                     double range_pixel_spacing_m, double azimuth_time_interval_s,
                                     const sd_state_vector *ref_orbit, uint64_t n_ref, int64_t ref_first_us,
                                     const sd_state_vector *sec_orbit, uint64_t n_sec, double wavelength_m,
                                     uint32_t az_looks, uint32_t rg_looks, float *coherence, float *phase) {
  SD_STAGE("interferogram");
  if (!ctx) return SD_ERR_INVALID_ARGUMENT;
  if (az_looks == 0 || rg_looks == 0)
    return set_error(ctx, SD_ERR_INSAR_INVALID_WINDOW_SIZE,
                     "coherence estimation window size must be > 0, got az=%u rg=%u", az_looks, rg_looks);
  if (samples > 0x7fffffffull) return set_error(ctx, SD_ERR_INVALID_ARGUMENT, "too many samples per line");
  if (!ref_orbit || !sec_orbit) return set_error(ctx, SD_ERR_INVALID_ARGUMENT, "null orbit");
  // the satellite states of every line (interferogram.rs:206-212), on the host
  std::vector<double> st(9 * lines);
  for (uint64_t l = 0; l < lines; ++l) {
    const int64_t t = ref_first_us + (int64_t)((double)l * azimuth_time_interval_s * 1e6);
    OrbitState a, b;
    const int ra = orbit_eval(ref_orbit, n_ref, t, &a), rb = ra ? ra : orbit_eval(sec_orbit, n_sec, t, &b);
    if (ra || rb)
      return set_error(ctx, SD_ERR_INSAR_ORBIT, "orbit interpolation error: %s",
                       (ra ? ra : rb) == ORB_INSUFFICIENT ? "insufficient state vectors for interpolation"
                                                          : "interpolation time outside orbit window");
    double *q = st.data() + 9 * l;
    q[0] = a.pos.x, q[1] = a.pos.y, q[2] = a.pos.z, q[3] = a.vel.x, q[4] = a.vel.y, q[5] = a.vel.z;
    q[6] = b.pos.x, q[7] = b.pos.y, q[8] = b.pos.z;
  }
  if (lines == 0 || samples == 0) return SD_OK;
  if (!ref || !sec || !coherence) return set_error(ctx, SD_ERR_INVALID_ARGUMENT, "null buffer");
  SD_CUDA(ctx, cudaSetDevice(ctx->device));
  cudaStream_t s = ctx->stream;
  const uint64_t n = lines * samples;
  const void *dref, *dsec;
  void *dcoh, *dph = nullptr;
  double *dst;
  float4 *dig;
  SD_TRY(stage_in(ctx, "ig.ref", ref, n * 8, &dref));
  SD_TRY(stage_in(ctx, "ig.sec", sec, n * 8, &dsec));
  SD_TRY(stage_out(ctx, "ig.coh", coherence, n * 4, &dcoh));
  if (phase) SD_TRY(stage_out(ctx, "ig.phase", phase, n * 4, &dph));
  SD_TRY(scratch_t(ctx, "ig.states", 9 * lines, &dst));
  SD_TRY(scratch_t(ctx, "ig.buf", n, &dig));
  SD_CUDA(ctx, cudaMemcpyAsync(dst, st.data(), lines * 72, cudaMemcpyHostToDevice, s));
  const double dtau = 2.0 * range_pixel_spacing_m / kC;
  const double k = 6.283185307179586 / wavelength_m;
  const dim3 g1((unsigned)((samples + 127) / 128), (unsigned)(lines < 65535 ? lines : 65535));
  SD_TIMED_BEGIN(ctx, "k_igram");
  k_igram<<<g1, 128, 0, s>>>((const float2 *)dref, (const float2 *)dsec, dst, lines, (uint32_t)samples,
                             slant_range_time_s, dtau, (double)valid_sample_offset, k, dig);
  SD_LAUNCHED(ctx);
  const int64_t ah = az_looks / 2, rh = rg_looks / 2;
  const size_t smem = (size_t)(kCohRows + 2 * ah) * (size_t)(kCohThreads + 2 * rh) * sizeof(float4);
  const uint64_t groups = (lines + kCohRows - 1) / kCohRows;
  const dim3 g2((unsigned)((samples + kCohThreads - 1) / kCohThreads), (unsigned)(groups < 65535 ? groups : 65535));
  SD_TIMED_BEGIN(ctx, "k_coherence");
  if (smem <= 96 * 1024) {
    SD_CUDA(ctx, cudaFuncSetAttribute(k_coherence<kCohRows, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)smem));
    k_coherence<kCohRows, true><<<g2, kCohThreads, smem, s>>>(dig, (int64_t)lines, (int64_t)samples, ah, rh,
                                                             (float *)dcoh, (float *)dph);
  } else {
    k_coherence<kCohRows, false><<<g2, kCohThreads, 0, s>>>(dig, (int64_t)lines, (int64_t)samples, ah, rh,
                                                           (float *)dcoh, (float *)dph);
  }
  SD_LAUNCHED(ctx);
  SD_TRY(finish_out(ctx, coherence, dcoh, n * 4));
  if (phase) SD_TRY(finish_out(ctx, phase, dph, n * 4));
  return sync(ctx);  // the host state table lives until here
}

namespace sd {
namespace {
// gaussian_elimination (coreg.rs:522-568): partial pivoting (the last row of
// the largest magnitude, as Iterator::max_by), 1e-12 pivot floor.
bool gauss6(double a[6][6], double b[6], double x[6]) {
  for (int col = 0; col < 6; ++col) {
    int p = col;
    for (int r = col + 1; r < 6; ++r)
      if (fabs(a[r][col]) >= fabs(a[p][col])) p = r;
    for (int k = 0; k < 6; ++k) std::swap(a[col][k], a[p][k]);
    std::swap(b[col], b[p]);
    if (fabs(a[col][col]) < 1e-12) return false;
    const double inv = 1.0 / a[col][col];
    for (int r = col + 1; r < 6; ++r) {
      const double f = a[r][col] * inv;
      for (int k = col; k < 6; ++k) a[r][k] -= f * a[col][k];
      b[r] -= f * b[col];
    }
  }
  for (int i = 5; i >= 0; --i) {
    double sum = b[i];
    for (int j = i + 1; j < 6; ++j) sum -= a[i][j] * x[j];
    x[i] = sum / a[i][i];
  }
  return true;
}

// fit_poly6 (coreg.rs:478-517) of value k (2: dl, 3: dc) of the points.
bool fit6(const std::vector<double4> &pts, int k, double coef[6], double *rms) {
  double ata[6][6] = {}, atb[6] = {};
  for (const double4 &q : pts) {
    const double l = q.x, c = q.y, y = k == 2 ? q.z : q.w;
    const double bs[6] = {1.0, l, c, l * l, l * c, c * c};
    for (int i = 0; i < 6; ++i) {
      atb[i] += bs[i] * y;
      for (int j = 0; j < 6; ++j) ata[i][j] += bs[i] * bs[j];
    }
  }
  if (!gauss6(ata, atb, coef)) return false;
  double sse = 0.0;
  for (const double4 &q : pts) {
    const double l = q.x, c = q.y, y = k == 2 ? q.z : q.w;
    const double res = y - (coef[0] + coef[1] * l + coef[2] * c + coef[3] * l * l + coef[4] * l * c + coef[5] * c * c);
    sse += res * res;
  }
  *rms = std::sqrt(sse / (double)pts.size());
  return true;
}
}  // namespace
}  // namespace sd

extern "C" int sd_coreg_offsets(sd_ctx *ctx, const sd_state_vector *ref_orbit, uint64_t n_ref, int64_t ref_first_us,
                                uint64_t ref_lines, uint64_t ref_samples, uint64_t ref_valid_sample_offset,
                                double ref_azimuth_time_interval_s, double ref_slant_range_time_s,
                                double ref_range_pixel_spacing_m, const sd_state_vector *sec_orbit, uint64_t n_sec,
                                int64_t sec_first_us, double sec_azimuth_time_interval_s,
                                double sec_slant_range_time_s, double sec_range_pixel_spacing_m,
                                uint64_t sec_first_sample, sd_coreg_result *out) {
  SD_STAGE("coreg_offsets");
  if (!ctx) return SD_ERR_INVALID_ARGUMENT;
  if (!ref_orbit || !sec_orbit || !out) return set_error(ctx, SD_ERR_INVALID_ARGUMENT, "null argument");
  SD_CUDA(ctx, cudaSetDevice(ctx->device));
  cudaStream_t s = ctx->stream;
  const void *dro, *dso;
  double4 *dpts;
  int *dok;
  SD_TRY(stage_in(ctx, "cg.ro", ref_orbit, n_ref * sizeof(sd_state_vector), &dro));
  SD_TRY(stage_in(ctx, "cg.so", sec_orbit, n_sec * sizeof(sd_state_vector), &dso));
  SD_TRY(scratch_t(ctx, "cg.pts", kGridAz * kGridRg, &dpts));
  SD_TRY(scratch_t(ctx, "cg.ok", kGridAz * kGridRg, &dok));
  CoregGeom g;
  g.ro = (const sd_state_vector *)dro, g.so = (const sd_state_vector *)dso, g.nr = n_ref, g.ns = n_sec;
  g.ref_first = ref_first_us, g.sec_first = sec_first_us;
  g.ref_ati = ref_azimuth_time_interval_s, g.ref_tau0 = ref_slant_range_time_s;
  g.ref_dtau = 2.0 * ref_range_pixel_spacing_m / kC, g.ref_off = (double)ref_valid_sample_offset;
  g.sec_ati = sec_azimuth_time_interval_s, g.sec_tau0 = sec_slant_range_time_s;
  g.sec_dtau = 2.0 * sec_range_pixel_spacing_m / kC, g.sec_off = (double)sec_first_sample;
  g.az_step = (double)ref_lines / (double)(kGridAz + 1), g.rg_step = (double)ref_samples / (double)(kGridRg + 1);
  SD_TIMED_BEGIN(ctx, "k_coreg_grid");
  k_coreg_grid<<<(kGridAz * kGridRg + 127) / 128, 128, 0, s>>>(g, dpts, dok);
  SD_LAUNCHED(ctx);
  std::vector<double4> pts(kGridAz * kGridRg);
  std::vector<int> ok(kGridAz * kGridRg);
  SD_CUDA(ctx, cudaMemcpyAsync(pts.data(), dpts, pts.size() * sizeof(double4), cudaMemcpyDeviceToHost, s));
  SD_CUDA(ctx, cudaMemcpyAsync(ok.data(), dok, ok.size() * sizeof(int), cudaMemcpyDeviceToHost, s));
  SD_TRY(sync(ctx));
  std::vector<double4> valid;  // grid order, as the reference's collect
  for (size_t i = 0; i < pts.size(); ++i)
    if (ok[i]) valid.push_back(pts[i]);
  out->n_valid = valid.size();
  if (valid.size() < 6)
    return set_error(ctx, SD_ERR_INSAR_COREG_GRID_TOO_SMALL,
                     "co-registration: need at least 6 valid grid points for polynomial fit, got %zu", valid.size());
  double ra, rr;
  if (!fit6(valid, 2, out->az_poly, &ra) || !fit6(valid, 3, out->rg_poly, &rr)) {
    out->n_valid = 0;
    return set_error(ctx, SD_ERR_INSAR_COREG_GRID_TOO_SMALL,
                     "co-registration: need at least 6 valid grid points for polynomial fit, got 0");
  }
  out->fit_residual_rms = std::sqrt((ra * ra + rr * rr) / 2.0);
  return SD_OK;
}
