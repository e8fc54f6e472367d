// TOPS azimuth deramping of a debursted IW SLC sub-swath (deramp_subswath,
// insar/deramp.rs:114-210).  Every CInt16 sample is rotated by
// exp(-j 2 pi f_DC(tau_c) t_az(l)), promoted to complex f32.
//
// The Doppler-centroid polynomial changes only along azimuth, so the host
// interpolates one (a0, a1, a2, t0) per line between the two bracketing
// estimates (interp_dc_poly, deramp.rs:227-276) and uploads them (32 B a
// line).  The device does the per-pixel part: slant-range time of the
// column, f_DC, the phase and its FP64 sincos, and the complex product, one
// thread per pixel with lines on grid.y.  HBM traffic is 4 B read + 8 B
// written a pixel; the FP64 sincos is the other bound.
#include <cmath>
#include <vector>

#include "runtime.cuh"

namespace sd {
namespace {

constexpr double kSpeedOfLight = 299792458.0;  // types.rs:11
constexpr double kTau = 6.283185307179586;      // std::f64::consts::TAU

__global__ void k_deramp(const short2 *__restrict__ in, const double2 *__restrict__ poly, uint64_t lines,
                         uint32_t samples, double near_tau, double dtau, uint64_t col_off, double ati,
                         float2 *__restrict__ out) {
  const uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= samples) return;
  // tau_col (deramp.rs:137-139)
  const double tau = near_tau + (double)(c + col_off) * dtau;
  for (uint64_t l = blockIdx.y; l < lines; l += gridDim.y) {
    const double2 p01 = __ldg(poly + 2 * l), p23 = __ldg(poly + 2 * l + 1);  // a0, a1 | a2, t0 of this line
    const double dt = tau - p23.y;
    const double f_dc = p01.x + p01.y * dt + p23.x * dt * dt;
    const double t_az = (double)l * ati;
    const double phi = kTau * f_dc * t_az;
    double s, co;
    sincos(phi, &s, &co);
    const uint64_t i = l * samples + c;
    const short2 v = __ldg(in + i);
    const double iv = (double)v.x, qv = (double)v.y;
    out[i] = make_float2((float)(iv * co + qv * s), (float)(qv * co - iv * s));
  }
}

}  // namespace
}  // namespace sd

using namespace sd;

extern "C" int sd_deramp_subswath(sd_ctx *ctx, const int16_t *iq, uint64_t lines, uint64_t samples,
                                  uint64_t valid_sample_offset, double slant_range_time_s,
                                  double range_pixel_spacing_m, double azimuth_time_interval_s,
                                  const sd_dc_estimate *estimates, uint64_t n_estimates, int64_t burst_start_us,
                                  int32_t swath_id, float *out) {
  SD_STAGE("deramp");
  if (!ctx) return SD_ERR_INVALID_ARGUMENT;
  if (n_estimates == 0 || !estimates)
    return set_error(ctx, SD_ERR_INSAR_NO_DC_ESTIMATES,
                     "subswath IW%d has no Doppler centroid estimates; InSAR requires an IW/EW SLC product with a "
                     "<dopplerCentroid> block",
                     swath_id);
  if (samples > 0xffffffffull) return set_error(ctx, SD_ERR_INVALID_ARGUMENT, "too many samples per line");
  // est_times_s (deramp.rs:150-158): microseconds since the first line, in seconds
  std::vector<double> et(n_estimates);
  for (uint64_t k = 0; k < n_estimates; ++k)
    et[k] = (double)(estimates[k].azimuth_time_us - burst_start_us) / 1e6;
  // line_poly (deramp.rs:163-169) by interp_dc_poly (227-276)
  const uint64_t n = n_estimates;
  std::vector<double> poly(4 * lines);
  auto lerp = [](double a, double b, double t) { return a + (b - a) * t; };
  for (uint64_t l = 0; l < lines; ++l) {
    const double t = (double)l * azimuth_time_interval_s;
    double *q = poly.data() + 4 * l;
    const sd_dc_estimate *e = nullptr;
    if (t < et[0]) {
      if (et[0] - t > 2.0)
        return set_error(ctx, SD_ERR_INSAR_AZIMUTH_TIME_BEFORE_DC,
                         "azimuth time %.6f s (relative) is before the first DC estimate at %.6f s", t, et[0]);
      e = &estimates[0];
    } else if (t >= et[n - 1]) {
      e = &estimates[n - 1];
    }
    if (e) {
      q[0] = e->data_dc_poly[0], q[1] = e->data_dc_poly[1], q[2] = e->data_dc_poly[2], q[3] = e->t0_s;
      continue;
    }
    uint64_t k = n - 2;  // the first window holding t
    for (uint64_t j = 0; j + 1 < n; ++j)
      if (t >= et[j] && t < et[j + 1]) {
        k = j;
        break;
      }
    const double alpha = (t - et[k]) / (et[k + 1] - et[k]);
    const sd_dc_estimate &e0 = estimates[k], &e1 = estimates[k + 1];
    for (int j = 0; j < 3; ++j) q[j] = lerp(e0.data_dc_poly[j], e1.data_dc_poly[j], alpha);
    q[3] = lerp(e0.t0_s, e1.t0_s, alpha);
  }
  if (lines == 0 || samples == 0) return SD_OK;
  if (!iq || !out) return set_error(ctx, SD_ERR_INVALID_ARGUMENT, "null buffer");
  SD_CUDA(ctx, cudaSetDevice(ctx->device));
  cudaStream_t s = ctx->stream;
  const void *din;
  void *dout;
  double *dpoly;
  SD_TRY(stage_in(ctx, "dr.in", iq, lines * samples * 4, &din));
  SD_TRY(stage_out(ctx, "dr.out", out, lines * samples * 8, &dout));
  SD_TRY(scratch_t(ctx, "dr.poly", 4 * lines, &dpoly));
  SD_CUDA(ctx, cudaMemcpyAsync(dpoly, poly.data(), lines * 32, cudaMemcpyHostToDevice, s));
  const double dtau = 2.0 * range_pixel_spacing_m / kSpeedOfLight;
  const dim3 grid((unsigned)((samples + 255) / 256), (unsigned)(lines < 65535 ? lines : 65535));
  SD_TIMED_BEGIN(ctx, "k_deramp");
  k_deramp<<<grid, 256, 0, s>>>((const short2 *)din, (const double2 *)dpoly, lines, (uint32_t)samples,
                                slant_range_time_s, dtau, valid_sample_offset, azimuth_time_interval_s,
                                (float2 *)dout);
  SD_LAUNCHED(ctx);
  SD_TRY(finish_out(ctx, out, dout, lines * samples * 8));
  return sync(ctx);  // the host polynomial table lives until here
}
