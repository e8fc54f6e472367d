// Ground-range projection (to_ground_range, ground_range.rs:303-427).
//
// The host builds what depends on columns only, in the reference's f64
// arithmetic: the incidence-angle profile from each sub-swath's mid-azimuth
// grid row (build_incidence_profile / RangeInterpolator /
// interpolate_at_slant_time, 148-296), the cumulative ground range and the
// output-column mapping (build_ground_to_slant_mapping, 441-485).  One
// device kernel then does the per-pixel work fused: each output pixel
// projects its azimuth_looks input lines to ground range (the f32 linear
// interpolation of 363-382) and averages them (the f64 mean of 395-416),
// so the projected slant-to-ground image is never written.  HBM-bound: the
// input is read about once (2 taps per output column, shared by
// neighbours), the output written once.
#include <algorithm>
#include <cmath>
#include <vector>

#include "runtime.cuh"

namespace sd {
namespace {

struct Interp {  // RangeInterpolator (164-240)
  std::vector<double> t, a;
  double tmin, tmax;
  // interpolate (205-240): None outside [tmin, tmax]
  bool at(double st, double *out) const {
    if (st < tmin || st > tmax) return false;
    const size_t i = (size_t)(std::lower_bound(t.begin(), t.end(), st) - t.begin());
    if (i < t.size() && t[i] == st) {
      *out = a[i];
      return true;
    }
    if (i == 0) {
      *out = a[0];
      return true;
    }
    if (i >= t.size()) {
      *out = a.back();
      return true;
    }
    const double frac = (st - t[i - 1]) / (t[i] - t[i - 1]);
    *out = a[i - 1] + frac * (a[i] - a[i - 1]);
    return true;
  }
};

// interpolate_at_slant_time (246-289)
bool angle_at(const std::vector<Interp> &in, double st, double *deg) {
  bool have = false;
  double best_d = 0.0, best_a = 0.0;
  for (const Interp &p : in) {
    double a;
    if (!p.at(st, &a)) continue;
    const double d = std::fabs(st - (p.tmin + p.tmax) / 2.0);
    if (!have || d < best_d) {
      have = true;
      best_d = d;
      best_a = a;
    }
  }
  if (have) {
    *deg = best_a;
    return true;
  }
  const Interp *near = nullptr;
  double nd = 0.0;
  for (const Interp &p : in) {
    const double d = st < p.tmin ? p.tmin - st : st - p.tmax;
    if (!near || d < nd) {
      near = &p;
      nd = d;
    }
  }
  if (near && nd < (near->tmax - near->tmin) * 0.01) return near->at(std::min(std::max(st, near->tmin), near->tmax), deg);
  return false;
}

// One output pixel: the mean over its azimuth_looks lines of the projected
// value (left == right: the column itself; else the f32 interpolation).
__global__ void k_grd(const float *__restrict__ d, uint64_t in_s, const int32_t *__restrict__ left,
                      const int32_t *__restrict__ right, const float *__restrict__ frac, uint32_t al,
                      float *__restrict__ out, uint64_t out_l, uint64_t out_s) {
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= out_l * out_s) return;
  const uint64_t ol = i / out_s, j = i - ol * out_s;
  const int32_t l0 = __ldg(left + j), r0 = __ldg(right + j);
  const float f = __ldg(frac + j);
  double sum = 0.0;
  uint32_t cnt = 0;
  for (uint32_t k = 0; k < al; ++k) {
    const float *row = d + (ol * al + k) * in_s;
    float v = __ldg(row + l0);
    if (r0 != l0) {
      const float v1 = __ldg(row + r0);
      v = (v != v || v1 != v1) ? NAN : v + (v1 - v) * f;
    }
    if (v == v) {
      sum += (double)v;
      ++cnt;
    }
  }
  out[i] = cnt ? (float)(sum / (double)cnt) : NAN;
}

}  // namespace
}  // namespace sd

using namespace sd;

extern "C" int sd_to_ground_range(sd_ctx *ctx, const float *data, uint64_t lines, uint64_t samples,
                                  double near_slant_range_time_s, double range_pixel_spacing_s,
                                  double range_pixel_spacing_m, const sd_grd_swath_grid *grids, int32_t n_grids,
                                  double target_spacing_m, double azimuth_pixel_spacing_m, float *out,
                                  sd_grd_info *info) {
  SD_STAGE("ground_range_projection");
  if (!ctx || !info) return SD_ERR_INVALID_ARGUMENT;
  if (lines == 0 || samples == 0)
    return set_error(ctx, SD_ERR_GRD_EMPTY_IMAGE, "merged image is empty (%llu lines x %llu samples)",
                     (unsigned long long)lines, (unsigned long long)samples);
  if (!(target_spacing_m > 0.0))
    return set_error(ctx, SD_ERR_GRD_INVALID_SPACING, "target pixel spacing must be positive, got %g", target_spacing_m);
  if (!std::isfinite(azimuth_pixel_spacing_m) || azimuth_pixel_spacing_m <= 0.0)
    return set_error(ctx, SD_ERR_GRD_INVALID_AZIMUTH_SPACING,
                     "input azimuth pixel spacing must be positive and finite, got %g", azimuth_pixel_spacing_m);
  if (samples > 0x7FFFFFFFull) return set_error(ctx, SD_ERR_INVALID_ARGUMENT, "too many samples");
  // ── incidence profile (148-160) ──
  std::vector<Interp> in;
  for (int32_t g = 0; g < n_grids; ++g) {
    const sd_grd_swath_grid &sg = grids[g];
    if (sg.n_points == 0 || !sg.points)
      return set_error(ctx, SD_ERR_GRD_NO_GRID_POINTS, "no geolocation grid points for IW%d", sg.swath_id);
    std::vector<uint32_t> ls;
    for (uint64_t k = 0; k < sg.n_points; ++k) ls.push_back(sg.points[k].line);
    std::sort(ls.begin(), ls.end());
    ls.erase(std::unique(ls.begin(), ls.end()), ls.end());
    const uint32_t mid = ls[ls.size() / 2];
    std::vector<std::pair<double, double>> pts;
    for (uint64_t k = 0; k < sg.n_points; ++k)
      if (sg.points[k].line == mid) pts.push_back({sg.points[k].slant_range_time_s, sg.points[k].incidence_angle_deg});
    std::stable_sort(pts.begin(), pts.end(), [](const auto &x, const auto &y) { return x.first < y.first; });
    Interp p;
    for (auto &q : pts) {
      p.t.push_back(q.first);
      p.a.push_back(q.second);
    }
    p.tmin = p.t.front();
    p.tmax = p.t.back();
    in.push_back(std::move(p));
  }
  std::stable_sort(in.begin(), in.end(), [](const Interp &x, const Interp &y) { return x.tmin < y.tmin; });
  const double deg2rad = 3.14159265358979323846 / 180.0;
  std::vector<double> gs(samples);
  for (uint64_t c = 0; c < samples; ++c) {
    const double st = near_slant_range_time_s + (double)c * range_pixel_spacing_s;
    double deg;
    if (!angle_at(in, st, &deg))
      return set_error(ctx, SD_ERR_GRD_INTERPOLATION_FAILED,
                       "incidence angle interpolation failed at column %llu: slant time %.6e s outside all grid ranges",
                       (unsigned long long)c, st);
    gs[c] = range_pixel_spacing_m / std::sin(deg * deg2rad);  // 326-332
  }
  // ── cumulative ground range and output columns (334-350) ──
  std::vector<double> cum(samples);
  double acc = 0.0;
  cum[0] = 0.0;
  for (uint64_t c = 1; c < samples; ++c) {
    acc += (gs[c - 1] + gs[c]) / 2.0;
    cum[c] = acc;
  }
  const uint64_t out_s = (uint64_t)std::floor(cum.back() / target_spacing_m);
  if (out_s == 0)
    return set_error(ctx, SD_ERR_GRD_INVALID_SPACING, "target pixel spacing must be positive, got %g", target_spacing_m);
  const uint64_t al = (uint64_t)std::max(std::round(target_spacing_m / azimuth_pixel_spacing_m), 1.0);  // 388-389
  const uint64_t out_l = lines / al;
  info->lines = out_l;
  info->samples = out_s;
  info->range_pixel_spacing_m = target_spacing_m;
  info->azimuth_pixel_spacing_m = azimuth_pixel_spacing_m * (double)al;
  info->range_looks = 1;
  info->azimuth_looks = al;
  if (!out || out_l == 0) return SD_OK;
  if (!data) return set_error(ctx, SD_ERR_INVALID_ARGUMENT, "null data");
  if (al > 0xFFFFFFFFull) return set_error(ctx, SD_ERR_INVALID_ARGUMENT, "azimuth looks too large");
  // ── build_ground_to_slant_mapping (441-485): left == right for Exact ──
  std::vector<int32_t> L(out_s), R(out_s);
  std::vector<float> F(out_s, 0.0f);
  uint64_t start = 0;
  for (uint64_t j = 0; j < out_s; ++j) {
    const double tg = (double)j * target_spacing_m;
    const uint64_t idx = (uint64_t)(std::lower_bound(cum.begin() + (ptrdiff_t)start, cum.end(), tg) - cum.begin());
    if (idx < samples && cum[idx] == tg) {
      L[j] = R[j] = (int32_t)idx;
      start = idx;
      continue;
    }
    if (idx == 0) {
      L[j] = R[j] = 0;
    } else if (idx >= samples) {
      L[j] = R[j] = (int32_t)(samples - 1);
    } else {
      L[j] = (int32_t)(idx - 1);
      R[j] = (int32_t)idx;
      F[j] = (float)((tg - cum[idx - 1]) / (cum[idx] - cum[idx - 1]));  // `frac as f32` at use (376)
      start = idx - 1;
    }
  }
  SD_CUDA(ctx, cudaSetDevice(ctx->device));
  cudaStream_t s = ctx->stream;
  const void *din;
  void *dout;
  int32_t *dL, *dR;
  float *dF;
  SD_TRY(stage_in(ctx, "grd.in", data, lines * samples * 4, &din));
  SD_TRY(stage_out(ctx, "grd.out", out, out_l * out_s * 4, &dout));
  SD_TRY(scratch_t(ctx, "grd.left", out_s, &dL));
  SD_TRY(scratch_t(ctx, "grd.right", out_s, &dR));
  SD_TRY(scratch_t(ctx, "grd.frac", out_s, &dF));
  SD_CUDA(ctx, cudaMemcpyAsync(dL, L.data(), out_s * 4, cudaMemcpyHostToDevice, s));
  SD_CUDA(ctx, cudaMemcpyAsync(dR, R.data(), out_s * 4, cudaMemcpyHostToDevice, s));
  SD_CUDA(ctx, cudaMemcpyAsync(dF, F.data(), out_s * 4, cudaMemcpyHostToDevice, s));
  SD_TIMED_BEGIN(ctx, "k_grd");
  k_grd<<<(unsigned)((out_l * out_s + 255) / 256), 256, 0, s>>>((const float *)din, samples, dL, dR, dF,
                                                                 (uint32_t)al, (float *)dout, out_l, out_s);
  SD_LAUNCHED(ctx);
  SD_TRY(finish_out(ctx, out, dout, out_l * out_s * 4));
  return sync(ctx);  // the host mapping vectors live until here
}
