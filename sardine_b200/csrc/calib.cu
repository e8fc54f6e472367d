// calib.cu — TOPS deburst, sigma0 calibration with NESZ, IW merge, and the
// fused calibrate+deburst+merge pass, on sm_100a.
//
// Replaces deburst_subswath / compute_overlap_lines (sardine/src/deburst.rs:
// 172-344), apply_calibration (apply_calibration.rs:374-572) and
// merge_subswaths (merge_subswaths.rs:207-450).
//
// Calibration LUTs are evaluated per (LUT vector, output column) once into
// small tables (a few MB, L2-resident); a pixel then costs two table reads
// per LUT, one f32 lerp in azimuth, and the reference's branchless f32
// formula.  The fused pass reads each contributing CInt16 sample once
// (4 B) and writes merged sigma0 and NESZ (8 B): overlap lines and
// out-of-window samples are never read.
#include <algorithm>
#include <cmath>
#include <mutex>
#include <vector>

#include "geo.cuh"
#include "runtime.cuh"

namespace sd {
namespace {

__host__ __device__ __forceinline__ float lerpf(float a, float b, float t) {
  t = t < 0.0f ? 0.0f : (t > 1.0f ? 1.0f : t);  // f32::clamp (NaN passes through)
  return a + (b - a) * t;
}

// bracket_azimuth (apply_calibration.rs:190-202)
void bracket(const std::vector<int64_t> &lines, int64_t tl, int32_t *lo, int32_t *hi) {
  size_t a = 0, b = lines.size();
  while (a < b) {
    size_t mid = a + (b - a) / 2;
    if (lines[mid] < tl) a = mid + 1;
    else if (lines[mid] > tl) b = mid;
    else {
      *lo = *hi = (int32_t)mid;
      return;
    }
  }
  if (a == 0) {
    *lo = *hi = 0;
    return;
  }
  if (a >= lines.size()) {
    *lo = *hi = (int32_t)lines.size() - 1;
    return;
  }
  *lo = (int32_t)a - 1;
  *hi = (int32_t)a;
}

// One LUT family (sigma0 K or range noise N) flattened for the device.
struct LutHost {
  std::vector<int64_t> lines;
  std::vector<uint32_t> px, pm;  // pixels and their running max (cursor semantics)
  std::vector<float> val;
  std::vector<uint64_t> off, cnt;
};

LutHost flatten(const sd_lut_vector *v, uint64_t n) {
  LutHost L;
  for (uint64_t i = 0; i < n; ++i) {
    L.lines.push_back(v[i].line);
    L.off.push_back(L.px.size());
    L.cnt.push_back(v[i].n);
    uint32_t m = 0;
    for (uint64_t k = 0; k < v[i].n; ++k) {
      L.px.push_back(v[i].pixels[k]);
      if (k >= 1) m = std::max(m, v[i].pixels[k]);
      L.pm.push_back(m);
      L.val.push_back(v[i].values[k]);
    }
  }
  return L;
}

struct LutDev {
  const uint32_t *px, *pm;
  const float *val;
  const uint64_t *off, *cnt;
};

// tab[v][c] = lut_cursor_eval(vector v, col_offset + c) (apply_calibration.rs:212-225,
// 311-354).  The reference's monotone cursor equals the count of i >= 1 whose
// running max pixels[1..=i] is <= col.
__global__ void k_lut_table(LutDev L, uint64_t n_vec, uint64_t tab_cols, uint64_t col_offset, float *tab) {
  uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n_vec * tab_cols) return;
  uint64_t v = i / tab_cols, c = i % tab_cols;
  const uint32_t col = (uint32_t)(c + col_offset);
  const uint32_t *px = L.px + L.off[v];
  const uint32_t *pm = L.pm + L.off[v];
  const float *val = L.val + L.off[v];
  const uint64_t n = L.cnt[v];
  uint64_t lo = 1, hi = n;  // upper_bound over pm[1..n)
  while (lo < hi) {
    uint64_t mid = (lo + hi) / 2;
    if (pm[mid] <= col) lo = mid + 1; else hi = mid;
  }
  uint64_t cur = lo - 1;
  float out;
  if (px[cur] > col) out = val[0];
  else if (cur + 1 < n) {
    float t = (float)(col - px[cur]) / (float)(px[cur + 1] - px[cur]);
    out = lerpf(val[cur], val[cur + 1], t);
  } else out = val[cur];
  tab[i] = out;
}

struct LineParams {  // per output line, per LUT family
  int32_t lo, hi;
  float t;
};

struct CalSwathDev {
  const int16_t *iq;          // raster base
  uint64_t stride;            // raster width in IQ pairs
  const uint64_t *line_map;   // output line -> raster row
  uint64_t col0;              // raster column of calibrated column 0
  const float *cal_tab, *nr_tab;
  uint64_t tab_cols;
  const LineParams *cal_lp, *nr_lp;
  const float *az;
};

__device__ __forceinline__ void calibrate_px(const CalSwathDev &s, uint64_t l, uint64_t c, float *sig,
                                             float *nesz) {
  const uint64_t row = s.line_map[l];
  const uint32_t iqw = __ldg((const uint32_t *)(s.iq) + row * s.stride + s.col0 + c);
  const int32_t i = (int32_t)(int16_t)(iqw & 0xFFFF), q = (int32_t)(int16_t)(iqw >> 16);
  const float power = (float)(int32_t)((uint32_t)(i * i) + (uint32_t)(q * q));
  const LineParams cl = s.cal_lp[l], nl = s.nr_lp[l];
  float k = __ldg(s.cal_tab + (uint64_t)cl.lo * s.tab_cols + c);
  if (cl.lo != cl.hi) k = lerpf(k, __ldg(s.cal_tab + (uint64_t)cl.hi * s.tab_cols + c), cl.t);
  float nr = __ldg(s.nr_tab + (uint64_t)nl.lo * s.tab_cols + c);
  if (nl.lo != nl.hi) nr = lerpf(nr, __ldg(s.nr_tab + (uint64_t)nl.hi * s.tab_cols + c), nl.t);
  // apply_cal_row (apply_calibration.rs:288-309)
  const float k2 = k * k;
  const float valid = (k2 > 0.0f) ? 1.0f : 0.0f;
  const float inv_k2 = (k2 > 0.0f) ? 1.0f / k2 : 0.0f;
  const float noise_val = nr * s.az[l];
  *sig = maxf_nan(power - noise_val, 0.0f) * inv_k2 * valid;
  *nesz = noise_val * inv_k2 * valid;
}

__global__ void k_calibrate(CalSwathDev s, uint64_t lines, uint64_t samples, float *out, float *nesz) {
  uint64_t c = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  uint64_t l = blockIdx.y;
  if (c >= samples || l >= lines) return;
  float a, b;
  calibrate_px(s, l, c, &a, &b);
  out[l * samples + c] = a;
  nesz[l * samples + c] = b;
}

struct FillRange {  // merge_subswaths.rs:326-352
  uint64_t col_end, vs, ve, in_start;
};

struct MergeDev {
  int n;
  FillRange fr[8];
  CalSwathDev sw[8];
  const float *sig[8];
  const float *nz[8];
  uint64_t in_samples[8];
};

// Fused: merged pixel (l, c) <- owning swath's calibrated raster sample.
// One block per (line, 2048-column chunk): the line's per-swath raster row,
// LUT brackets and azimuth-noise factor are read once into shared memory;
// each thread then handles 8 columns 256 apart (coalesced), in 32-bit
// column arithmetic.
constexpr int FU_THREADS = 256, FU_PER_THREAD = 8, FU_COLS = FU_THREADS * FU_PER_THREAD;

struct FuLine {
  const uint32_t *row;
  float az;
  LineParams cal, nr;
  uint32_t col_end, vs, ve, in_start;
};

__global__ void __launch_bounds__(FU_THREADS) k_fused(MergeDev m, uint64_t lines, uint64_t cols, float *out,
                                                     float *nesz) {
  __shared__ FuLine sl[8];
  const uint64_t chunks = (cols + FU_COLS - 1) / FU_COLS;
  const uint64_t l = blockIdx.x / chunks;
  const uint32_t c0 = (uint32_t)((blockIdx.x % chunks) * FU_COLS);
  if (l >= lines) return;
  if (threadIdx.x < (unsigned)m.n) {
    const int k = threadIdx.x;
    const CalSwathDev &s = m.sw[k];
    FuLine f;
    f.row = (const uint32_t *)s.iq + s.line_map[l] * s.stride + s.col0;
    f.az = s.az[l];
    f.cal = s.cal_lp[l];
    f.nr = s.nr_lp[l];
    f.col_end = (uint32_t)m.fr[k].col_end;
    f.vs = (uint32_t)m.fr[k].vs;
    f.ve = (uint32_t)m.fr[k].ve;
    f.in_start = (uint32_t)m.fr[k].in_start;
    sl[k] = f;
  }
  __syncthreads();
  float *orow = out + l * cols;
  float *nrow = nesz + l * cols;
#pragma unroll
  for (int j = 0; j < FU_PER_THREAD; ++j) {
    const uint32_t c = c0 + (uint32_t)(j * FU_THREADS) + threadIdx.x;
    if (c >= cols) break;
    float a = NAN, b = NAN;
    for (int k = 0; k < m.n; ++k) {
      const FuLine &f = sl[k];
      if (c < f.col_end) {
        if (c >= f.vs && c < f.ve) {
          const uint32_t cc = f.in_start + (c - f.vs);
          const CalSwathDev &s = m.sw[k];
          const uint32_t iqw = __ldg(f.row + cc);
          const int32_t i = (int32_t)(int16_t)(iqw & 0xFFFF), q = (int32_t)(int16_t)(iqw >> 16);
          const float power = (float)(int32_t)((uint32_t)(i * i) + (uint32_t)(q * q));
          float kk = __ldg(s.cal_tab + (uint64_t)f.cal.lo * s.tab_cols + cc);
          if (f.cal.lo != f.cal.hi) kk = lerpf(kk, __ldg(s.cal_tab + (uint64_t)f.cal.hi * s.tab_cols + cc), f.cal.t);
          float nr = __ldg(s.nr_tab + (uint64_t)f.nr.lo * s.tab_cols + cc);
          if (f.nr.lo != f.nr.hi) nr = lerpf(nr, __ldg(s.nr_tab + (uint64_t)f.nr.hi * s.tab_cols + cc), f.nr.t);
          // apply_cal_row (apply_calibration.rs:288-309)
          const float k2 = kk * kk;
          const float valid = (k2 > 0.0f) ? 1.0f : 0.0f;
          const float inv_k2 = (k2 > 0.0f) ? 1.0f / k2 : 0.0f;
          const float noise_val = nr * f.az;
          a = maxf_nan(power - noise_val, 0.0f) * inv_k2 * valid;
          b = noise_val * inv_k2 * valid;
        }
        break;
      }
    }
    orow[c] = a;
    nrow[c] = b;
  }
}

// Plain merge of calibrated swaths.
__global__ void k_merge(MergeDev m, uint64_t lines, uint64_t cols, float *out, float *nesz) {
  uint64_t c = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  uint64_t l = blockIdx.y;
  if (c >= cols || l >= lines) return;
  float a = NAN, b = NAN;
  for (int k = 0; k < m.n; ++k) {
    if (c < m.fr[k].col_end) {
      if (c >= m.fr[k].vs && c < m.fr[k].ve) {
        uint64_t src = l * m.in_samples[k] + m.fr[k].in_start + (c - m.fr[k].vs);
        a = __ldg(m.sig[k] + src);
        b = __ldg(m.nz[k] + src);
      }
      break;
    }
  }
  out[l * cols + c] = a;
  nesz[l * cols + c] = b;
}

__global__ void k_deburst_copy(const uint32_t *raw, uint64_t stride, const uint64_t *line_map, uint64_t col0,
                               uint64_t lines, uint64_t samples, uint32_t *out) {
  uint64_t c = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  uint64_t l = blockIdx.y;
  if (c >= samples || l >= lines) return;
  out[l * samples + c] = __ldg(raw + line_map[l] * stride + col0 + c);
}

}  // namespace

// ── host planning (shared by the entry points) ─────────────────────────────
int overlap_lines(sd_ctx *ctx, const sd_burst *bk, const sd_burst *bk1, double ati, uint64_t lps,
                  int64_t *ov) {
  int64_t dt_us = bk1->azimuth_time_us - bk->azimuth_time_us;
  double dt_s = (double)dt_us * 1e-6;
  int64_t step = f2i64(std::round(dt_s / ati));
  *ov = (int64_t)lps - step;
  if (*ov <= 0)
    return set_error(ctx, SD_ERR_DEBURST_INVALID_OVERLAP,
                     "non-positive overlap between burst %llu and burst %llu: computed overlap = %lld lines",
                     (unsigned long long)bk->burst_index, (unsigned long long)bk1->burst_index, (long long)*ov);
  if (*ov < 50 || *ov > 400)
    return set_error(ctx, SD_ERR_DEBURST_IMPLAUSIBLE_OVERLAP,
                     "implausible overlap between burst %llu and burst %llu: %lld lines is outside [50, 400]",
                     (unsigned long long)bk->burst_index, (unsigned long long)bk1->burst_index, (long long)*ov);
  return SD_OK;
}

struct DeburstPlan {
  uint64_t lines = 0, samples = 0, offset = 0;
  std::vector<uint64_t> line_map;  // out line -> tiff row
};

int deburst_plan(sd_ctx *ctx, const sd_subswath *sw, const sd_burst *b, uint64_t n, uint64_t tiff_height,
                 DeburstPlan *plan) {
  if (n == 0) return set_error(ctx, SD_ERR_DEBURST_NO_BURSTS, "burst list is empty");
  if (n != sw->burst_count)
    return set_error(ctx, SD_ERR_DEBURST_BURST_COUNT_MISMATCH, "subswath declares %llu bursts but %llu were given",
                     (unsigned long long)sw->burst_count, (unsigned long long)n);
  const uint64_t lps = sw->lines_per_burst;
  if (tiff_height < n * lps)
    return set_error(ctx, SD_ERR_DEBURST_TIFF_TOO_SMALL, "TIFF height %llu is too small for %llu bursts × %llu lines",
                     (unsigned long long)tiff_height, (unsigned long long)n, (unsigned long long)lps);
  uint64_t fv = 0, lv = UINT64_MAX;
  for (uint64_t i = 0; i < n; ++i) {
    fv = std::max<uint64_t>(fv, b[i].first_valid_sample);
    lv = std::min<uint64_t>(lv, b[i].last_valid_sample);
  }
  if (fv >= lv)
    return set_error(ctx, SD_ERR_DEBURST_EMPTY_VALID_WINDOW,
                     "no valid range window after intersecting all burst valid-sample extents: first_valid=%llu, last_valid=%llu",
                     (unsigned long long)fv, (unsigned long long)lv);
  std::vector<uint64_t> ovs;
  for (uint64_t k = 0; k + 1 < n; ++k) {
    int64_t ov;
    SD_TRY(overlap_lines(ctx, &b[k], &b[k + 1], sw->azimuth_time_interval_s, lps, &ov));
    ovs.push_back((uint64_t)ov);
  }
  plan->line_map.clear();
  for (uint64_t k = 0; k < n; ++k) {
    uint64_t lf = k == 0 ? 0 : (ovs[k - 1] + 1) / 2;
    uint64_t le = k == n - 1 ? lps : lps - ovs[k] / 2;
    for (uint64_t l = lf; l < le; ++l) plan->line_map.push_back(b[k].first_line + l);
  }
  plan->lines = plan->line_map.size();
  plan->samples = lv - fv;
  plan->offset = fv;
  return SD_OK;
}

// Calibration planning: LUT checks (apply_calibration.rs:380-462) and per-line
// azimuth brackets for `lines` output lines starting at tiff_line_origin.
struct CalPlan {
  LutHost cal, nr;
  std::vector<LineParams> cal_lp, nr_lp;
  std::vector<float> az;
  uint32_t cal_gap = 0, nr_gap = 0;
};

int cal_plan(sd_ctx *ctx, const sd_lut_vector *cal, uint64_t n_cal, const sd_lut_vector *nr, uint64_t n_nr,
             const sd_noise_azimuth *az, uint64_t col_offset, uint64_t samples, uint64_t tiff_line_origin,
             uint64_t lines, CalPlan *P) {
  if ((n_cal && !cal) || (n_nr && !nr))
    return set_error(ctx, SD_ERR_INVALID_ARGUMENT, "null LUT vector array with a non-zero count");
  for (uint64_t i = 0; i < n_cal + n_nr; ++i) {
    const sd_lut_vector &v = i < n_cal ? cal[i] : nr[i - n_cal];
    if (v.n && (!v.pixels || !v.values))
      return set_error(ctx, SD_ERR_INVALID_ARGUMENT, "LUT vector at line %d has %llu knots but a null array",
                       v.line, (unsigned long long)v.n);
  }
  if (az && az->n && (!az->lines || !az->values))
    return set_error(ctx, SD_ERR_INVALID_ARGUMENT, "azimuth noise vector has %llu knots but a null array",
                     (unsigned long long)az->n);
  if (n_cal == 0) return set_error(ctx, SD_ERR_CAL_NO_CALIBRATION_VECTORS, "calibration LUT has no vectors");
  if (n_nr == 0) return set_error(ctx, SD_ERR_CAL_NO_NOISE_RANGE_VECTORS, "noise range LUT has no vectors");
  const uint32_t SLACK = 600;
  uint64_t req = col_offset + samples;
  const uint32_t required_last = (uint32_t)(req == 0 ? 0 : req - 1);
  P->cal_gap = P->nr_gap = 0;
  for (int fam = 0; fam < 2; ++fam) {
    const sd_lut_vector *v = fam == 0 ? cal : nr;
    uint64_t n = fam == 0 ? n_cal : n_nr;
    uint32_t &gapmax = fam == 0 ? P->cal_gap : P->nr_gap;
    for (uint64_t i = 0; i < n; ++i) {
      if (v[i].n == 0)
        return set_error(ctx, fam == 0 ? SD_ERR_CAL_NO_CALIBRATION_VECTORS : SD_ERR_CAL_NO_NOISE_RANGE_VECTORS,
                         fam == 0 ? "calibration LUT has no vectors" : "noise range LUT has no vectors");
      uint32_t m = v[i].pixels[v[i].n - 1];
      if (m < required_last) {
        uint32_t gap = required_last - m;
        if (gap > SLACK)
          return set_error(ctx, SD_ERR_CAL_LUT_RANGE_INSUFFICIENT,
                           "calibration vector at line %d covers pixels up to %u, but output requires up to pixel %u",
                           v[i].line, m, required_last);
        gapmax = std::max(gapmax, gap);
      }
    }
  }
  P->cal = flatten(cal, n_cal);
  P->nr = flatten(nr, n_nr);
  P->cal_lp.resize(lines);
  P->nr_lp.resize(lines);
  P->az.resize(lines);
  std::vector<int64_t> az_lines;
  const bool az_avail = az && az->n > 0;
  if (az_avail)
    for (uint64_t i = 0; i < az->n; ++i) az_lines.push_back(az->lines[i]);
  for (uint64_t l = 0; l < lines; ++l) {
    const int64_t tl = (int64_t)(tiff_line_origin + l);
    for (int fam = 0; fam < 2; ++fam) {
      const std::vector<int64_t> &ln = fam == 0 ? P->cal.lines : P->nr.lines;
      LineParams lp;
      bracket(ln, tl, &lp.lo, &lp.hi);
      lp.t = lp.lo == lp.hi ? 0.0f : (float)(tl - ln[lp.lo]) / (float)(ln[lp.hi] - ln[lp.lo]);
      (fam == 0 ? P->cal_lp : P->nr_lp)[l] = lp;
    }
    float f = 1.0f;
    if (az_avail) {
      int32_t lo, hi;
      bracket(az_lines, tl, &lo, &hi);
      if (az_lines[hi] == az_lines[lo]) f = az->values[lo];
      else {
        float t = (float)(tl - az_lines[lo]) / (float)(az_lines[hi] - az_lines[lo]);
        f = lerpf(az->values[lo], az->values[hi], t);
      }
    }
    P->az[l] = f;
  }
  return SD_OK;
}

template <class T>
static int upload(sd_ctx *ctx, const std::string &name, const std::vector<T> &v, T **d) {
  SD_TRY(scratch_t(ctx, name.c_str(), std::max<size_t>(v.size(), 1), d));
  if (!v.empty()) SD_CUDA(ctx, cudaMemcpyAsync(*d, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, ctx->stream));
  return SD_OK;
}

// Upload a CalPlan and build its LUT tables for `samples` columns.
int cal_device(sd_ctx *ctx, const std::string &tag, const CalPlan &P, uint64_t col_offset, uint64_t samples,
               CalSwathDev *s) {
  for (int fam = 0; fam < 2; ++fam) {
    const LutHost &L = fam == 0 ? P.cal : P.nr;
    std::string t = tag + (fam == 0 ? ".cal" : ".nr");
    LutDev d;
    uint32_t *px, *pm;
    float *val;
    uint64_t *off, *cnt;
    SD_TRY(upload(ctx, t + ".px", L.px, &px));
    SD_TRY(upload(ctx, t + ".pm", L.pm, &pm));
    SD_TRY(upload(ctx, t + ".val", L.val, &val));
    SD_TRY(upload(ctx, t + ".off", L.off, &off));
    SD_TRY(upload(ctx, t + ".cnt", L.cnt, &cnt));
    d.px = px;
    d.pm = pm;
    d.val = val;
    d.off = off;
    d.cnt = cnt;
    float *tab;
    uint64_t nv = L.lines.size();
    SD_TRY(scratch_t(ctx, (t + ".tab").c_str(), nv * std::max<uint64_t>(samples, 1), &tab));
    if (samples > 0) {
      SD_TIMED_BEGIN(ctx, "k_lut_table");
      k_lut_table<<<grid_for(nv * samples, 256), 256, 0, ctx->stream>>>(d, nv, samples, col_offset, tab);
      SD_LAUNCHED(ctx);
    }
    (fam == 0 ? s->cal_tab : s->nr_tab) = tab;
  }
  s->tab_cols = samples;
  LineParams *clp, *nlp;
  float *az;
  SD_TRY(upload(ctx, tag + ".cal_lp", P.cal_lp, &clp));
  SD_TRY(upload(ctx, tag + ".nr_lp", P.nr_lp, &nlp));
  SD_TRY(upload(ctx, tag + ".az", P.az, &az));
  s->cal_lp = clp;
  s->nr_lp = nlp;
  s->az = az;
  return SD_OK;
}

// merge_subswaths geometry (merge_subswaths.rs:207-352)
int merge_plan(sd_ctx *ctx, int n, const uint64_t *lines, const uint64_t *samples, const uint64_t *voff,
               const sd_subswath *sw, const int64_t *az_start, sd_merged_info *info, FillRange *fr) {
  std::memset(info, 0, sizeof(*info));
  if (n <= 0) return set_error(ctx, SD_ERR_MERGE_EMPTY_INPUTS, "at least 1 subswath input is required, got 0");
  if (n > 8) return set_error(ctx, SD_ERR_INVALID_ARGUMENT, "at most 8 sub-swaths are supported");
  info->n_swaths = n;
  if (n == 1) {
    if (samples[0] == 0) return set_error(ctx, SD_ERR_MERGE_EMPTY_SWATH, "subswath 0 has zero range samples");
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
    fr[0] = {samples[0], 0, samples[0], 0};
    return SD_OK;
  }
  const double rps = sw[0].range_pixel_spacing_m;
  for (int i = 1; i < n; ++i)
    if (std::fabs(sw[i].range_pixel_spacing_m - rps) > 1e-3)
      return set_error(ctx, SD_ERR_MERGE_INCONSISTENT_PIXEL_SPACING,
                       "range pixel spacing inconsistency: swath 0 = %e m, swath %d = %e m", rps, i,
                       sw[i].range_pixel_spacing_m);
  for (int i = 0; i < n; ++i)
    if (samples[i] == 0) return set_error(ctx, SD_ERR_MERGE_EMPTY_SWATH, "subswath %d has zero range samples", i);
  const double dt = rps * 2.0 / SPEED_OF_LIGHT;
  double st[8];
  int64_t offs[8], ends[8];
  for (int i = 0; i < n; ++i) st[i] = sw[i].slant_range_time_s + (double)voff[i] * dt;
  for (int i = 0; i < n; ++i) {
    offs[i] = f2i64(std::round((st[i] - st[0]) / dt));
    ends[i] = offs[i] + (int64_t)samples[i];
  }
  const uint64_t out_cols = (uint64_t)ends[n - 1];
  uint64_t out_lines = UINT64_MAX;
  int64_t azmin = az_start[0];
  for (int i = 0; i < n; ++i) {
    out_lines = std::min(out_lines, lines[i]);
    azmin = std::min(azmin, az_start[i]);
  }
  info->lines = out_lines;
  info->samples = out_cols;
  info->near_slant_range_time_s = st[0];
  info->range_pixel_spacing_s = dt;
  info->range_pixel_spacing_m = rps;
  info->azimuth_start_time_us = azmin;
  for (int i = 0; i < n; ++i) {
    info->swath_out_offset[i] = offs[i];
    info->swath_lines[i] = lines[i];
    info->swath_valid_offset[i] = voff[i];
    info->swath_seam[i] = (i + 1 < n) ? (uint64_t)((ends[i] + offs[i + 1]) / 2) : out_cols;
  }
  for (int i = 0; i < n; ++i) {
    uint64_t cs = i == 0 ? 0 : info->swath_seam[i - 1];
    uint64_t ce = i == n - 1 ? out_cols : info->swath_seam[i];
    uint64_t off = (uint64_t)offs[i];
    uint64_t vs = std::max(cs, off);
    uint64_t ve = std::min(ce, off + samples[i]);
    fr[i] = {ce, vs, ve, vs >= off ? vs - off : 0};
  }
  return SD_OK;
}

}  // namespace sd

using namespace sd;

extern "C" int sd_compute_overlap_lines(sd_ctx *ctx, const sd_burst *bk, const sd_burst *bk1, double ati,
                                        uint64_t lps, uint64_t *overlap) {
  if (!bk || !bk1 || !overlap) return SD_ERR_INVALID_ARGUMENT;
  int64_t ov = 0;
  int rc = overlap_lines(ctx, bk, bk1, ati, lps, &ov);
  *overlap = ov > 0 ? (uint64_t)ov : 0;
  return rc;
}

extern "C" int sd_deburst_plan(sd_ctx *ctx, const sd_subswath *sw, const sd_burst *bursts, uint64_t n,
                               uint64_t tiff_height, uint64_t *lines, uint64_t *samples, uint64_t *off) {
  if (!sw || (!bursts && n) || !lines || !samples || !off) return SD_ERR_INVALID_ARGUMENT;
  DeburstPlan p;
  SD_TRY(deburst_plan(ctx, sw, bursts, n, tiff_height, &p));
  *lines = p.lines;
  *samples = p.samples;
  *off = p.offset;
  return SD_OK;
}

extern "C" int sd_deburst_subswath(sd_ctx *ctx, const int16_t *slc, uint64_t tiff_width, uint64_t tiff_height,
                                   const sd_subswath *sw, const sd_burst *bursts, uint64_t n, int16_t *out) {
  SD_STAGE("deburst");
  if (!ctx || !sw || !slc || !out) return SD_ERR_INVALID_ARGUMENT;
  SD_CUDA(ctx, cudaSetDevice(ctx->device));
  DeburstPlan p;
  SD_TRY(deburst_plan(ctx, sw, bursts, n, tiff_height, &p));
  if (p.offset + p.samples > tiff_width)
    return set_error(ctx, SD_ERR_INVALID_ARGUMENT, "valid window exceeds raster width");
  const void *d_raw;
  void *d_out;
  uint64_t *d_map;
  SD_TRY(stage_in(ctx, "db.raw", slc, tiff_width * tiff_height * 4, &d_raw));
  SD_TRY(stage_out(ctx, "db.out", out, p.lines * p.samples * 4, &d_out));
  SD_TRY(upload(ctx, "db.map", p.line_map, &d_map));
  dim3 grid(grid_for(p.samples, 256), (unsigned)p.lines);
  SD_TIMED_BEGIN(ctx, "k_deburst_copy");
  k_deburst_copy<<<grid, 256, 0, ctx->stream>>>((const uint32_t *)d_raw, tiff_width, d_map, p.offset, p.lines,
                                                 p.samples, (uint32_t *)d_out);
  SD_LAUNCHED(ctx);
  SD_TRY(finish_out(ctx, out, d_out, p.lines * p.samples * 4));
  return sync(ctx);
}

extern "C" int sd_apply_calibration(sd_ctx *ctx, const int16_t *iq, uint64_t lines, uint64_t samples,
                                    uint64_t col_offset, const sd_lut_vector *cal, uint64_t n_cal,
                                    const sd_lut_vector *nr, uint64_t n_nr, const sd_noise_azimuth *az,
                                    uint64_t tiff_line_origin, float *out, float *nesz, uint32_t *cal_gap,
                                    uint32_t *nr_gap) {
  SD_STAGE("calibration");
  if (!ctx) return SD_ERR_INVALID_ARGUMENT;
  SD_CUDA(ctx, cudaSetDevice(ctx->device));
  CalPlan P;
  SD_TRY(cal_plan(ctx, cal, n_cal, nr, n_nr, az, col_offset, samples, tiff_line_origin, lines, &P));
  if (cal_gap) *cal_gap = P.cal_gap;
  if (nr_gap) *nr_gap = P.nr_gap;
  if (lines == 0 || samples == 0) return SD_OK;
  if (!iq || !out || !nesz) return set_error(ctx, SD_ERR_INVALID_ARGUMENT, "null buffer");
  CalSwathDev s{};
  SD_TRY(cal_device(ctx, "cal", P, col_offset, samples, &s));
  const void *d_iq;
  void *d_out, *d_nesz;
  SD_TRY(stage_in(ctx, "cal.iq", iq, lines * samples * 4, &d_iq));
  SD_TRY(stage_out(ctx, "cal.out", out, lines * samples * 4, &d_out));
  SD_TRY(stage_out(ctx, "cal.nesz", nesz, lines * samples * 4, &d_nesz));
  std::vector<uint64_t> ident(lines);
  for (uint64_t l = 0; l < lines; ++l) ident[l] = l;
  uint64_t *d_map;
  SD_TRY(upload(ctx, "cal.map", ident, &d_map));
  s.iq = (const int16_t *)d_iq;
  s.stride = samples;
  s.line_map = d_map;
  s.col0 = 0;
  dim3 grid(grid_for(samples, 256), (unsigned)lines);
  SD_TIMED_BEGIN(ctx, "k_calibrate");
  k_calibrate<<<grid, 256, 0, ctx->stream>>>(s, lines, samples, (float *)d_out, (float *)d_nesz);
  SD_LAUNCHED(ctx);
  SD_TRY(finish_out(ctx, out, d_out, lines * samples * 4));
  SD_TRY(finish_out(ctx, nesz, d_nesz, lines * samples * 4));
  return sync(ctx);
}

extern "C" int sd_merge_subswaths(sd_ctx *ctx, int32_t n, const float *const *sig, const float *const *nz,
                                  const uint64_t *lines, const uint64_t *samples, const uint64_t *voff,
                                  const uint32_t *cal_gap, const uint32_t *nr_gap, const sd_subswath *sw,
                                  const int64_t *az_start, float *out, float *out_nesz, sd_merged_info *info) {
  SD_STAGE("merge_subswaths");
  if (!ctx || !info) return SD_ERR_INVALID_ARGUMENT;
  FillRange fr[8];
  SD_TRY(merge_plan(ctx, n, lines, samples, voff, sw, az_start, info, fr));
  uint32_t cg = 0, ng = 0;
  for (int i = 0; i < n; ++i) {
    cg = std::max(cg, cal_gap ? cal_gap[i] : 0u);
    ng = std::max(ng, nr_gap ? nr_gap[i] : 0u);
  }
  info->cal_lut_extrapolation_gap_px = cg;
  info->noise_lut_extrapolation_gap_px = ng;
  if (!out) return SD_OK;
  if (!out_nesz) return set_error(ctx, SD_ERR_INVALID_ARGUMENT, "null nesz buffer");
  SD_CUDA(ctx, cudaSetDevice(ctx->device));
  MergeDev m{};
  m.n = n;
  for (int i = 0; i < n; ++i) {
    const void *ds, *dn;
    char nm[32];
    snprintf(nm, sizeof nm, "mg.sig%d", i);
    SD_TRY(stage_in(ctx, nm, sig[i], lines[i] * samples[i] * 4, &ds));
    snprintf(nm, sizeof nm, "mg.nz%d", i);
    SD_TRY(stage_in(ctx, nm, nz[i], lines[i] * samples[i] * 4, &dn));
    m.sig[i] = (const float *)ds;
    m.nz[i] = (const float *)dn;
    m.in_samples[i] = samples[i];
    m.fr[i] = fr[i];
  }
  const uint64_t L = info->lines, Cc = info->samples;
  void *d_out, *d_nesz;
  SD_TRY(stage_out(ctx, "mg.out", out, L * Cc * 4, &d_out));
  SD_TRY(stage_out(ctx, "mg.nesz", out_nesz, L * Cc * 4, &d_nesz));
  if (L > 0 && Cc > 0) {
    dim3 grid(grid_for(Cc, 256), (unsigned)L);
    SD_TIMED_BEGIN(ctx, "k_merge");
    k_merge<<<grid, 256, 0, ctx->stream>>>(m, L, Cc, (float *)d_out, (float *)d_nesz);
    SD_LAUNCHED(ctx);
  }
  SD_TRY(finish_out(ctx, out, d_out, L * Cc * 4));
  SD_TRY(finish_out(ctx, out_nesz, d_nesz, L * Cc * 4));
  return sync(ctx);
}

extern "C" int sd_calibrate_deburst_merge(sd_ctx *ctx, int32_t n, const sd_swath_input *sw, float *out,
                                          float *out_nesz, sd_merged_info *info) {
  SD_STAGE("cal_deburst_merge");
  if (!ctx || !sw || !info) return SD_ERR_INVALID_ARGUMENT;
  if (n <= 0) return set_error(ctx, SD_ERR_MERGE_EMPTY_INPUTS, "at least 1 subswath input is required, got 0");
  if (n > 8) return set_error(ctx, SD_ERR_INVALID_ARGUMENT, "at most 8 sub-swaths are supported");
  // per swath: deburst plan, then calibration plan (scene_prep.rs:635-658)
  DeburstPlan dp[8];
  CalPlan cp[8];
  uint64_t lines[8], samples[8], voff[8];
  uint32_t cg[8], ng[8];
  sd_subswath subs[8];
  int64_t az0[8];
  for (int k = 0; k < n; ++k) {
    SD_TRY(deburst_plan(ctx, &sw[k].sw, sw[k].bursts, sw[k].n_bursts, sw[k].tiff_height, &dp[k]));
    if (dp[k].offset + dp[k].samples > sw[k].tiff_width)
      return set_error(ctx, SD_ERR_INVALID_ARGUMENT, "valid window exceeds raster width in swath %d", k);
    SD_TRY(cal_plan(ctx, sw[k].cal, sw[k].n_cal, sw[k].noise_range, sw[k].n_noise_range, &sw[k].noise_azimuth,
                    dp[k].offset, dp[k].samples, sw[k].bursts[0].first_line, dp[k].lines, &cp[k]));
    lines[k] = dp[k].lines;
    samples[k] = dp[k].samples;
    voff[k] = dp[k].offset;
    cg[k] = cp[k].cal_gap;
    ng[k] = cp[k].nr_gap;
    subs[k] = sw[k].sw;
    az0[k] = sw[k].bursts[0].azimuth_time_us;
  }
  FillRange fr[8];
  SD_TRY(merge_plan(ctx, n, lines, samples, voff, subs, az0, info, fr));
  uint32_t cgm = 0, ngm = 0;
  for (int k = 0; k < n; ++k) {
    cgm = std::max(cgm, cg[k]);
    ngm = std::max(ngm, ng[k]);
  }
  info->cal_lut_extrapolation_gap_px = cgm;
  info->noise_lut_extrapolation_gap_px = ngm;
  if (!out) return SD_OK;
  if (!out_nesz) return set_error(ctx, SD_ERR_INVALID_ARGUMENT, "null nesz buffer");
  SD_CUDA(ctx, cudaSetDevice(ctx->device));
  MergeDev m{};
  m.n = n;
  const uint64_t L = info->lines, Cc = info->samples;
  for (int k = 0; k < n; ++k) {
    char tag[32];
    snprintf(tag, sizeof tag, "fu%d", k);
    CalSwathDev s{};
    // only the first L lines of each swath reach the merged raster
    cp[k].cal_lp.resize(L);
    cp[k].nr_lp.resize(L);
    cp[k].az.resize(L);
    SD_TRY(cal_device(ctx, tag, cp[k], dp[k].offset, dp[k].samples, &s));
    const void *d_raw;
    SD_TRY(stage_in(ctx, (std::string(tag) + ".raw").c_str(), sw[k].slc_iq,
                    sw[k].tiff_width * sw[k].tiff_height * 4, &d_raw));
    dp[k].line_map.resize(L);
    uint64_t *d_map;
    SD_TRY(upload(ctx, std::string(tag) + ".map", dp[k].line_map, &d_map));
    s.iq = (const int16_t *)d_raw;
    s.stride = sw[k].tiff_width;
    s.line_map = d_map;
    s.col0 = dp[k].offset;
    m.sw[k] = s;
    m.fr[k] = fr[k];
  }
  void *d_out, *d_nesz;
  SD_TRY(stage_out(ctx, "fu.out", out, L * Cc * 4, &d_out));
  SD_TRY(stage_out(ctx, "fu.nesz", out_nesz, L * Cc * 4, &d_nesz));
  if (L > 0 && Cc > 0) {
    const uint64_t nblk = ((Cc + FU_COLS - 1) / FU_COLS) * L;
    if (nblk > 0x7FFFFFFFull) return set_error(ctx, SD_ERR_INVALID_ARGUMENT, "merged raster too large");
    SD_TIMED_BEGIN(ctx, "k_fused");
    k_fused<<<(unsigned)nblk, FU_THREADS, 0, ctx->stream>>>(m, L, Cc, (float *)d_out, (float *)d_nesz);
    SD_LAUNCHED(ctx);
  }
  SD_TRY(finish_out(ctx, out, d_out, L * Cc * 4));
  SD_TRY(finish_out(ctx, out_nesz, d_nesz, L * Cc * 4));
  return sync(ctx);
}

// ═══════════════════════════════════════════════════════════════════════════
// Allocation-free calibration
//
// Some callers cannot allocate device memory once they are running: a
// serving process that reserved its whole HBM budget up front in its own
// pool, a pipeline stage that must not let cudaMalloc/cudaFree serialise the
// device behind other streams, or a host that only hands this library
// buffers it already owns.  sd_apply_calibration_noalloc gives them the same
// result as sd_apply_calibration without any device allocation: its working
// memory (LUT vectors, per-column LUT tables, per-line brackets) lives in
// one file-scope __device__ array of fixed size, and the caller passes the
// deburst raster and both outputs as device memory it owns.
// ═══════════════════════════════════════════════════════════════════════════
namespace sd {
namespace {

// Capacity of the static working memory (20 MiB; every device that loads the
// library keeps it for the life of the process).
constexpr uint64_t NA_MAX_VECTORS = 64;          // per LUT family
constexpr uint64_t NA_MAX_POINTS = 64 * 1024;    // LUT knots per family, all vectors
constexpr uint64_t NA_MAX_SAMPLES = 32 * 1024;   // output columns
constexpr uint64_t NA_MAX_LINES = 32 * 1024;     // output lines
constexpr size_t NA_SCRATCH_BYTES = 20u << 20;

static __device__ __align__(256) unsigned char g_noalloc_scratch[NA_SCRATCH_BYTES];

struct NaLayout {  // byte offsets inside the static array
  size_t off[2][5];  // per family: px, pm, val, off, cnt
  size_t tab[2];
  size_t lp[2];
  size_t az;
  size_t total;
};

size_t na_align(size_t x) { return (x + 255) & ~(size_t)255; }

NaLayout na_layout(const CalPlan &P, uint64_t lines, uint64_t samples) {
  NaLayout L{};
  size_t o = 0;
  for (int f = 0; f < 2; ++f) {
    const LutHost &H = f == 0 ? P.cal : P.nr;
    size_t pts = H.px.size(), nv = H.lines.size();
    size_t sz[5] = {pts * 4, pts * 4, pts * 4, nv * 8, nv * 8};
    for (int k = 0; k < 5; ++k) {
      L.off[f][k] = o;
      o = na_align(o + std::max<size_t>(sz[k], 1));
    }
  }
  for (int f = 0; f < 2; ++f) {
    const LutHost &H = f == 0 ? P.cal : P.nr;
    L.tab[f] = o;
    o = na_align(o + std::max<size_t>(H.lines.size() * samples * 4, 1));
  }
  for (int f = 0; f < 2; ++f) {
    L.lp[f] = o;
    o = na_align(o + std::max<size_t>(lines * sizeof(LineParams), 1));
  }
  L.az = o;
  o = na_align(o + std::max<size_t>(lines * 4, 1));
  L.total = o;
  return L;
}

// k_calibrate with output line l read from raster row l (no line-map buffer).
__global__ void k_calibrate_direct(CalSwathDev s, uint64_t lines, uint64_t samples, float *out, float *nesz) {
  uint64_t c = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  uint64_t l = blockIdx.y;
  if (c >= samples || l >= lines) return;
  const uint32_t iqw = __ldg((const uint32_t *)(s.iq) + l * s.stride + c);
  const int32_t i = (int32_t)(int16_t)(iqw & 0xFFFF), q = (int32_t)(int16_t)(iqw >> 16);
  const float power = (float)(int32_t)((uint32_t)(i * i) + (uint32_t)(q * q));
  const LineParams cl = s.cal_lp[l], nl = s.nr_lp[l];
  float k = __ldg(s.cal_tab + (uint64_t)cl.lo * s.tab_cols + c);
  if (cl.lo != cl.hi) k = lerpf(k, __ldg(s.cal_tab + (uint64_t)cl.hi * s.tab_cols + c), cl.t);
  float nrv = __ldg(s.nr_tab + (uint64_t)nl.lo * s.tab_cols + c);
  if (nl.lo != nl.hi) nrv = lerpf(nrv, __ldg(s.nr_tab + (uint64_t)nl.hi * s.tab_cols + c), nl.t);
  const float k2 = k * k;
  const float valid = (k2 > 0.0f) ? 1.0f : 0.0f;
  const float inv_k2 = (k2 > 0.0f) ? 1.0f / k2 : 0.0f;
  const float noise_val = nrv * s.az[l];
  out[l * samples + c] = maxf_nan(power - noise_val, 0.0f) * inv_k2 * valid;
  nesz[l * samples + c] = noise_val * inv_k2 * valid;
}

template <class T>
int na_copy(sd_ctx *c, unsigned char *base, size_t off, const std::vector<T> &v) {
  if (!v.empty())
    SD_CUDA(c, cudaMemcpyAsync(base + off, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, c->stream));
  return SD_OK;
}

int noalloc_run(sd_ctx *c, const int16_t *iq, uint64_t lines, uint64_t samples, uint64_t col_offset,
                const sd_lut_vector *cal, uint64_t n_cal, const sd_lut_vector *nr, uint64_t n_nr,
                const sd_noise_azimuth *az, uint64_t tiff_line_origin, float *out, float *nesz,
                uint32_t *cal_gap, uint32_t *nr_gap) {
  // The LUT tables, line parameters and azimuth vector are staged from host
  // vectors that live only for this call: a capturing stream would record
  // copies from memory that is gone when the graph replays.
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(c->stream, &cap) != cudaSuccess) {
    const cudaError_t e = cudaGetLastError();
    return set_error(c, SD_ERR_CUDA, "cudaStreamIsCapturing failed: %s", cudaGetErrorString(e));
  }
  if (cap != cudaStreamCaptureStatusNone)
    return set_error(c, SD_ERR_INVALID_ARGUMENT,
                     "allocation-free calibration stages host data per call and cannot run on a capturing stream");
  if ((n_cal && !cal) || (n_nr && !nr))
    return set_error(c, SD_ERR_INVALID_ARGUMENT, "null LUT vector array with a non-zero count");
  // size limits first: the static working memory is fixed
  if (n_cal > NA_MAX_VECTORS || n_nr > NA_MAX_VECTORS)
    return set_error(c, SD_ERR_INVALID_ARGUMENT,
                     "allocation-free calibration supports at most %llu LUT vectors per family (got %llu / %llu)",
                     (unsigned long long)NA_MAX_VECTORS, (unsigned long long)n_cal, (unsigned long long)n_nr);
  uint64_t pts_cal = 0, pts_nr = 0;
  for (uint64_t i = 0; cal && i < n_cal; ++i) pts_cal += cal[i].n;
  for (uint64_t i = 0; nr && i < n_nr; ++i) pts_nr += nr[i].n;
  if (pts_cal > NA_MAX_POINTS || pts_nr > NA_MAX_POINTS)
    return set_error(c, SD_ERR_INVALID_ARGUMENT,
                     "allocation-free calibration supports at most %llu LUT knots per family (got %llu / %llu)",
                     (unsigned long long)NA_MAX_POINTS, (unsigned long long)pts_cal, (unsigned long long)pts_nr);
  if (samples > NA_MAX_SAMPLES || lines > NA_MAX_LINES)
    return set_error(c, SD_ERR_INVALID_ARGUMENT,
                     "allocation-free calibration supports at most %llu x %llu (lines x samples); got %llu x %llu",
                     (unsigned long long)NA_MAX_LINES, (unsigned long long)NA_MAX_SAMPLES,
                     (unsigned long long)lines, (unsigned long long)samples);
  CalPlan P;
  SD_TRY(cal_plan(c, cal, n_cal, nr, n_nr, az, col_offset, samples, tiff_line_origin, lines, &P));
  if (cal_gap) *cal_gap = P.cal_gap;
  if (nr_gap) *nr_gap = P.nr_gap;
  if (lines == 0 || samples == 0) return SD_OK;
  if (!iq || !out || !nesz) return set_error(c, SD_ERR_INVALID_ARGUMENT, "null buffer");
  if (!is_device_ptr(iq) || !is_device_ptr(out) || !is_device_ptr(nesz))
    return set_error(c, SD_ERR_INVALID_ARGUMENT,
                     "allocation-free calibration needs device (or managed) memory for the raster and both outputs");
  NaLayout L = na_layout(P, lines, samples);
  if (L.total > NA_SCRATCH_BYTES)
    return set_error(c, SD_ERR_INVALID_ARGUMENT, "working set %zu B exceeds the %zu B static scratch", L.total,
                     NA_SCRATCH_BYTES);
  // The array's device address on the current device.  It is looked up on
  // every call (a table lookup, not a stream operation): an address cached
  // across calls would go stale after cudaDeviceReset or a recreated primary
  // context, when the module reloads elsewhere.  The first call on a device
  // also loads the module there.
  unsigned char *base = nullptr;
  {
    void *p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p) {
      cudaGetLastError();
      return set_error(c, SD_ERR_CUDA, "cudaGetSymbolAddress(g_noalloc_scratch) failed: %s",
                       cudaGetErrorString(e));
    }
    base = (unsigned char *)p;
  }
  CalSwathDev s{};
  for (int f = 0; f < 2; ++f) {
    const LutHost &H = f == 0 ? P.cal : P.nr;
    SD_TRY(na_copy(c, base, L.off[f][0], H.px));
    SD_TRY(na_copy(c, base, L.off[f][1], H.pm));
    SD_TRY(na_copy(c, base, L.off[f][2], H.val));
    SD_TRY(na_copy(c, base, L.off[f][3], H.off));
    SD_TRY(na_copy(c, base, L.off[f][4], H.cnt));
    LutDev d{(const uint32_t *)(base + L.off[f][0]), (const uint32_t *)(base + L.off[f][1]),
             (const float *)(base + L.off[f][2]), (const uint64_t *)(base + L.off[f][3]),
             (const uint64_t *)(base + L.off[f][4])};
    float *tab = (float *)(base + L.tab[f]);
    uint64_t nv = H.lines.size();
    SD_TIMED_BEGIN(c, "k_lut_table");
    k_lut_table<<<grid_for(nv * samples, 256), 256, 0, c->stream>>>(d, nv, samples, col_offset, tab);
    SD_LAUNCHED(c);
    (f == 0 ? s.cal_tab : s.nr_tab) = tab;
  }
  SD_TRY(na_copy(c, base, L.lp[0], P.cal_lp));
  SD_TRY(na_copy(c, base, L.lp[1], P.nr_lp));
  SD_TRY(na_copy(c, base, L.az, P.az));
  s.tab_cols = samples;
  s.cal_lp = (const LineParams *)(base + L.lp[0]);
  s.nr_lp = (const LineParams *)(base + L.lp[1]);
  s.az = (const float *)(base + L.az);
  s.iq = iq;
  s.stride = samples;
  s.line_map = nullptr;
  s.col0 = 0;
  // identity line map without a buffer: one launch per line block
  for (uint64_t l0 = 0; l0 < lines; l0 += 65535) {
    uint64_t nl = std::min<uint64_t>(65535, lines - l0);
    CalSwathDev sl = s;
    sl.iq = iq + l0 * samples * 2;
    sl.cal_lp = s.cal_lp + l0;
    sl.nr_lp = s.nr_lp + l0;
    sl.az = s.az + l0;
    dim3 grid(grid_for(samples, 256), (unsigned)nl);
    SD_TIMED_BEGIN(c, "k_calibrate_noalloc");
    k_calibrate_direct<<<grid, 256, 0, c->stream>>>(sl, nl, samples, out + l0 * samples, nesz + l0 * samples);
    SD_LAUNCHED(c);
  }
  return SD_OK;
}

}  // namespace
}  // namespace sd

extern "C" int sd_apply_calibration_noalloc(void *stream, const int16_t *deburst_iq, uint64_t lines,
                                            uint64_t samples, uint64_t valid_sample_offset,
                                            const sd_lut_vector *cal, uint64_t n_cal,
                                            const sd_lut_vector *noise_range, uint64_t n_noise_range,
                                            const sd_noise_azimuth *noise_azimuth, uint64_t tiff_line_origin,
                                            float *out_sigma0, float *out_nesz, uint32_t *cal_gap_px,
                                            uint32_t *noise_gap_px, char *err, uint64_t err_len) {
  SD_STAGE("calibration");
  sd_ctx c;  // host-side bookkeeping only; owns no device memory
  int dev = 0;
  int rc;
  if (cudaGetDevice(&dev) != cudaSuccess) {
    cudaGetLastError();
    rc = sd::set_error(&c, SD_ERR_CUDA, "no current CUDA device");
  } else {
    c.device = dev;
    c.stream = (cudaStream_t)stream;
    rc = sd::noalloc_run(&c, deburst_iq, lines, samples, valid_sample_offset, cal, n_cal, noise_range,
                         n_noise_range, noise_azimuth, tiff_line_origin, out_sigma0, out_nesz, cal_gap_px,
                         noise_gap_px);
  }
  if (err && err_len > 0) {
    size_t n = std::min<size_t>(c.last_error.size(), err_len - 1);
    memcpy(err, c.last_error.data(), n);
    err[n] = 0;
  }
  c.stream = nullptr;  // the caller's stream is not ours to destroy
  return rc;
}
