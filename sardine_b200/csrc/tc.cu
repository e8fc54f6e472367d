// tc.cu — terrain_correction (terrain_correction.rs:1245-1836) of one scene
// onto its output grid: the single-job form of the stages in tc_kernels.cuh.
#include "tc_kernels.cuh"

namespace sd {

// ── host side ─────────────────────────────────────────────────────────────
int tc_output_grid_host(const sd_scene *scene, const sd_tc_config *cfg, sd_geocoded_info *info) {
  std::memset(info, 0, sizeof(*info));
  if (!(cfg->pixel_spacing > 0.0)) return SD_ERR_TC_CONFIG;
  const double sp = cfg->pixel_spacing;
  double n, s, w, e;
  if (cfg->crs == SD_CRS_WGS84) {
    n = std::ceil(scene->max_lat_deg / sp) * sp;
    s = std::floor(scene->min_lat_deg / sp) * sp;
    w = std::floor(scene->min_lon_deg / sp) * sp;
    e = std::ceil(scene->max_lon_deg / sp) * sp;
  } else if (cfg->crs == SD_CRS_UTM_NORTH || cfg->crs == SD_CRS_UTM_SOUTH) {
    if (cfg->utm_zone < 1 || cfg->utm_zone > 60) return SD_ERR_TC_PROJECTION;
    Utm u = make_utm(cfg->utm_zone, cfg->crs == SD_CRS_UTM_SOUTH);
    const double corners[4][2] = {{scene->min_lon_deg, scene->min_lat_deg},
                                  {scene->min_lon_deg, scene->max_lat_deg},
                                  {scene->max_lon_deg, scene->min_lat_deg},
                                  {scene->max_lon_deg, scene->max_lat_deg}};
    double xmin = INFINITY, xmax = -INFINITY, ymin = INFINITY, ymax = -INFINITY;
    for (auto &cn : corners) {
      double x, y;
      utm_lonlat_to_xy(u, cn[0], cn[1], &x, &y);
      if (x < xmin) xmin = x;
      if (x > xmax) xmax = x;
      if (y < ymin) ymin = y;
      if (y > ymax) ymax = y;
    }
    n = std::ceil(ymax / sp) * sp;
    s = std::floor(ymin / sp) * sp;
    w = std::floor(xmin / sp) * sp;
    e = std::ceil(xmax / sp) * sp;
  } else {
    return SD_ERR_TC_PROJECTION;
  }
  uint64_t rows = f2u64(std::round((n - s) / sp));
  uint64_t cols = f2u64(std::round((e - w) / sp));
  info->rows = rows;
  info->cols = cols;
  info->origin_lat_deg = n;
  info->origin_lon_deg = w;
  info->pixel_spacing = sp;
  info->geotransform[0] = w;
  info->geotransform[1] = sp;
  info->geotransform[3] = n;
  info->geotransform[5] = -sp;
  info->total_pixel_count = rows * cols;
  if (rows == 0 || cols == 0) return SD_ERR_TC_CONFIG;
  return SD_OK;
}

}  // namespace sd

namespace sd {
// this unit's bounds-check word (see runtime.cuh)
SD_BOUNDS_ACCESSOR(bounds_read_tc)
}  // namespace sd

using namespace sd;

extern "C" int sd_tc_output_grid(sd_ctx *ctx, const sd_scene *scene, const sd_tc_config *cfg,
                                 sd_geocoded_info *info) {
  if (!scene || !cfg || !info) return SD_ERR_INVALID_ARGUMENT;
  int rc = tc_output_grid_host(scene, cfg, info);
  if (rc != SD_OK) set_error(ctx, rc, "output grid is empty or the CRS is invalid");
  return rc;
}
namespace sd {
namespace {

// Single job: k_main with the job record as a kernel parameter; the later
// stages specialised per resampling kernel.
int launch_pixels_single(sd_ctx *ctx, const TcWork *d_work, const uint64_t *totals, int kernel, bool split,
                         const TcDev *job) {
  if (kernel == SD_RESAMPLE_BICUBIC)
    return split ? launch_pixels_t<SD_RESAMPLE_BICUBIC, true>(ctx, d_work, totals, job)
                 : launch_pixels_t<SD_RESAMPLE_BICUBIC, false>(ctx, d_work, totals, job);
  if (kernel == SD_RESAMPLE_LANCZOS3)
    return split ? launch_pixels_t<SD_RESAMPLE_LANCZOS3, true>(ctx, d_work, totals, job)
                 : launch_pixels_t<SD_RESAMPLE_LANCZOS3, false>(ctx, d_work, totals, job);
  return split ? launch_pixels_t<SD_RESAMPLE_BILINEAR, true>(ctx, d_work, totals, job)
               : launch_pixels_t<SD_RESAMPLE_BILINEAR, false>(ctx, d_work, totals, job);
}

}  // namespace

int launch_main_param(sd_ctx *ctx, const void *job, cudaStream_t st) {
  const TcDev &p = *static_cast<const TcDev *>(job);
  const uint64_t items = main_items(p);
  if (items == 0) return SD_OK;
  if (items > 0x7FFFFFFFull) return set_error(ctx, SD_ERR_INVALID_ARGUMENT, "tile too large");
  const unsigned g = (unsigned)items;
  k_main<<<g, MAIN_THREADS, 0, st>>>(p);
  ctx->launches++;
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return set_error(ctx, SD_ERR_CUDA, "kernel launch failed: %s", cudaGetErrorString(e));
  return SD_OK;
}

}  // namespace sd

static int tc_run(sd_ctx *ctx, const sd_radar_image *image, const sd_scene *scene, const sd_dem *dem,
                  const sd_geoid *geoid, const sd_geo_grid_point *grid, uint64_t n_grid,
                  const sd_tc_config *cfg, uint64_t row_begin, uint64_t row_end, float *out_data,
                  float *out_cos_lia, uint8_t *out_mask, int64_t *out_times, sd_geocoded_info *info) {
  if (!ctx) return SD_ERR_INVALID_ARGUMENT;
  if (!image || !scene || !dem || !geoid || !cfg || !info || !out_data)
    return set_error(ctx, SD_ERR_INVALID_ARGUMENT, "null argument");
  if (cfg->compute_lia && (!out_cos_lia || !out_mask))
    return set_error(ctx, SD_ERR_INVALID_ARGUMENT, "compute_lia needs cos_lia and mask buffers");
  SD_CUDA(ctx, cudaSetDevice(ctx->device));
  // argument checks in the reference's order (terrain_correction.rs:1262-1283)
  if (n_grid == 0) return set_error(ctx, SD_ERR_TC_NO_GRID_POINTS, "no geolocation grid points provided");
  if (!(cfg->pixel_spacing > 0.0)) return set_error(ctx, SD_ERR_TC_CONFIG, "pixel spacing must be positive");
  if (scene->n_sub_swaths <= 0)
    return set_error(ctx, SD_ERR_TC_NO_SUBSWATHS, "scene has no subswaths — cannot derive radar geometry");
  const double ati = scene->azimuth_time_interval_s;
  if (!std::isfinite(ati) || ati <= 0.0)
    return set_error(ctx, SD_ERR_TC_CONFIG, "invalid azimuth_time_interval_s in subswath metadata: %g", ati);
  // build_azimuth_time_lut (1080-1104): stable sort by latitude, keep first of near-duplicates
  std::vector<std::pair<double, int64_t>> lut;
  for (uint64_t k = 0; k < n_grid; ++k) lut.push_back({grid[k].latitude_deg, grid[k].azimuth_time_us});
  std::stable_sort(lut.begin(), lut.end(), [](auto &a, auto &b) { return a.first < b.first; });
  std::vector<double> lut_lat;
  std::vector<int64_t> lut_t;
  for (auto &pt : lut) {
    if (!lut_lat.empty() && std::fabs(pt.first - lut_lat.back()) < 1e-6) continue;
    lut_lat.push_back(pt.first);
    lut_t.push_back(pt.second);
  }
  if (lut_lat.empty()) return set_error(ctx, SD_ERR_TC_NO_GRID_POINTS, "no geolocation grid points provided");
  SD_TRY(sd_tc_output_grid(ctx, scene, cfg, info));
  if (cfg->projector_anchors <= 0)
    return set_error(ctx, SD_ERR_TC_CONFIG, "SARDINE_TC_PROJECTOR_ANCHORS must be >= 1 (default 256)");
  if (cfg->precision != SD_PRECISION_FP64 && cfg->precision != SD_PRECISION_SPLIT)
    return set_error(ctx, SD_ERR_TC_CONFIG, "unknown precision mode %d", cfg->precision);
  if (dem->width < 2 || dem->height < 2 || !(dem->pixel_size > 0.0))
    return set_error(ctx, SD_ERR_INVALID_ARGUMENT, "DEM grid must be at least 2x2 with positive spacing");
  if (image->lines == 0 || image->samples == 0)
    return set_error(ctx, SD_ERR_INVALID_ARGUMENT, "radar image is empty");

  TcDev p{};
  if (row_end == 0 || row_end > info->rows) row_end = info->rows;
  if (row_begin >= row_end)
    return set_error(ctx, SD_ERR_INVALID_ARGUMENT, "empty row band [%llu, %llu)",
                     (unsigned long long)row_begin, (unsigned long long)row_end);
  p.rows = row_end - row_begin;
  p.row0 = row_begin;
  p.cols = info->cols;
  p.lat_north = info->origin_lat_deg;
  p.lon_west = info->origin_lon_deg;
  p.sp = cfg->pixel_spacing;
  p.utm = cfg->crs != SD_CRS_WGS84;
  if (p.utm) p.proj = make_utm(cfg->utm_zone, cfg->crs == SD_CRS_UTM_SOUTH);
  p.step_deg = p.utm ? p.sp / 111320.0 : p.sp;  // cardinal_neighbour_step_deg (452-465)
  p.lines = image->lines;
  p.samples = image->samples;
  p.az_start = image->azimuth_start_time_us;
  p.ati = ati;
  p.near_range = image->near_slant_range_time_s * SPEED_OF_LIGHT / 2.0;
  p.rps = image->range_pixel_spacing_m;
  p.max_iter = cfg->max_newton_iterations < 0 ? 0 : cfg->max_newton_iterations;
  p.tol = cfg->newton_tolerance_s;
  p.flatten = cfg->flatten != 0;
  p.compute_lia = cfg->compute_lia != 0;
  p.need_geom = p.flatten || p.compute_lia;
  p.resampling = cfg->resampling;
  p.nesz_mask = std::isfinite(cfg->noise_floor_margin_db) && image->nesz != nullptr;
  p.nesz_factor = p.nesz_mask ? std::pow(10.0f, cfg->noise_floor_margin_db / 10.0f) : 0.0f;
  const uint64_t npx = p.rows * p.cols;
  cudaStream_t st = ctx->stream;

  // ── inputs ──
  const void *d_img, *d_nesz = nullptr, *d_dem, *d_geoid = nullptr, *d_svs;
  SD_TRY(stage_in(ctx, "tc.img", image->data, image->lines * image->samples * sizeof(float), &d_img));
  if (p.nesz_mask)
    SD_TRY(stage_in(ctx, "tc.nesz", image->nesz, image->lines * image->samples * sizeof(float), &d_nesz));
  SD_TRY(stage_in(ctx, "tc.dem", dem->data, dem->width * dem->height * sizeof(float), &d_dem));
  if (geoid->kind == SD_GEOID_GRID) {
    if (!geoid->undulations_m) return set_error(ctx, SD_ERR_INVALID_ARGUMENT, "geoid grid is null");
    SD_TRY(stage_in(ctx, "tc.geoid", geoid->undulations_m, 73 * 144 * sizeof(float), &d_geoid));
  }
  const uint64_t nsv = scene->n_state_vectors;
  SD_TRY(stage_in(ctx, "tc.svs", scene->state_vectors, std::max<uint64_t>(nsv, 1) * sizeof(sd_state_vector), &d_svs));
  double *d_lut_lat;
  int64_t *d_lut_t;
  SD_TRY(scratch_t(ctx, "tc.lut_lat", lut_lat.size(), &d_lut_lat));
  SD_TRY(scratch_t(ctx, "tc.lut_t", lut_t.size(), &d_lut_t));
  SD_CUDA(ctx, cudaMemcpyAsync(d_lut_lat, lut_lat.data(), lut_lat.size() * 8, cudaMemcpyHostToDevice, st));
  SD_CUDA(ctx, cudaMemcpyAsync(d_lut_t, lut_t.data(), lut_t.size() * 8, cudaMemcpyHostToDevice, st));
  p.img = (const float *)d_img;
  p.nesz = (const float *)d_nesz;
  p.geoid = (const float *)d_geoid;
  p.lut_lat = d_lut_lat;
  p.lut_t = d_lut_t;
  p.lut_n = (int)lut_lat.size();
  p.dem.data = (const float *)d_dem;
  p.dem.width = dem->width;
  p.dem.height = dem->height;
  p.dem.origin_y = dem->origin_y;
  p.dem.origin_x = dem->origin_x;
  p.dem.pixel_size = dem->pixel_size;
  p.dem.inv_ps = 1.0 / dem->pixel_size;
  p.dem.kind = dem->kind;
  if (dem->kind == SD_DEM_PROJECTED_UTM) {
    if (dem->utm_zone < 1 || dem->utm_zone > 60)
      return set_error(ctx, SD_ERR_TC_DEM, "projected DEM needs a UTM zone in 1..60");
    p.dem.utm = make_utm(dem->utm_zone, dem->utm_south != 0);
  }
  p.orb.svs = (const sd_state_vector *)d_svs;
  p.orb.n = nsv;
  p.orb.tab = nullptr;
  p.orb.tab_t0 = 0;
  p.orb.tab_n = 0;
  p.orb.poly = nullptr;
  SD_TRY(upload_orbit_poly(ctx, "tc.orbit_poly", scene->state_vectors, nsv, &p.orb));

  // ── per-row scratch, per-pixel scratch and outputs ──
  int64_t *d_row_guess, *d_knots;
  double *d_row_flat, *d_ax = nullptr, *d_alon = nullptr, *d_alat = nullptr;
  SD_TRY(scratch_t(ctx, "tc.row_guess", p.rows, &d_row_guess));
  SD_TRY(scratch_t(ctx, "tc.row_flat", p.rows, &d_row_flat));
  SD_TRY(scratch_t(ctx, "tc.knots", p.rows * KNOTS, &d_knots));
  unsigned long long *d_trange;
  SD_TRY(scratch_t(ctx, "tc.trange", 2, &d_trange));
  p.row_guess = d_row_guess;
  p.row_flat = d_row_flat;
  p.knot_t = d_knots;
  p.trange = d_trange;
  unsigned long long tr_init[2] = {~0ull, 0ull};
  SD_CUDA(ctx, cudaMemcpyAsync(d_trange, tr_init, sizeof tr_init, cudaMemcpyHostToDevice, st));
  std::vector<double> ax;
  if (p.utm) {
    // project_row anchors (output_crs.rs:383-396); x positions are row-independent
    const uint64_t n_anchors = std::min<uint64_t>((uint64_t)cfg->projector_anchors, p.cols);
    const double x_start = p.lon_west + 0.5 * p.sp;
    const double x_end = x_start + ((double)p.cols - 1.0) * p.sp;
    const double anchor_dx = (x_end - x_start) / (double)n_anchors;
    for (uint64_t a = 0; a <= n_anchors; ++a) ax.push_back(x_start + (double)a * anchor_dx);
    p.n_anchors = (int)n_anchors;
    p.n_pts = (int)n_anchors + 1;
    SD_TRY(scratch_t(ctx, "tc.ax", ax.size(), &d_ax));
    SD_TRY(scratch_t(ctx, "tc.alon", p.rows * p.n_pts, &d_alon));
    SD_TRY(scratch_t(ctx, "tc.alat", p.rows * p.n_pts, &d_alat));
    SD_CUDA(ctx, cudaMemcpyAsync(d_ax, ax.data(), ax.size() * 8, cudaMemcpyHostToDevice, st));
    p.ax = d_ax;
    p.alon = d_alon;
    p.alat = d_alat;
    if (p.dem.kind == SD_DEM_PROJECTED_UTM) {
      UtmLocal *d_aloc;
      SD_TRY(scratch_t(ctx, "tc.aloc", p.rows * p.n_pts, &d_aloc));
      p.aloc = d_aloc;
    }
  }
  double *d_tp, *d_fct = nullptr;
  SD_TRY(scratch_t(ctx, "tc.target", 3 * npx, &d_tp));
  if (p.need_geom) SD_TRY(scratch_t(ctx, "tc.facet", 4 * npx, &d_fct));
  p.tp = d_tp;
  p.fct = d_fct;
  SD_TRY(scratch_t(ctx, "tc.fb", npx, &p.fb));
  SD_TRY(scratch_t(ctx, "tc.cc", npx, &p.cc));
  SD_TRY(scratch_t(ctx, "tc.sel", npx, &p.sel));
  void *d_out, *d_cos = nullptr, *d_mask = nullptr;
  SD_TRY(stage_out(ctx, "tc.out", out_data, npx * sizeof(float), &d_out));
  if (p.compute_lia) {
    SD_TRY(stage_out(ctx, "tc.cos", out_cos_lia, npx * sizeof(float), &d_cos));
    SD_TRY(stage_out(ctx, "tc.mask", out_mask, npx, &d_mask));
  }
  void *d_times = nullptr;
  if (out_times) SD_TRY(stage_out(ctx, "tc.times", out_times, npx * sizeof(int64_t), &d_times));
  p.out = (float *)d_out;
  p.cos_lia = (float *)d_cos;
  p.mask = (uint8_t *)d_mask;
  p.az_time = (int64_t *)d_times;
  p.flags = ctx->d_flags;
  p.counters = ctx->d_counters;
  p.db = ctx->db_out;
  p.db_floor = ctx->db_floor;
  SD_CUDA(ctx, cudaMemsetAsync(ctx->d_flags, 0, 64 * sizeof(int), st));
  SD_CUDA(ctx, cudaMemsetAsync(ctx->d_counters, 0, 64 * sizeof(unsigned long long), st));
  // The candidate-set scheme needs tol <= 1 us (then at most three
  // consecutive microseconds can satisfy |delta| < tol).  Larger tolerances
  // leave every pixel to the row walk's exact path.
  p.fast = (p.tol <= 1e-6) ? 1 : 0;
  set_main_segments(&p);
  p.split = cfg->precision == SD_PRECISION_SPLIT;
  if (p.split) {  // FP64 re-sample queue of every k_cand item
    const uint64_t items = stage_items(WK_SEL, p);
    SD_TRY(scratch_t(ctx, "tc.rs_cnt", items, &p.rs_cnt));
    SD_TRY(scratch_t(ctx, "tc.rs_ent", items * RS_CAP, &p.rs_ent));
  }

  // ── one-job work table ──
  TcWorkHost wk;
  TcWork *d_work = nullptr;
  SD_TRY(work_upload(ctx, "tc.work", &p, 1, &wk, &d_work));
  SD_TRY(launch_rows(ctx, d_work, wk.totals, &p));  // k_heights in its parameter form
  unsigned long long tr[2];
  SD_CUDA(ctx, cudaMemcpyAsync(tr, d_trange, sizeof tr, cudaMemcpyDeviceToHost, st));
  SD_TRY(sync(ctx));

  // ── orbit table over the row models' time span, inside the SV window ──
  if (nsv >= 8 && tr[0] <= tr[1]) {
    int64_t tmin = (int64_t)(tr[0] ^ 0x8000000000000000ull);
    int64_t tmax = (int64_t)(tr[1] ^ 0x8000000000000000ull);
    // +-0.1 s covers the height and interpolation spread of pixel roots
    // around the row models; iterates outside the table are evaluated directly.
    int64_t t0 = std::max(scene->state_vectors[0].time_us, tmin - 100000);
    int64_t t1 = std::min(scene->state_vectors[nsv - 1].time_us, tmax + 100000);
    // a table larger than the grid costs more to build than it saves
    if (t1 >= t0 && (uint64_t)(t1 - t0 + 1) <= npx) {
      SD_TRY(build_orbit_table(ctx, "tc.orbit_table", "tc.orbit_taylor", (const sd_state_vector *)d_svs, nsv, t0,
                               t1, tmin, tmax, &p.orb));
      // the job record on the device carries the table
      SD_CUDA(ctx, cudaMemcpyAsync((void *)wk.d_jobs, &p, sizeof(TcDev), cudaMemcpyHostToDevice, st));
    }
  }
  const bool split = cfg->precision == SD_PRECISION_SPLIT;
  SD_TRY(launch_pixels_single(ctx, d_work, wk.totals, p.resampling, split, &p));
  int flags[64];
  unsigned long long cnt[kCounters + SD_NEWTON_ITER_HIST_SIZE];
  SD_CUDA(ctx, cudaMemcpyAsync(flags, ctx->d_flags, sizeof flags, cudaMemcpyDeviceToHost, st));
  SD_CUDA(ctx, cudaMemcpyAsync(cnt, ctx->d_counters, sizeof cnt, cudaMemcpyDeviceToHost, st));
  SD_TRY(sync(ctx));
  if (flags[5]) return set_error(ctx, SD_ERR_INTERNAL, "terrain correction: a converged pixel lost its DEM height");
  if (flags[0]) {
    return set_error(ctx, SD_ERR_TC_ORBIT,
                     "orbit interpolation failed: interpolation time outside orbit window; "
                     "refusing to extrapolate");
  }
  // dB output: the statistics of the converted raster while it is on the device
  if (p.db) SD_TRY(db_finish(ctx, (const float *)d_out, npx, cnt[kCntDb], cnt[kCntDb + 1]));
  SD_TRY(finish_out(ctx, out_data, d_out, npx * sizeof(float)));
  if (p.compute_lia) {
    SD_TRY(finish_out(ctx, out_cos_lia, d_cos, npx * sizeof(float)));
    SD_TRY(finish_out(ctx, out_mask, d_mask, npx));
  }
  if (out_times) SD_TRY(finish_out(ctx, out_times, d_times, npx * sizeof(int64_t)));
  info->valid_pixel_count = cnt[0];
  info->dem_missing_count = cnt[1];
  info->outside_footprint_count = cnt[2];
  info->non_converged_count = cnt[3];
  info->degenerate_geometry_count = cnt[4];
  info->flat_masked_count = cnt[5];
  info->noise_masked_count = cnt[6];
  for (int k = 0; k < SD_NEWTON_ITER_HIST_SIZE; ++k) info->newton_iter_histogram[k] = cnt[kCounters + k];
  log_newton_hist(cnt + kCounters, SD_NEWTON_ITER_HIST_SIZE);
  info->diag_exact_path_pixels = (uint64_t)flags[1];
  info->diag_fp64_redo_pixels = (uint64_t)flags[2];
  info->diag_fp64_resampled = (uint64_t)flags[4];
  SD_TRY(sync(ctx));
  return SD_OK;
}

extern "C" int sd_terrain_correction(sd_ctx *ctx, const sd_radar_image *image, const sd_scene *scene,
                                     const sd_dem *dem, const sd_geoid *geoid,
                                     const sd_geo_grid_point *grid, uint64_t n_grid,
                                     const sd_tc_config *cfg, float *out_data, float *out_cos_lia,
                                     uint8_t *out_mask, sd_geocoded_info *info) {
  SD_STAGE("terrain_correction");
  return tc_run(ctx, image, scene, dem, geoid, grid, n_grid, cfg, 0, 0, out_data, out_cos_lia, out_mask,
                nullptr, info);
}

extern "C" int sd_terrain_correction_with_times(sd_ctx *ctx, const sd_radar_image *image,
                                                const sd_scene *scene, const sd_dem *dem,
                                                const sd_geoid *geoid, const sd_geo_grid_point *grid,
                                                uint64_t n_grid, const sd_tc_config *cfg, float *out_data,
                                                float *out_cos_lia, uint8_t *out_mask,
                                                int64_t *out_azimuth_time_us, sd_geocoded_info *info) {
  SD_STAGE("terrain_correction");
  if (!ctx) return SD_ERR_INVALID_ARGUMENT;
  if (!out_azimuth_time_us) return set_error(ctx, SD_ERR_INVALID_ARGUMENT, "null time buffer");
  return tc_run(ctx, image, scene, dem, geoid, grid, n_grid, cfg, 0, 0, out_data, out_cos_lia, out_mask,
                out_azimuth_time_us, info);
}

extern "C" int sd_terrain_correction_rows(sd_ctx *ctx, const sd_radar_image *image, const sd_scene *scene,
                                          const sd_dem *dem, const sd_geoid *geoid,
                                          const sd_geo_grid_point *grid, uint64_t n_grid,
                                          const sd_tc_config *cfg, uint64_t row_begin, uint64_t row_end,
                                          float *out_data, float *out_cos_lia, uint8_t *out_mask,
                                          int64_t *out_azimuth_time_us, sd_geocoded_info *info) {
  SD_STAGE("terrain_correction");
  return tc_run(ctx, image, scene, dem, geoid, grid, n_grid, cfg, row_begin, row_end, out_data, out_cos_lia,
                out_mask, out_azimuth_time_us, info);
}

namespace sd {
namespace {
__global__ void k_orbit_states(OrbitDev o, const int64_t *t, uint64_t m, double *out, int *flag) {
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= m) return;
  OrbitState s;
  double vsq;
  if (orbit_at(o, t[i], &s, &vsq) != ORB_OK) {
    atomicOr(flag, 1);
    return;
  }
  double *r = out + 9 * i;
  r[0] = s.pos.x, r[1] = s.pos.y, r[2] = s.pos.z;
  r[3] = s.vel.x, r[4] = s.vel.y, r[5] = s.vel.z;
  r[6] = s.acc.x, r[7] = s.acc.y, r[8] = s.acc.z;
}
}  // namespace
}  // namespace sd

extern "C" int sd_orbit_states(sd_ctx *ctx, const sd_state_vector *svs, uint64_t n, const int64_t *t_us,
                               uint64_t m, double *out) {
  if (!ctx) return SD_ERR_INVALID_ARGUMENT;
  if (!svs || (m && (!t_us || !out))) return set_error(ctx, SD_ERR_INVALID_ARGUMENT, "null argument");
  if (m == 0) return SD_OK;
  SD_CUDA(ctx, cudaSetDevice(ctx->device));
  const void *d_svs, *d_t;
  void *d_out;
  SD_TRY(stage_in(ctx, "orb.svs", svs, n * sizeof(sd_state_vector), &d_svs));
  SD_TRY(stage_in(ctx, "orb.t", t_us, m * sizeof(int64_t), &d_t));
  SD_TRY(stage_out(ctx, "orb.out", out, m * 9 * sizeof(double), &d_out));
  OrbitDev o{};
  o.svs = (const sd_state_vector *)d_svs;
  o.n = n;
  SD_TRY(upload_orbit_poly(ctx, "orb.poly", svs, n, &o));
  SD_CUDA(ctx, cudaMemsetAsync(ctx->d_flags, 0, sizeof(int), ctx->stream));
  SD_TIMED_BEGIN(ctx, "k_orbit_states");
  k_orbit_states<<<grid_for(m, 128), 128, 0, ctx->stream>>>(o, (const int64_t *)d_t, m, (double *)d_out,
                                                            ctx->d_flags);
  SD_LAUNCHED(ctx);
  int flag = 0;
  SD_CUDA(ctx, cudaMemcpyAsync(&flag, ctx->d_flags, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  SD_TRY(finish_out(ctx, out, d_out, m * 9 * sizeof(double)));
  SD_TRY(sync(ctx));
  if (flag)
    return set_error(ctx, SD_ERR_TC_ORBIT,
                     "orbit interpolation failed: interpolation time outside orbit window; refusing to extrapolate");
  return SD_OK;
}
