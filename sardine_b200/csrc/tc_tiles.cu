// tc_tiles.cu — device-resident scenes and batched tiles: any number of
// output windows over any resident scenes, geocoded by one persistent launch
// per stage (optionally replayed from a CUDA graph), then filtered and
// cropped (speckle.cu).
#include <mutex>

#include "tc_kernels.cuh"

namespace sd {
// this unit's bounds-check word (see runtime.cuh)
SD_BOUNDS_ACCESSOR(bounds_read_tiles)
}  // namespace sd

using namespace sd;

namespace sd {
namespace {

// Tile batches: the persistent work-table kernels; the resampler is read
// per job.  stages: the PX_* stages to launch (the others run per tile).
int launch_pixels_batch(sd_ctx *ctx, const TcWork *d_work, const uint64_t *totals, bool split,
                        unsigned stages = PX_ALL) {
  return split ? launch_pixels_t<KDYN, true>(ctx, d_work, totals, nullptr, stages)
               : launch_pixels_t<KDYN, false>(ctx, d_work, totals, nullptr, stages);
}

// One launch per tile over the side streams (largest tiles first, each to
// the least loaded stream), joined back into the context's stream; timed as
// `name`.  launch(i, stream) launches tile i's kernel.
template <class F>
int fork_per_tile(sd_ctx *ctx, const std::vector<TcDev> &jobs, const char *name, F launch) {
  for (int k = 0; k < SD_SIDE_STREAMS; ++k) {
    if (!ctx->side[k]) SD_CUDA(ctx, cudaStreamCreateWithFlags(&ctx->side[k], cudaStreamNonBlocking));
    if (!ctx->ev_join[k]) SD_CUDA(ctx, cudaEventCreateWithFlags(&ctx->ev_join[k], cudaEventDisableTiming));
  }
  if (!ctx->ev_fork) SD_CUDA(ctx, cudaEventCreateWithFlags(&ctx->ev_fork, cudaEventDisableTiming));
  const int ns = (int)std::min<size_t>(SD_SIDE_STREAMS, jobs.size());
  SD_TIMED_BEGIN(ctx, name);
  SD_CUDA(ctx, cudaEventRecord(ctx->ev_fork, ctx->stream));
  for (int k = 0; k < ns; ++k) SD_CUDA(ctx, cudaStreamWaitEvent(ctx->side[k], ctx->ev_fork, 0));
  std::vector<size_t> order(jobs.size());
  for (size_t i = 0; i < order.size(); ++i) order[i] = i;
  std::sort(order.begin(), order.end(),
            [&](size_t a, size_t b) { return jobs[a].rows * jobs[a].cols > jobs[b].rows * jobs[b].cols; });
  uint64_t load[SD_SIDE_STREAMS] = {};
  for (size_t i : order) {
    int k = 0;
    for (int q = 1; q < ns; ++q)
      if (load[q] < load[k]) k = q;
    SD_TRY(launch(i, ctx->side[k]));
    load[k] += jobs[i].rows * jobs[i].cols;
  }
  for (int k = 0; k < ns; ++k) {
    SD_CUDA(ctx, cudaEventRecord(ctx->ev_join[k], ctx->side[k]));
    SD_CUDA(ctx, cudaStreamWaitEvent(ctx->stream, ctx->ev_join[k], 0));
  }
  ::sd::timing_end(ctx);
  return SD_OK;
}

// k_main per tile in its parameter form (job record in the kernel's
// parameter space rather than in shared memory); small tiles overlap on
// the side streams.
int fork_main_per_tile(sd_ctx *ctx, const std::vector<TcDev> &jobs) {
  return fork_per_tile(ctx, jobs, "k_main (per tile)",
                       [&](size_t i, cudaStream_t s) { return launch_main_param(ctx, &jobs[i], s); });
}

// k_cand in its parameter form, one launch per tile, each specialised on
// the tile's resampling kernel.
int fork_cand_per_tile(sd_ctx *ctx, const std::vector<TcDev> &jobs, bool split) {
  return fork_per_tile(ctx, jobs, split ? "k_cand<SPLIT> (per tile)" : "k_cand (per tile)",
                       [&](size_t i, cudaStream_t s) {
                         return split ? launch_cand_param<true>(ctx, jobs[i], s)
                                      : launch_cand_param<false>(ctx, jobs[i], s);
                       });
}

// k_row_anchors in its parameter form, one launch per tile.
int fork_anchors_per_tile(sd_ctx *ctx, const std::vector<TcDev> &jobs) {
  return fork_per_tile(ctx, jobs, "k_row_anchors (per tile)",
                       [&](size_t i, cudaStream_t s) { return launch_anchors_param(ctx, jobs[i], s); });
}

// k_heights in its parameter form, one launch per tile (d_work: the batch's
// work table, whose deferral queue the tiles share).
int fork_heights_per_tile(sd_ctx *ctx, const std::vector<TcDev> &jobs, const TcWork *d_work) {
  return fork_per_tile(ctx, jobs, "k_heights (per tile)", [&](size_t i, cudaStream_t s) {
    return launch_heights_param(ctx, jobs[i], (int)i, d_work, s);
  });
}

}  // namespace
}  // namespace sd

// ── device-resident scenes and batched tiles ───────────────────────────────
// A scene keeps its radar image (and NESZ), DEM, geoid, state vectors, the
// azimuth-time LUT and an FP64 orbit table over the image's azimuth span in
// device memory; a batch of tiles (output windows of any size over any of
// the resident scenes) then runs as one launch per stage over a work table.

struct sd_scene_dev {
  int device = 0;
  std::vector<void *> owned;
  uint64_t bytes = 0;
  const float *img = nullptr, *nesz = nullptr;
  uint64_t lines = 0, samples = 0;
  int64_t az_start = 0;
  double ati = 0.0, near_range = 0.0, rps = 0.0;
  DemView dem{};
  const float *geoid = nullptr;
  const sd_state_vector *svs = nullptr;
  uint64_t nsv = 0;
  const double *lut_lat = nullptr;
  const int64_t *lut_t = nullptr;
  int lut_n = 0;
  OrbitDev orb{};
};

namespace sd {
namespace {

int scene_copy(sd_ctx *ctx, sd_scene_dev *s, const void *src, size_t bytes, const void **dst) {
  if (!src) {
    *dst = nullptr;
    return SD_OK;
  }
  if (is_device_ptr(src)) {  // borrowed: the caller keeps it alive
    *dst = src;
    return SD_OK;
  }
  void *d = nullptr;
  cudaError_t e = cudaMalloc(&d, bytes ? bytes : 16);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return set_error(ctx, SD_ERR_OUT_OF_MEMORY, "scene upload: cudaMalloc(%zu) failed: %s", bytes,
                     cudaGetErrorString(e));
  }
  s->owned.push_back(d);
  s->bytes += bytes;
  SD_CUDA(ctx, cudaMemcpyAsync(d, src, bytes, cudaMemcpyHostToDevice, ctx->stream));
  *dst = d;
  return SD_OK;
}

// build_azimuth_time_lut (terrain_correction.rs:1080-1104): stable sort by
// latitude, keep the first of near-duplicates.
void build_lut(const sd_geo_grid_point *grid, uint64_t n, std::vector<double> &lat, std::vector<int64_t> &t) {
  std::vector<std::pair<double, int64_t>> lut;
  for (uint64_t k = 0; k < n; ++k) lut.push_back({grid[k].latitude_deg, grid[k].azimuth_time_us});
  std::stable_sort(lut.begin(), lut.end(), [](auto &a, auto &b) { return a.first < b.first; });
  for (auto &pt : lut) {
    if (!lat.empty() && std::fabs(pt.first - lat.back()) < 1e-6) continue;
    lat.push_back(pt.first);
    t.push_back(pt.second);
  }
}

struct TilePlan {
  TcDev job;
  SpJob sp;
  int halo = 0;
  bool crop = false;  // the speckle/crop stage writes the final rasters
  void *user[3] = {nullptr, nullptr, nullptr};
  void *dev_final[3] = {nullptr, nullptr, nullptr};
  size_t final_bytes[3] = {0, 0, 0};
};

size_t al256(size_t x) { return (x + 255) & ~(size_t)255; }

// Runs `body` (a sequence of launches on ctx->stream) through a CUDA graph
// cached under `key`; the graph is re-captured when `tag` (the address of
// the work table it reads) changes.
template <class F>
int run_graph(sd_ctx *ctx, int key, const void *tag, F body) {
  auto &m = ctx->graph_exec;
  auto it = m.find(key);
  if (it != m.end() && it->second.tag != tag) {
    cudaGraphExecDestroy(it->second.exec);
    m.erase(it);
    it = m.end();
  }
  if (it == m.end()) {
    const uint64_t l0 = ctx->launches;
    SD_CUDA(ctx, cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
    int rc = body();
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamEndCapture(ctx->stream, &g);
    if (rc != SD_OK) {
      if (g) cudaGraphDestroy(g);
      return rc;
    }
    if (e != cudaSuccess) return set_error(ctx, SD_ERR_CUDA, "graph capture failed: %s", cudaGetErrorString(e));
    cudaGraphExec_t ex = nullptr;
    e = cudaGraphInstantiate(&ex, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) return set_error(ctx, SD_ERR_CUDA, "graph instantiate failed: %s", cudaGetErrorString(e));
    it = m.emplace(key, sd_ctx::GraphRec{ex, tag, ctx->launches - l0}).first;
    ctx->launches = l0;
  }
  SD_CUDA(ctx, cudaGraphLaunch(it->second.exec, ctx->stream));
  ctx->launches += it->second.launches;
  return SD_OK;
}

}  // namespace
}  // namespace sd

extern "C" int sd_scene_create(sd_ctx *ctx, const sd_radar_image *image, const sd_scene *scene,
                               const sd_dem *dem, const sd_geoid *geoid, const sd_geo_grid_point *grid,
                               uint64_t n_grid, sd_scene_dev **out) {
  SD_STAGE("scene_upload");
  if (!ctx) return SD_ERR_INVALID_ARGUMENT;
  if (!image || !scene || !dem || !geoid || !out || (n_grid && !grid))
    return set_error(ctx, SD_ERR_INVALID_ARGUMENT, "null argument");
  *out = nullptr;
  SD_CUDA(ctx, cudaSetDevice(ctx->device));
  if (n_grid == 0) return set_error(ctx, SD_ERR_TC_NO_GRID_POINTS, "no geolocation grid points provided");
  if (scene->n_sub_swaths <= 0)
    return set_error(ctx, SD_ERR_TC_NO_SUBSWATHS, "scene has no subswaths — cannot derive radar geometry");
  const double ati = scene->azimuth_time_interval_s;
  if (!std::isfinite(ati) || ati <= 0.0)
    return set_error(ctx, SD_ERR_TC_CONFIG, "invalid azimuth_time_interval_s in subswath metadata: %g", ati);
  if (dem->width < 2 || dem->height < 2 || !(dem->pixel_size > 0.0) || !dem->data)
    return set_error(ctx, SD_ERR_INVALID_ARGUMENT, "DEM grid must be at least 2x2 with positive spacing");
  if (image->lines == 0 || image->samples == 0 || !image->data)
    return set_error(ctx, SD_ERR_INVALID_ARGUMENT, "radar image is empty");
  if (dem->kind == SD_DEM_PROJECTED_UTM && (dem->utm_zone < 1 || dem->utm_zone > 60))
    return set_error(ctx, SD_ERR_TC_DEM, "projected DEM needs a UTM zone in 1..60");
  if (geoid->kind == SD_GEOID_GRID && !geoid->undulations_m)
    return set_error(ctx, SD_ERR_INVALID_ARGUMENT, "geoid grid is null");
  if (!scene->state_vectors || scene->n_state_vectors == 0)
    return set_error(ctx, SD_ERR_TC_ORBIT, "orbit has no state vectors");
  std::vector<double> lut_lat;
  std::vector<int64_t> lut_t;
  build_lut(grid, n_grid, lut_lat, lut_t);
  if (lut_lat.empty()) return set_error(ctx, SD_ERR_TC_NO_GRID_POINTS, "no geolocation grid points provided");

  std::unique_ptr<sd_scene_dev> s(new sd_scene_dev);
  s->device = ctx->device;
  const void *d;
  const size_t img_bytes = image->lines * image->samples * sizeof(float);
  SD_TRY(scene_copy(ctx, s.get(), image->data, img_bytes, &d));
  s->img = (const float *)d;
  SD_TRY(scene_copy(ctx, s.get(), image->nesz, img_bytes, &d));
  s->nesz = (const float *)d;
  SD_TRY(scene_copy(ctx, s.get(), dem->data, dem->width * dem->height * sizeof(float), &d));
  s->dem.data = (const float *)d;
  s->dem.width = dem->width;
  s->dem.height = dem->height;
  s->dem.origin_y = dem->origin_y;
  s->dem.origin_x = dem->origin_x;
  s->dem.pixel_size = dem->pixel_size;
  s->dem.inv_ps = 1.0 / dem->pixel_size;
  s->dem.kind = dem->kind;
  if (dem->kind == SD_DEM_PROJECTED_UTM) s->dem.utm = make_utm(dem->utm_zone, dem->utm_south != 0);
  if (geoid->kind == SD_GEOID_GRID) {
    SD_TRY(scene_copy(ctx, s.get(), geoid->undulations_m, 73 * 144 * sizeof(float), &d));
    s->geoid = (const float *)d;
  }
  const uint64_t nsv = scene->n_state_vectors;
  SD_TRY(scene_copy(ctx, s.get(), scene->state_vectors, nsv * sizeof(sd_state_vector), &d));
  s->svs = (const sd_state_vector *)d;
  s->nsv = nsv;
  SD_TRY(scene_copy(ctx, s.get(), lut_lat.data(), lut_lat.size() * 8, &d));
  s->lut_lat = (const double *)d;
  SD_TRY(scene_copy(ctx, s.get(), lut_t.data(), lut_t.size() * 8, &d));
  s->lut_t = (const int64_t *)d;
  s->lut_n = (int)lut_lat.size();
  s->lines = image->lines;
  s->samples = image->samples;
  s->az_start = image->azimuth_start_time_us;
  s->ati = ati;
  s->near_range = image->near_slant_range_time_s * SPEED_OF_LIGHT / 2.0;
  s->rps = image->range_pixel_spacing_m;
  s->orb.svs = s->svs;
  s->orb.n = nsv;
  // the orbit as window polynomials (a few KB; used outside the table)
  if (nsv >= 8) {
    std::vector<OrbPoly> w(nsv - 7);
    orbit_poly_build(scene->state_vectors, nsv, w.data());
    SD_TRY(scene_copy(ctx, s.get(), w.data(), w.size() * sizeof(OrbPoly), &d));
    s->orb.poly = (const OrbPoly *)d;
  }
  // orbit table over the image's azimuth span +-0.2 s, inside the SV window
  if (nsv >= 8) {
    int64_t t0 = std::max(scene->state_vectors[0].time_us, s->az_start - 200000);
    int64_t t1 = std::min(scene->state_vectors[nsv - 1].time_us,
                          s->az_start + (int64_t)std::llround((double)s->lines * ati * 1e6) + 200000);
    const int64_t max_entries = 96ll * 1000 * 1000;
    if (t1 - t0 + 1 > max_entries) t1 = t0 + max_entries - 1;
    if (t1 >= t0) {
      const size_t n = (size_t)(t1 - t0 + 1);
      void *tab = nullptr;
      cudaError_t e = cudaMalloc(&tab, n * 5 * sizeof(double2));
      if (e != cudaSuccess) {
        cudaGetLastError();
        return set_error(ctx, SD_ERR_OUT_OF_MEMORY, "scene orbit table: cudaMalloc failed");
      }
      s->owned.push_back(tab);
      s->bytes += n * 5 * sizeof(double2);
      SD_TIMED_BEGIN(ctx, "k_orbit_table");
      k_orbit_table<<<grid_for(n, 128), 128, 0, ctx->stream>>>(s->svs, nsv, t0, (int64_t)n, (double2 *)tab);
      SD_LAUNCHED(ctx);
      s->orb.tab = (const double2 *)tab;
      s->orb.tab_t0 = t0;
      s->orb.tab_n = (int64_t)n;
      const size_t tay_bytes = (size_t)tay_count(s->orb.tab_n) * sizeof(OrbTaylor);
      void *tay = nullptr;
      e = cudaMalloc(&tay, tay_bytes);
      if (e != cudaSuccess) {
        cudaGetLastError();
        return set_error(ctx, SD_ERR_OUT_OF_MEMORY, "scene orbit expansions: cudaMalloc failed");
      }
      s->owned.push_back(tay);
      s->bytes += tay_bytes;
      SD_TRY(launch_orbit_taylor(ctx, &s->orb, (OrbTaylor *)tay));
    }
  }
  SD_TRY(sync(ctx));
  *out = s.release();
  return SD_OK;
}

extern "C" void sd_scene_destroy(sd_scene_dev *s) {
  if (!s) return;
  cudaSetDevice(s->device);
  for (void *p : s->owned) cudaFree(p);
  delete s;
}

extern "C" uint64_t sd_scene_device_bytes(const sd_scene_dev *s) { return s ? s->bytes : 0; }

namespace sd {
namespace {

// Validates tile i and fills its plan (grid, configuration, halo); device
// pointers are assigned later.
int tile_plan(sd_ctx *ctx, const sd_tile &t, uint64_t i, TilePlan *pl) {
  const sd_tc_config &cfg = t.cfg;
  if (!t.scene) return set_error(ctx, SD_ERR_INVALID_ARGUMENT, "tile %llu: no scene", (unsigned long long)i);
  if (t.scene->device != ctx->device)
    return set_error(ctx, SD_ERR_INVALID_ARGUMENT, "tile %llu: scene lives on another device", (unsigned long long)i);
  if (!t.out_data) return set_error(ctx, SD_ERR_INVALID_ARGUMENT, "tile %llu: null output", (unsigned long long)i);
  if (cfg.compute_lia && (!t.out_cos_lia || !t.out_mask))
    return set_error(ctx, SD_ERR_INVALID_ARGUMENT, "tile %llu: compute_lia needs cos_lia and mask buffers",
                     (unsigned long long)i);
  if (!(cfg.pixel_spacing > 0.0))
    return set_error(ctx, SD_ERR_TC_CONFIG, "tile %llu: pixel spacing must be positive", (unsigned long long)i);
  if (t.rows == 0 || t.cols == 0)
    return set_error(ctx, SD_ERR_TC_CONFIG, "tile %llu: empty output grid", (unsigned long long)i);
  if (cfg.precision != SD_PRECISION_FP64 && cfg.precision != SD_PRECISION_SPLIT)
    return set_error(ctx, SD_ERR_TC_CONFIG, "tile %llu: unknown precision mode %d", (unsigned long long)i,
                     cfg.precision);
  if (cfg.crs != SD_CRS_WGS84 && cfg.crs != SD_CRS_UTM_NORTH && cfg.crs != SD_CRS_UTM_SOUTH)
    return set_error(ctx, SD_ERR_TC_PROJECTION, "tile %llu: unknown CRS", (unsigned long long)i);
  if (cfg.crs != SD_CRS_WGS84 && (cfg.utm_zone < 1 || cfg.utm_zone > 60))
    return set_error(ctx, SD_ERR_TC_PROJECTION, "tile %llu: UTM zone must be 1..60", (unsigned long long)i);
  if (cfg.crs != SD_CRS_WGS84 && cfg.projector_anchors <= 0)
    return set_error(ctx, SD_ERR_TC_CONFIG, "SARDINE_TC_PROJECTOR_ANCHORS must be >= 1 (default 256)");
  if (t.speckle >= 0) {
    int rc = speckle_validate(1, 1, 1, t.speckle, (uint64_t)t.speckle_window, t.enl, t.damping);
    if (rc != SD_OK)
      return set_error(ctx, rc, "tile %llu: invalid speckle filter parameters", (unsigned long long)i);
  } else if (t.speckle != -1) {
    return set_error(ctx, SD_ERR_INVALID_ARGUMENT, "tile %llu: speckle must be -1 or SD_SPECKLE_*",
                     (unsigned long long)i);
  }
  speckle_coefs(t.speckle, (uint64_t)t.speckle_window, t.enl, t.damping, &pl->sp);
  if (pl->sp.half > SP_MAX_HALF)
    return set_error(ctx, SD_ERR_SPECKLE_BAD_WINDOW, "tile %llu: speckle window above %d",
                     (unsigned long long)i, 2 * SP_MAX_HALF + 1);
  const sd_scene_dev &s = *t.scene;
  pl->halo = pl->sp.half;
  const uint64_t rows = t.rows + 2 * (uint64_t)pl->halo, cols = t.cols + 2 * (uint64_t)pl->halo;
  TcDev &p = pl->job;
  std::memset(&p, 0, sizeof p);
  p.rows = rows;
  p.cols = cols;
  p.sp = cfg.pixel_spacing;
  p.lat_north = t.origin_y + (double)pl->halo * p.sp;
  p.lon_west = t.origin_x - (double)pl->halo * p.sp;
  p.utm = cfg.crs != SD_CRS_WGS84;
  if (p.utm) p.proj = make_utm(cfg.utm_zone, cfg.crs == SD_CRS_UTM_SOUTH);
  p.step_deg = p.utm ? p.sp / 111320.0 : p.sp;
  if (p.utm) {
    p.n_anchors = (int)std::min<uint64_t>((uint64_t)cfg.projector_anchors, cols);
    p.n_pts = p.n_anchors + 1;
  }
  p.lut_lat = s.lut_lat;
  p.lut_t = s.lut_t;
  p.lut_n = s.lut_n;
  p.orb = s.orb;
  p.dem = s.dem;
  p.geoid = s.geoid;
  p.img = s.img;
  p.lines = s.lines;
  p.samples = s.samples;
  p.az_start = s.az_start;
  p.ati = s.ati;
  p.near_range = s.near_range;
  p.rps = s.rps;
  p.max_iter = cfg.max_newton_iterations < 0 ? 0 : cfg.max_newton_iterations;
  p.tol = cfg.newton_tolerance_s;
  p.flatten = cfg.flatten != 0;
  p.compute_lia = cfg.compute_lia != 0;
  p.need_geom = p.flatten || p.compute_lia;
  p.resampling = cfg.resampling;
  p.nesz_mask = std::isfinite(cfg.noise_floor_margin_db) && s.nesz != nullptr;
  p.nesz = p.nesz_mask ? s.nesz : nullptr;
  p.nesz_factor = p.nesz_mask ? std::pow(10.0f, cfg.noise_floor_margin_db / 10.0f) : 0.0f;
  p.fast = (p.tol <= 1e-6) ? 1 : 0;
  set_main_segments(&p);
  pl->crop = pl->halo > 0 || t.speckle >= 0;
  pl->user[0] = t.out_data;
  pl->user[1] = p.compute_lia ? t.out_cos_lia : nullptr;
  pl->user[2] = p.compute_lia ? t.out_mask : nullptr;
  const size_t npx = t.rows * t.cols;
  pl->final_bytes[0] = npx * 4;
  pl->final_bytes[1] = p.compute_lia ? npx * 4 : 0;
  pl->final_bytes[2] = p.compute_lia ? npx : 0;
  return SD_OK;
}

}  // namespace
}  // namespace sd

extern "C" int sd_tc_tiles_launch(sd_ctx *ctx, const sd_tile *tiles, uint64_t n) {
  SD_STAGE("terrain_correction_tiles");
  if (!ctx) return SD_ERR_INVALID_ARGUMENT;
  if (ctx->tiles_pending)
    return set_error(ctx, SD_ERR_BUSY, "the previous tile batch has not been collected (sd_tc_tiles_finish)");
  if (n == 0) return set_error(ctx, SD_ERR_INVALID_ARGUMENT, "empty tile batch");
  if (!tiles) return set_error(ctx, SD_ERR_INVALID_ARGUMENT, "null tiles");
  if (n > (1u << 20)) return set_error(ctx, SD_ERR_INVALID_ARGUMENT, "too many tiles in one batch");
  SD_CUDA(ctx, cudaSetDevice(ctx->device));
  cudaStream_t st = ctx->stream;
  std::vector<TilePlan> plans(n);
  for (uint64_t i = 0; i < n; ++i) SD_TRY(tile_plan(ctx, tiles[i], i, &plans[i]));

  // ── arena: per-row, per-pixel and staging buffers of every tile ──
  size_t cur = 0;
  auto take = [&](size_t bytes) {
    size_t o = cur;
    cur += al256(bytes ? bytes : 1);
    return o;
  };
  struct Offs {
    size_t guess, flat, knots, alon, alat, aloc, tp, fct, fb, cc, sel, rscnt, rsent, hout[3], fin[3];
  };
  std::vector<Offs> of(n);
  size_t ax_total = 0;
  for (uint64_t i = 0; i < n; ++i) {
    const TcDev &p = plans[i].job;
    const size_t npx = p.rows * p.cols;
    Offs &o = of[i];
    o.guess = take(p.rows * 8);
    o.flat = take(p.rows * 8);
    o.knots = take(p.rows * KNOTS * 8);
    o.alon = o.alat = o.aloc = SIZE_MAX;
    if (p.utm) {
      o.alon = take(p.rows * p.n_pts * 8);
      o.alat = take(p.rows * p.n_pts * 8);
      if (p.dem.kind == SD_DEM_PROJECTED_UTM) o.aloc = take(p.rows * p.n_pts * sizeof(UtmLocal));
      ax_total += p.n_pts;
    }
    o.tp = take(3 * npx * sizeof(double));
    o.fct = p.need_geom ? take(4 * npx * sizeof(double)) : SIZE_MAX;
    o.fb = take(npx * sizeof(int64_t));
    o.cc = take(npx * 4);
    o.sel = take(npx);
    o.rscnt = o.rsent = SIZE_MAX;
    if (tiles[i].cfg.precision == SD_PRECISION_SPLIT) {
      o.rscnt = take(stage_items(WK_SEL, p) * 4);
      o.rsent = take(stage_items(WK_SEL, p) * RS_CAP * sizeof(RsEnt));
    }
    for (int k = 0; k < 3; ++k) {
      o.hout[k] = o.fin[k] = SIZE_MAX;
      const size_t esz = k == 2 ? 1 : 4;
      if (plans[i].final_bytes[k] == 0) continue;
      if (plans[i].crop) o.hout[k] = take(npx * esz);
      if (!is_device_ptr(plans[i].user[k])) o.fin[k] = take(plans[i].final_bytes[k]);
    }
  }
  unsigned char *arena = nullptr;
  SD_TRY(scratch_t(ctx, "tiles.arena", cur, &arena));
  double *d_ax = nullptr;
  SD_TRY(scratch_t(ctx, "tiles.ax", std::max<size_t>(ax_total, 1), &d_ax));
  unsigned long long *d_cnt = nullptr;
  int *d_flg = nullptr;
  SD_TRY(scratch_t(ctx, "tiles.counters", n * 32, &d_cnt));
  SD_TRY(scratch_t(ctx, "tiles.flags", n * 8, &d_flg));
  if (ctx->tile_cap < n) {
    if (ctx->h_tile_counters) cudaFreeHost(ctx->h_tile_counters);
    if (ctx->h_tile_flags) cudaFreeHost(ctx->h_tile_flags);
    ctx->h_tile_counters = nullptr;
    ctx->h_tile_flags = nullptr;
    ctx->tile_cap = 0;
    SD_CUDA(ctx, cudaHostAlloc((void **)&ctx->h_tile_counters, n * 32 * 8, cudaHostAllocDefault));
    SD_CUDA(ctx, cudaHostAlloc((void **)&ctx->h_tile_flags, n * 8 * 4, cudaHostAllocDefault));
    ctx->tile_cap = n;
  }
  if (!ctx->tiles_done) SD_CUDA(ctx, cudaEventCreateWithFlags(&ctx->tiles_done, cudaEventDisableTiming));

  // ── job records ──
  std::vector<double> ax_h;
  ax_h.reserve(ax_total);
  std::vector<TcDev> grp[2];
  std::vector<SpJob> spj;
  for (uint64_t i = 0; i < n; ++i) {
    TilePlan &pl = plans[i];
    TcDev &p = pl.job;
    const Offs &o = of[i];
    p.row_guess = (int64_t *)(arena + o.guess);
    p.row_flat = (double *)(arena + o.flat);
    p.knot_t = (int64_t *)(arena + o.knots);
    if (p.utm) {
      const double x_start = p.lon_west + 0.5 * p.sp;
      const double x_end = x_start + ((double)p.cols - 1.0) * p.sp;
      const double anchor_dx = (x_end - x_start) / (double)p.n_anchors;
      p.ax = d_ax + ax_h.size();
      for (int a = 0; a <= p.n_anchors; ++a) ax_h.push_back(x_start + (double)a * anchor_dx);
      p.alon = (const double *)(arena + o.alon);
      p.alat = (const double *)(arena + o.alat);
      p.aloc = o.aloc != SIZE_MAX ? (const UtmLocal *)(arena + o.aloc) : nullptr;
    }
    p.tp = (const double *)(arena + o.tp);
    p.fct = o.fct != SIZE_MAX ? (const double *)(arena + o.fct) : nullptr;
    p.fb = (int64_t *)(arena + o.fb);
    p.cc = (uint32_t *)(arena + o.cc);
    p.sel = (uint8_t *)(arena + o.sel);
    p.rs_cnt = o.rscnt != SIZE_MAX ? (uint32_t *)(arena + o.rscnt) : nullptr;
    p.rs_ent = o.rsent != SIZE_MAX ? (RsEnt *)(arena + o.rsent) : nullptr;
    for (int k = 0; k < 3; ++k) {
      if (pl.final_bytes[k] == 0) continue;
      pl.dev_final[k] = o.fin[k] != SIZE_MAX ? (void *)(arena + o.fin[k]) : pl.user[k];
    }
    void *tc_out[3];
    for (int k = 0; k < 3; ++k)
      tc_out[k] = pl.final_bytes[k] == 0 ? nullptr : (pl.crop ? (void *)(arena + o.hout[k]) : pl.dev_final[k]);
    p.out = (float *)tc_out[0];
    p.cos_lia = (float *)tc_out[1];
    p.mask = (uint8_t *)tc_out[2];
    p.az_time = nullptr;
    p.counters = d_cnt + 32 * i;
    p.flags = d_flg + 8 * i;
    p.trange = nullptr;
    const int g = tiles[i].cfg.precision == SD_PRECISION_SPLIT ? 1 : 0;
    p.split = g;
    grp[g].push_back(p);
    if (pl.crop) {
      SpJob j = pl.sp;
      j.in = p.out;
      j.cos_in = p.cos_lia;
      j.mask_in = p.mask;
      j.out = (float *)pl.dev_final[0];
      j.cos_out = (float *)pl.dev_final[1];
      j.mask_out = (uint8_t *)pl.dev_final[2];
      j.rows = (int64_t)tiles[i].rows;
      j.cols = (int64_t)tiles[i].cols;
      j.halo = pl.halo;
      spj.push_back(j);
    }
  }
  if (!ax_h.empty())
    SD_CUDA(ctx, cudaMemcpyAsync(d_ax, ax_h.data(), ax_h.size() * 8, cudaMemcpyHostToDevice, st));

  // ── stages: one launch each over all tiles of a precision group ──
  const bool use_graph = ctx->graphs && !ctx->timing;
  for (int g = 0; g < 2; ++g) {
    if (grp[g].empty()) continue;
    const char *wname = g ? "tiles.work1" : "tiles.work0";
    TcWorkHost wk;
    TcWork *d_work = nullptr;
    // in graph mode the table keeps one address for up to 1024 jobs
    if (use_graph && grp[g].size() < 1024) {
      void *tmp = nullptr;
      SD_TRY(scratch(ctx, wname, work_bytes(1024), &tmp));
    }
    SD_TRY(work_upload(ctx, wname, grp[g].data(), (int)grp[g].size(), &wk, &d_work));
    const bool split = g == 1;
    if (ctx->main_cps < 0) {  // per-tile parameter launches of k_heights and k_main
      const bool hp = heights_param_enabled(), ap = anchors_param_enabled() && wk.totals[WK_ANCH];
      if (ap) SD_TRY(fork_anchors_per_tile(ctx, grp[g]));
      SD_TRY(launch_rows(ctx, d_work, wk.totals, nullptr, !hp, !ap));
      if (hp) {
        SD_TRY(fork_heights_per_tile(ctx, grp[g], d_work));
        SD_TRY(launch_heights_fix(ctx, d_work, wk.totals));
      }
      SD_TRY(fork_main_per_tile(ctx, grp[g]));
      if (cand_param_enabled()) {
        SD_TRY(launch_pixels_batch(ctx, d_work, wk.totals, split, PX_SCAN));
        SD_TRY(fork_cand_per_tile(ctx, grp[g], split));
        SD_TRY(launch_pixels_batch(ctx, d_work, wk.totals, split, PX_POST));
      } else {
        SD_TRY(launch_pixels_batch(ctx, d_work, wk.totals, split, PX_ALL & ~PX_MAIN));
      }
    } else if (use_graph) {
      static const uint64_t kFull[kWk] = {~0ull, ~0ull, ~0ull, ~0ull, ~0ull, ~0ull, ~0ull};
      SD_TRY(run_graph(ctx, g + 2 * ctx->main_cps, d_work, [&]() -> int {
        SD_TRY(launch_rows(ctx, d_work, kFull));
        return launch_pixels_batch(ctx, d_work, kFull, split);
      }));
    } else {
      SD_TRY(launch_rows(ctx, d_work, wk.totals));
      SD_TRY(launch_pixels_batch(ctx, d_work, wk.totals, split));
    }
  }
  if (!spj.empty()) {
    // SpWork | SpJob[m] | pre[m + 1]
    const size_t m = spj.size();
    const size_t o_jobs = 64, o_pre = o_jobs + al256(m * sizeof(SpJob));
    size_t bytes = o_pre + (m + 1) * 8;
    if (use_graph) bytes = std::max(bytes, o_jobs + al256(1024 * sizeof(SpJob)) + 1025 * 8);
    unsigned char *d_sw = nullptr;
    SD_TRY(scratch_t(ctx, "tiles.spwork", bytes, &d_sw));
    std::vector<unsigned char> h(o_pre + (m + 1) * 8);
    const int tx = ctx->sp_tx, ty = ctx->sp_ty;
    SpWork w{};
    w.n_jobs = (int)m;
    w.tx = tx;
    w.ty = ty;
    w.jobs = (const SpJob *)(d_sw + o_jobs);
    w.pre = (const uint64_t *)(d_sw + o_pre);
    std::memcpy(h.data(), &w, sizeof w);
    std::memcpy(h.data() + o_jobs, spj.data(), m * sizeof(SpJob));
    uint64_t *pre = (uint64_t *)(h.data() + o_pre), acc = 0;
    for (size_t j = 0; j < m; ++j) {
      pre[j] = acc;
      acc += speckle_tile_items(spj[j], tx, ty);
    }
    pre[m] = acc;
    SD_CUDA(ctx, cudaMemcpyAsync(d_sw, h.data(), h.size(), cudaMemcpyHostToDevice, st));
    if (use_graph && m < 1024) {
      SD_TRY(run_graph(ctx, 1 << 20 | tx << 10 | ty, d_sw, [&]() -> int {
        return speckle_tiles_launch(ctx, (const SpWork *)d_sw, acc, true, tx, ty);
      }));
    } else {
      SD_TRY(speckle_tiles_launch(ctx, (const SpWork *)d_sw, acc, false, tx, ty));
    }
  }
  // ── results to the caller's host buffers, counters to pinned memory ──
  for (uint64_t i = 0; i < n; ++i)
    for (int k = 0; k < 3; ++k)
      if (plans[i].final_bytes[k] && plans[i].dev_final[k] != plans[i].user[k])
        SD_CUDA(ctx, cudaMemcpyAsync(plans[i].user[k], plans[i].dev_final[k], plans[i].final_bytes[k],
                                     cudaMemcpyDeviceToHost, st));
  SD_CUDA(ctx, cudaMemcpyAsync(ctx->h_tile_counters, d_cnt, n * 32 * 8, cudaMemcpyDeviceToHost, st));
  SD_CUDA(ctx, cudaMemcpyAsync(ctx->h_tile_flags, d_flg, n * 8 * 4, cudaMemcpyDeviceToHost, st));
  SD_CUDA(ctx, cudaEventRecord(ctx->tiles_done, st));
  ctx->tile_info.assign(n, sd_geocoded_info{});
  for (uint64_t i = 0; i < n; ++i) {
    sd_geocoded_info &f = ctx->tile_info[i];
    f.rows = tiles[i].rows;
    f.cols = tiles[i].cols;
    f.origin_lat_deg = tiles[i].origin_y;
    f.origin_lon_deg = tiles[i].origin_x;
    f.pixel_spacing = tiles[i].cfg.pixel_spacing;
    f.geotransform[0] = tiles[i].origin_x;
    f.geotransform[1] = tiles[i].cfg.pixel_spacing;
    f.geotransform[3] = tiles[i].origin_y;
    f.geotransform[5] = -tiles[i].cfg.pixel_spacing;
    f.total_pixel_count = tiles[i].rows * tiles[i].cols;
  }
  ctx->tile_n = n;
  ctx->tiles_pending = true;
  return SD_OK;
}

extern "C" int sd_tc_tiles_copy_out(sd_ctx *ctx, void *host_dst, const void *dev_src, uint64_t bytes) {
  if (!ctx) return SD_ERR_INVALID_ARGUMENT;
  if (!ctx->tiles_pending) return set_error(ctx, SD_ERR_INVALID_ARGUMENT, "no tile batch in flight");
  if (bytes == 0) return SD_OK;
  if (!host_dst || !dev_src) return set_error(ctx, SD_ERR_INVALID_ARGUMENT, "null buffer");
  SD_CUDA(ctx, cudaSetDevice(ctx->device));
  // behind the batch's kernels on its stream; the batch completes after it
  SD_CUDA(ctx, cudaMemcpyAsync(host_dst, dev_src, bytes, cudaMemcpyDeviceToHost, ctx->stream));
  SD_CUDA(ctx, cudaEventRecord(ctx->tiles_done, ctx->stream));
  return SD_OK;
}

extern "C" int sd_tc_tiles_poll(sd_ctx *ctx) {
  if (!ctx) return SD_ERR_INVALID_ARGUMENT;
  if (!ctx->tiles_pending) return SD_OK;
  cudaError_t e = cudaEventQuery(ctx->tiles_done);
  if (e == cudaSuccess) return SD_OK;
  if (e == cudaErrorNotReady) return SD_ERR_BUSY;
  return set_error(ctx, SD_ERR_CUDA, "tile batch failed: %s", cudaGetErrorString(e));
}

extern "C" int sd_tc_tiles_finish(sd_ctx *ctx, sd_geocoded_info *infos, uint64_t n) {
  if (!ctx) return SD_ERR_INVALID_ARGUMENT;
  if (!ctx->tiles_pending) return set_error(ctx, SD_ERR_INVALID_ARGUMENT, "no tile batch in flight");
  if (n != ctx->tile_n || (n && !infos))
    return set_error(ctx, SD_ERR_INVALID_ARGUMENT, "infos must hold the %llu tiles of the batch",
                     (unsigned long long)ctx->tile_n);
  ctx->tiles_pending = false;
  SD_CUDA(ctx, cudaEventSynchronize(ctx->tiles_done));
  SD_TRY(sync(ctx));
  int orbit_bad = -1;
  bool internal_bad = false;
  for (uint64_t i = 0; i < n; ++i) {
    sd_geocoded_info f = ctx->tile_info[i];
    const unsigned long long *c = ctx->h_tile_counters + 32 * i;
    f.valid_pixel_count = c[0];
    f.dem_missing_count = c[1];
    f.outside_footprint_count = c[2];
    f.non_converged_count = c[3];
    f.degenerate_geometry_count = c[4];
    f.flat_masked_count = c[5];
    f.noise_masked_count = c[6];
    for (int k = 0; k < SD_NEWTON_ITER_HIST_SIZE; ++k) f.newton_iter_histogram[k] = c[kCounters + k];
    f.diag_exact_path_pixels = (uint64_t)ctx->h_tile_flags[8 * i + 1];
    f.diag_fp64_redo_pixels = (uint64_t)ctx->h_tile_flags[8 * i + 2];
    f.diag_fp64_resampled = (uint64_t)ctx->h_tile_flags[8 * i + 4];
    if (ctx->h_tile_flags[8 * i] && orbit_bad < 0) orbit_bad = (int)i;
    if (ctx->h_tile_flags[8 * i + 5]) internal_bad = true;
    infos[i] = f;
  }
  if (internal_bad) return set_error(ctx, SD_ERR_INTERNAL, "tiles: a converged pixel lost its DEM height");
  if (orbit_bad >= 0)
    return set_error(ctx, SD_ERR_TC_ORBIT,
                     "tile %d: orbit interpolation failed: interpolation time outside orbit window; "
                     "refusing to extrapolate",
                     orbit_bad);
  return SD_OK;
}

extern "C" int sd_tc_tiles(sd_ctx *ctx, const sd_tile *tiles, uint64_t n, sd_geocoded_info *infos) {
  SD_STAGE("terrain_correction_tiles");
  SD_TRY(sd_tc_tiles_launch(ctx, tiles, n));
  return sd_tc_tiles_finish(ctx, infos, n);
}

extern "C" int sd_ctx_set_graphs(sd_ctx *ctx, int enable) {
  if (!ctx) return SD_ERR_INVALID_ARGUMENT;
  ctx->graphs = enable != 0;
  return SD_OK;
}

extern "C" int sd_ctx_reserve(sd_ctx *ctx, uint64_t tile_arena_bytes) {
  if (!ctx) return SD_ERR_INVALID_ARGUMENT;
  SD_CUDA(ctx, cudaSetDevice(ctx->device));
  // the arena plus the per-batch tables at their largest graph-mode size
  void *p = nullptr;
  SD_TRY(scratch(ctx, "tiles.arena", tile_arena_bytes, &p));
  SD_TRY(scratch(ctx, "tiles.work0", work_bytes(1024), &p));
  SD_TRY(scratch(ctx, "tiles.work1", work_bytes(1024), &p));
  SD_TRY(scratch(ctx, "tiles.spwork", 64 + al256(1024 * sizeof(SpJob)) + 1025 * 8, &p));
  SD_TRY(scratch(ctx, "tiles.counters", 1024 * 32 * 8, &p));
  SD_TRY(scratch(ctx, "tiles.flags", 1024 * 8 * 4, &p));
  SD_TRY(scratch(ctx, "tiles.ax", 1024 * 257 * 8, &p));
  // k_heights' deferral queues at the capacity work_upload asks for a batch
  // that fills the arena (a tile pixel takes at least 37 arena bytes), so an
  // admitted batch never regrows them (a regrow frees memory, which
  // synchronises the device and would stall the other contexts' batches)
  SD_TRY(scratch(ctx, "tiles.work0.hq", heights_queue_bytes(tile_arena_bytes / 37), &p));
  SD_TRY(scratch(ctx, "tiles.work1.hq", heights_queue_bytes(tile_arena_bytes / 37), &p));
  return SD_OK;
}

extern "C" int sd_ctx_set_tile_shape(sd_ctx *ctx, int32_t speckle_tx, int32_t speckle_ty,
                                     int32_t main_ctas_per_sm) {
  if (!ctx) return SD_ERR_INVALID_ARGUMENT;
  if (!speckle_shape_ok(speckle_tx, speckle_ty))
    return set_error(ctx, SD_ERR_INVALID_ARGUMENT, "speckle block %dx%d: need tx >= 8, tx*ty <= 1024, tx*ty %% 32 == 0",
                     speckle_tx, speckle_ty);
  if (main_ctas_per_sm < -1 || main_ctas_per_sm > 64)
    return set_error(ctx, SD_ERR_INVALID_ARGUMENT, "main_ctas_per_sm must be -1..64");
  ctx->sp_tx = speckle_tx;
  ctx->sp_ty = speckle_ty;
  ctx->main_cps = main_ctas_per_sm;
  return SD_OK;
}
