// Output path: dB conversion with the run's dB statistics, the overview
// pyramid and tiles of a Cloud-Optimised GeoTIFF.
//
//   sd_to_db          to_db_inplace (export.rs:59-99) fused with
//                     compute_db_stats (run.rs:63-97)
//   sd_downsample_2x  downsample_2x (export.rs:362-392)
//   sd_write_cog      write_cog_with_crs / write_cog_raw_inner
//                     (export.rs:329-355, 417-760), GeoKeys from
//                     geo_key_directory (output_crs.rs:265-287)
//
// All three are HBM-bound passes: one read and one write per pixel (the dB
// pass), 4 reads and 1 write per overview pixel, 1 read and 1 padded write
// per tile pixel.  The file itself is written by the host from pinned
// buffers while the next tiles are packed and copied.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>

#include "runtime.cuh"

namespace sd {
namespace {

constexpr int DB_THREADS = 256;
constexpr int DB_PER_THREAD = 16;
constexpr int DB_CHUNK = DB_THREADS * DB_PER_THREAD;  // elements per block, element e = k * 256 + tid

// Per-block partials of the dB pass (one entry per DB_CHUNK elements).
struct DbPart {
  double sum;       // f64 sum of the finite dB values
  float mn, mx;     // their min and max
  uint32_t cnt;     // number of finite dB values
  uint32_t cv, nm;  // converted and noise-masked elements
  uint32_t pad;
};

__device__ __forceinline__ double warp_sum_d(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// to_db_inplace on one DB_CHUNK per block (NaN kept; v <= floor -> NaN and
// counted as noise-masked; else 10 log10 v), with the block's statistics of
// the finite results.
// CONVERT false: the statistics of a raster already in dB (read only).
template <bool CONVERT>
__global__ void __launch_bounds__(DB_THREADS) k_to_db(float *__restrict__ d, uint64_t n, float floor_lin,
                                                      DbPart *__restrict__ part) {
  __shared__ double s_sum[DB_THREADS / 32];
  __shared__ float s_mn[DB_THREADS / 32], s_mx[DB_THREADS / 32];
  __shared__ uint32_t s_cnt[DB_THREADS / 32], s_cv[DB_THREADS / 32], s_nm[DB_THREADS / 32];
  const uint64_t base = (uint64_t)blockIdx.x * DB_CHUNK;
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  uint32_t cv = 0, nm = 0, cnt = 0;
  double sum = 0.0;
  float mn = INFINITY, mx = -INFINITY;
  // element of slot k: base + 4 (g DB_THREADS + tid) + j with g = k / 4,
  // j = k % 4, so a thread's four consecutive elements are one 16-byte word
  // (128-bit loads and stores when the raster is 16-byte aligned)
  constexpr int G = DB_PER_THREAD / 4;
  const bool vec = (reinterpret_cast<uintptr_t>(d) & 15) == 0;
  float x[DB_PER_THREAD];
#pragma unroll
  for (int g = 0; g < G; ++g) {  // all loads in flight before any use
    const uint64_t i0 = base + 4 * ((uint64_t)g * DB_THREADS + tid);
    if (vec && i0 + 3 < n) {
      const float4 q = CONVERT ? __ldcs(reinterpret_cast<const float4 *>(d + i0))
                               : __ldg(reinterpret_cast<const float4 *>(d + i0));
      x[4 * g] = q.x, x[4 * g + 1] = q.y, x[4 * g + 2] = q.z, x[4 * g + 3] = q.w;
    } else {
#pragma unroll
      for (int j = 0; j < 4; ++j) x[4 * g + j] = i0 + j < n ? (CONVERT ? __ldcs(d + i0 + j) : __ldg(d + i0 + j)) : NAN;
    }
  }
#pragma unroll
  for (int k = 0; k < DB_PER_THREAD; ++k) {
    const uint64_t i = base + 4 * ((uint64_t)(k / 4) * DB_THREADS + tid) + k % 4;
    float v = x[k];
    if (i >= n || v != v) continue;
    if (CONVERT) {
      int cls;
      v = db_value(v, floor_lin, &cls);
      if (cls == 1) ++nm;
      else ++cv;
      x[k] = v;
    }
    if (isfinite(v)) {
      mn = fminf(mn, v);
      mx = fmaxf(mx, v);
      sum += (double)v;
      ++cnt;
    }
  }
  if (CONVERT) {  // the converted words back (NaN elements unchanged)
#pragma unroll
    for (int g = 0; g < G; ++g) {
      const uint64_t i0 = base + 4 * ((uint64_t)g * DB_THREADS + tid);
      if (vec && i0 + 3 < n) {
        __stcs(reinterpret_cast<float4 *>(d + i0), make_float4(x[4 * g], x[4 * g + 1], x[4 * g + 2], x[4 * g + 3]));
      } else {
#pragma unroll
        for (int j = 0; j < 4; ++j)
          if (i0 + j < n) d[i0 + j] = x[4 * g + j];
      }
    }
  }
  sum = warp_sum_d(sum);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    mn = fminf(mn, __shfl_xor_sync(0xffffffffu, mn, o));
    mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
    cv += __shfl_xor_sync(0xffffffffu, cv, o);
    nm += __shfl_xor_sync(0xffffffffu, nm, o);
  }
  if (lane == 0) {
    s_sum[wid] = sum;
    s_mn[wid] = mn;
    s_mx[wid] = mx;
    s_cnt[wid] = cnt;
    s_cv[wid] = cv;
    s_nm[wid] = nm;
  }
  __syncthreads();
  if (tid == 0) {
    DbPart p{0.0, INFINITY, -INFINITY, 0, 0, 0, 0};
    for (int w = 0; w < DB_THREADS / 32; ++w) {  // fixed order: deterministic
      p.sum += s_sum[w];
      p.mn = fminf(p.mn, s_mn[w]);
      p.mx = fmaxf(p.mx, s_mx[w]);
      p.cnt += s_cnt[w];
      p.cv += s_cv[w];
      p.nm += s_nm[w];
    }
    part[blockIdx.x] = p;  // the host sums the blocks (no contended atomics)
  }
}

// The median sample of compute_db_stats: every stride-th finite value in
// element order.  first[b] = finite values before block b.  The finite
// counts of every (round, warp) go to shared memory once; each thread then
// adds up its own prefix (one barrier per chunk).
__global__ void __launch_bounds__(DB_THREADS) k_db_sample(const float *__restrict__ d, uint64_t n,
                                                          const uint64_t *__restrict__ first, uint64_t stride,
                                                          float *__restrict__ sample, uint64_t n_sample) {
  // Round g of the block covers elements base + g * 1024 .. + 1024; lane l of
  // warp w holds four consecutive ones, base + g * 1024 + 4 (32 w + l) + j
  // (one 16-byte load).  A finite value's rank in element order is: the
  // block's first rank, the counts of earlier rounds, of earlier warps in the
  // round, of earlier lanes in the warp, and of the lane's earlier elements.
  constexpr int NW = DB_THREADS / 32, G = DB_PER_THREAD / 4, RND = 4 * DB_THREADS;
  __shared__ uint32_t s_c[G][NW];
  __shared__ uint64_t s_first[G];  // first sample rank at or after each round's start
  const uint64_t base = (uint64_t)blockIdx.x * DB_CHUNK;
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  const bool vec = (reinterpret_cast<uintptr_t>(d) & 15) == 0;
  float x[DB_PER_THREAD];
  unsigned m[DB_PER_THREAD];
#pragma unroll
  for (int g = 0; g < G; ++g) {
    const uint64_t i0 = base + (uint64_t)g * RND + 4 * (uint64_t)tid;
    if (vec && i0 + 3 < n) {
      const float4 q = __ldcs(reinterpret_cast<const float4 *>(d + i0));
      x[4 * g] = q.x, x[4 * g + 1] = q.y, x[4 * g + 2] = q.z, x[4 * g + 3] = q.w;
    } else {
#pragma unroll
      for (int j = 0; j < 4; ++j) x[4 * g + j] = i0 + j < n ? __ldcs(d + i0 + j) : NAN;
    }
  }
#pragma unroll
  for (int g = 0; g < G; ++g) {
    uint32_t wc = 0;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      m[4 * g + j] = __ballot_sync(0xffffffffu, isfinite(x[4 * g + j]));
      wc += __popc(m[4 * g + j]);
    }
    if (lane == 0) s_c[g][wid] = wc;
  }
  __syncthreads();
  if (tid < G) {  // thread g: the rank at round g's start (uniform over the block)
    uint64_t rk = first[blockIdx.x];
    for (int j = 0; j < tid; ++j)
      for (int w = 0; w < NW; ++w) rk += s_c[j][w];
    s_first[tid] = rk + (stride - rk % stride) % stride;
  }
  __syncthreads();
  const unsigned lt = (1u << lane) - 1u;
  uint64_t rank = first[blockIdx.x];
#pragma unroll
  for (int g = 0; g < G; ++g) {
    uint32_t before = 0, total = 0;
#pragma unroll
    for (int w = 0; w < NW; ++w) {
      const uint32_t c = s_c[g][w];
      before += w < wid ? c : 0u;
      total += c;
    }
#pragma unroll
    for (int j = 0; j < 4; ++j) before += __popc(m[4 * g + j] & lt);  // earlier lanes' elements
    const uint64_t f = s_first[g];
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      if ((m[4 * g + j] >> lane) & 1u) {
        const uint64_t rk = rank + before;
        // stride >= 1024: at most one sample per round, the one at rank f
        const bool take = stride >= (uint64_t)RND ? rk == f : (rk >= f && (rk - f) % stride == 0);
        if (take && rk / stride < n_sample) sample[rk / stride] = x[4 * g + j];
        ++before;  // this lane's next element comes after this one
      }
    }
    rank += total;
  }
}

// downsample_2x: the f64 mean of the non-NaN, in-range pixels of each 2x2
// patch (row-major order within the patch), NaN when there are none.
__global__ void k_downsample_2x(const float *__restrict__ src, uint64_t c, uint64_t r, float *__restrict__ dst,
                                uint64_t oc, uint64_t orows) {
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= oc * orows) return;
  const uint64_t y = i / oc, x = i - y * oc;
  double sum = 0.0;
  uint32_t cnt = 0;
#pragma unroll
  for (int a = 0; a < 2; ++a)
#pragma unroll
    for (int b = 0; b < 2; ++b) {
      const uint64_t sy = 2 * y + a, sx = 2 * x + b;
      if (sy < r && sx < c) {
        const float v = __ldg(src + sy * c + sx);
        if (v == v) {
          sum += (double)v;
          cnt += 1;
        }
      }
    }
  dst[i] = cnt > 0 ? (float)(sum / (double)cnt) : NAN;
}

// Tiles [t0, t0 + nt) of a level in file order (row-major tile grid of nx
// columns), each ts x ts (ts = 1 << lts >= 64), NaN outside the raster.
// Each thread writes 4 consecutive floats of one tile row (one 16-byte store).
__global__ void k_tile_pack(const float *__restrict__ src, uint64_t c, uint64_t r, int lts, uint32_t nx,
                            uint32_t t0, uint32_t nt, float4 *__restrict__ dst) {
  const uint64_t q = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;  // float4 index in the chunk
  const int lq = 2 * lts - 2;                                          // float4s per tile = 1 << lq
  if (q >= ((uint64_t)nt << lq)) return;
  const uint32_t t = t0 + (uint32_t)(q >> lq), w = (uint32_t)(q & ((1ull << lq) - 1)) << 2;
  const uint32_t ty = t / nx, tx = t - ty * nx;
  const uint64_t gy = ((uint64_t)ty << lts) + (w >> lts), gx = ((uint64_t)tx << lts) + (w & ((1u << lts) - 1));
  float v[4];
#pragma unroll
  for (int k = 0; k < 4; ++k) v[k] = (gy < r && gx + k < c) ? __ldg(src + gy * c + gx + k) : NAN;
  dst[q] = make_float4(v[0], v[1], v[2], v[3]);
}

unsigned grid_of(uint64_t n, unsigned per) { return (unsigned)((n + per - 1) / per); }

// geo_key_directory (output_crs.rs:265-287)
std::vector<uint16_t> cog_geo_keys(int32_t crs, int32_t zone) {
  if (crs == SD_CRS_WGS84) return {1, 1, 0, 3, 1024, 0, 1, 2, 1025, 0, 1, 1, 2048, 0, 1, 4326};
  const uint16_t epsg = (uint16_t)((crs == SD_CRS_UTM_SOUTH ? 32700 : 32600) + zone);
  return {1, 1, 0, 4, 1024, 0, 1, 1, 1025, 0, 1, 1, 3072, 0, 1, epsg, 3076, 0, 1, 9001};
}

struct Bytes {
  std::vector<uint8_t> b;
  template <class T>
  void put(T v) {
    const uint8_t *p = (const uint8_t *)&v;
    b.insert(b.end(), p, p + sizeof(T));
  }
};

struct FileCloser {
  FILE *f = nullptr;
  ~FileCloser() {
    if (f) std::fclose(f);
  }
};

struct PinnedBufs {
  void *p[2] = {nullptr, nullptr};
  cudaEvent_t ev[2] = {nullptr, nullptr};
  ~PinnedBufs() {
    for (int k = 0; k < 2; ++k) {
      if (ev[k]) cudaEventDestroy(ev[k]);
      if (p[k]) cudaFreeHost(p[k]);
    }
  }
};

}  // namespace
}  // namespace sd

using namespace sd;

namespace sd {
namespace {

// compute_db_stats from the dB pass's block partials: min, max and the f64
// sum in block order; the median of every max(cnt / 100000, 1)-th finite
// value in element order (k_db_sample) by nth_element on the host.
int db_stats_parts(sd_ctx *ctx, const float *d, uint64_t n, const std::vector<DbPart> &part, float st[4]) {
  const uint64_t nb = part.size();
  double sum = 0.0;
  uint64_t cnt = 0;
  float mn = INFINITY, mx = -INFINITY;
  std::vector<uint64_t> first(nb);
  for (uint64_t b = 0; b < nb; ++b) {
    first[b] = cnt;
    sum += part[b].sum;
    cnt += part[b].cnt;
    mn = std::min(mn, part[b].mn);
    mx = std::max(mx, part[b].mx);
  }
  st[0] = st[1] = st[2] = st[3] = NAN;
  if (cnt == 0) return SD_OK;
  cudaStream_t s = ctx->stream;
  const uint64_t stride = std::max<uint64_t>(cnt / 100000, 1);
  const uint64_t n_sample = (cnt + stride - 1) / stride;
  uint64_t *d_first;
  float *d_sample;
  SD_TRY(scratch_t(ctx, "db.first", nb, &d_first));
  SD_TRY(scratch_t(ctx, "db.sample", n_sample, &d_sample));
  SD_CUDA(ctx, cudaMemcpyAsync(d_first, first.data(), nb * 8, cudaMemcpyHostToDevice, s));
  SD_TIMED_BEGIN(ctx, "k_db_sample");
  k_db_sample<<<(unsigned)nb, DB_THREADS, 0, s>>>(d, n, d_first, stride, d_sample, n_sample);
  SD_LAUNCHED(ctx);
  std::vector<float> sample(n_sample);
  SD_CUDA(ctx, cudaMemcpyAsync(sample.data(), d_sample, n_sample * 4, cudaMemcpyDeviceToHost, s));
  SD_TRY(sync(ctx));
  std::nth_element(sample.begin(), sample.begin() + n_sample / 2, sample.end());
  st[0] = mn;
  st[1] = mx;
  st[2] = (float)(sum / (double)cnt);
  st[3] = sample[n_sample / 2];
  return SD_OK;
}

// The dB pass (CONVERT: to_db_inplace; else the statistics only) over device
// memory d, its partials copied back.
template <bool CONVERT>
int db_pass(sd_ctx *ctx, float *d, uint64_t n, float floor_lin, std::vector<DbPart> *part) {
  const uint64_t nb = (n + DB_CHUNK - 1) / DB_CHUNK;
  if (nb > 0x7FFFFFFFull) return set_error(ctx, SD_ERR_INVALID_ARGUMENT, "raster too large");
  DbPart *d_part;
  SD_TRY(scratch_t(ctx, "db.part", nb, &d_part));
  SD_TIMED_BEGIN(ctx, CONVERT ? "k_to_db" : "k_db_stats");
  k_to_db<CONVERT><<<(unsigned)nb, DB_THREADS, 0, ctx->stream>>>(d, n, floor_lin, d_part);
  SD_LAUNCHED(ctx);
  part->resize(nb);
  SD_CUDA(ctx, cudaMemcpyAsync(part->data(), d_part, nb * sizeof(DbPart), cudaMemcpyDeviceToHost, ctx->stream));
  return sync(ctx);
}

}  // namespace

int db_stats_device(sd_ctx *ctx, const float *d, uint64_t n, float st[4]) {
  st[0] = st[1] = st[2] = st[3] = NAN;
  if (n == 0) return SD_OK;
  std::vector<DbPart> part;
  SD_TRY(db_pass<false>(ctx, const_cast<float *>(d), n, 0.0f, &part));
  return db_stats_parts(ctx, d, n, part, st);
}

int db_finish(sd_ctx *ctx, const float *d_out, uint64_t n, uint64_t converted, uint64_t masked) {
  ctx->db_valid = false;
  ctx->db_counts[0] = converted;
  ctx->db_counts[1] = masked;
  SD_TRY(db_stats_device(ctx, d_out, n, ctx->db_stats));
  ctx->db_valid = true;
  return SD_OK;
}

}  // namespace sd

extern "C" int sd_to_db(sd_ctx *ctx, float *data, uint64_t n, float noise_floor_linear, uint64_t *counts,
                        float *stats) {
  SD_STAGE("db_conversion");
  if (!ctx) return SD_ERR_INVALID_ARGUMENT;
  if (!(noise_floor_linear >= 0.0f))
    return set_error(ctx, SD_ERR_EXPORT_INVALID_NOISE_FLOOR, "noise_floor_linear must be non-negative; got %g",
                     (double)noise_floor_linear);
  if (n > 0 && !data) return set_error(ctx, SD_ERR_INVALID_ARGUMENT, "null data");
  uint64_t cv = 0, nm = 0;
  float st[4] = {NAN, NAN, NAN, NAN};
  if (n > 0) {
    SD_CUDA(ctx, cudaSetDevice(ctx->device));
    const void *din;
    SD_TRY(stage_in(ctx, "db.data", data, n * sizeof(float), &din));
    float *d = (float *)din;
    std::vector<DbPart> part;
    SD_TRY(db_pass<true>(ctx, d, n, noise_floor_linear, &part));
    for (const DbPart &q : part) {
      cv += q.cv;
      nm += q.nm;
    }
    if (stats) SD_TRY(db_stats_parts(ctx, d, n, part, st));
    SD_TRY(finish_out(ctx, data, d, n * sizeof(float)));
    SD_TRY(sync(ctx));
  }
  if (counts) {
    counts[0] = cv;
    counts[1] = nm;
  }
  if (stats) std::memcpy(stats, st, sizeof st);
  return SD_OK;
}

extern "C" int sd_ctx_set_db_output(sd_ctx *ctx, int32_t enable, float noise_floor_linear) {
  if (!ctx) return SD_ERR_INVALID_ARGUMENT;
  if (enable && !(noise_floor_linear >= 0.0f))
    return set_error(ctx, SD_ERR_EXPORT_INVALID_NOISE_FLOOR, "noise_floor_linear must be non-negative; got %g",
                     (double)noise_floor_linear);
  ctx->db_out = enable != 0;
  ctx->db_floor = enable ? noise_floor_linear : 0.0f;
  ctx->db_valid = false;
  return SD_OK;
}

extern "C" int sd_ctx_db_result(sd_ctx *ctx, uint64_t *counts, float *stats) {
  if (!ctx) return SD_ERR_INVALID_ARGUMENT;
  if (!ctx->db_valid)
    return set_error(ctx, SD_ERR_INVALID_ARGUMENT, "no call with dB output has completed on this context");
  if (counts) counts[0] = ctx->db_counts[0], counts[1] = ctx->db_counts[1];
  if (stats) std::memcpy(stats, ctx->db_stats, sizeof ctx->db_stats);
  return SD_OK;
}

extern "C" int sd_downsample_2x(sd_ctx *ctx, const float *src, uint64_t cols, uint64_t rows, float *dst) {
  SD_STAGE("export_overviews");
  if (!ctx) return SD_ERR_INVALID_ARGUMENT;
  if (cols == 0 || rows == 0) return SD_OK;
  if (!src || !dst) return set_error(ctx, SD_ERR_INVALID_ARGUMENT, "null buffer");
  SD_CUDA(ctx, cudaSetDevice(ctx->device));
  const uint64_t oc = (cols + 1) / 2, orows = (rows + 1) / 2;
  const void *din;
  void *dout;
  SD_TRY(stage_in(ctx, "ds.in", src, cols * rows * 4, &din));
  SD_TRY(stage_out(ctx, "ds.out", dst, oc * orows * 4, &dout));
  SD_TIMED_BEGIN(ctx, "k_downsample_2x");
  k_downsample_2x<<<grid_of(oc * orows, 256), 256, 0, ctx->stream>>>((const float *)din, cols, rows,
                                                                      (float *)dout, oc, orows);
  SD_LAUNCHED(ctx);
  SD_TRY(finish_out(ctx, dst, dout, oc * orows * 4));
  return sync(ctx);
}

extern "C" int sd_write_cog(sd_ctx *ctx, const char *path, const float *data, uint64_t cols, uint64_t rows,
                            const double *gt, int32_t crs, int32_t utm_zone, uint32_t tile_size) {
  SD_STAGE("export_geotiff");
  if (!ctx) return SD_ERR_INVALID_ARGUMENT;
  if (!path || !gt) return set_error(ctx, SD_ERR_INVALID_ARGUMENT, "null path or geotransform");
  const double pw = gt[1], ph = -gt[5];
  if (!std::isfinite(pw) || pw <= 0.0 || !std::isfinite(ph) || ph <= 0.0)
    return set_error(ctx, SD_ERR_EXPORT_INVALID_GEOTRANSFORM,
                     "geotransform pixel width/height must be positive and finite; got [%g, %g, %g, %g, %g, %g]",
                     gt[0], gt[1], gt[2], gt[3], gt[4], gt[5]);
  if (tile_size < 64 || tile_size > 4096 || (tile_size & (tile_size - 1)) != 0)
    return set_error(ctx, SD_ERR_EXPORT_INVALID_TILE_SIZE,
                     "COG tile size must be a power of two >= 64 and <= 4096; got %u", tile_size);
  if (crs != SD_CRS_WGS84 && !((crs == SD_CRS_UTM_NORTH || crs == SD_CRS_UTM_SOUTH) && utm_zone >= 1 && utm_zone <= 60))
    return set_error(ctx, SD_ERR_INVALID_ARGUMENT, "unsupported CRS %d (zone %d)", crs, utm_zone);
  if (cols == 0 || rows == 0 || !data) return set_error(ctx, SD_ERR_INVALID_ARGUMENT, "empty raster");
  SD_CUDA(ctx, cudaSetDevice(ctx->device));
  cudaStream_t s = ctx->stream;
  const uint64_t ts = tile_size;
  int lts = 0;
  while ((1ull << lts) < ts) ++lts;
  const std::vector<uint16_t> keys = cog_geo_keys(crs, utm_zone);

  // ── overview pyramid on the device (finest level first) ──
  const void *din;
  SD_TRY(stage_in(ctx, "cog.full", data, cols * rows * 4, &din));
  std::vector<uint64_t> lc, lr;
  {
    uint64_t c = (cols + 1) / 2, r = (rows + 1) / 2;
    while (true) {
      lc.push_back(c);
      lr.push_back(r);
      if (!(c > ts || r > ts)) break;
      c = (c + 1) / 2;
      r = (r + 1) / 2;
    }
  }
  const size_t n_ovr = lc.size();
  std::vector<uint64_t> loff(n_ovr);
  uint64_t ov_total = 0;
  for (size_t k = 0; k < n_ovr; ++k) {
    loff[k] = ov_total;
    ov_total += lc[k] * lr[k];
  }
  float *d_ov;
  SD_TRY(scratch_t(ctx, "cog.ovr", ov_total, &d_ov));
  SD_TIMED_BEGIN(ctx, "k_downsample_2x");
  for (size_t k = 0; k < n_ovr; ++k) {
    const float *src = k == 0 ? (const float *)din : d_ov + loff[k - 1];
    const uint64_t sc = k == 0 ? cols : lc[k - 1], sr = k == 0 ? rows : lr[k - 1];
    k_downsample_2x<<<grid_of(lc[k] * lr[k], 256), 256, 0, s>>>(src, sc, sr, d_ov + loff[k], lc[k], lr[k]);
  }
  SD_LAUNCHED(ctx);

  // ── layout: IFDs coarsest overview first, full resolution last ──
  struct Lvl {
    const float *src;
    uint64_t c, r, nx, ny, nt;
  };
  std::vector<Lvl> lv;
  for (size_t k = n_ovr; k-- > 0;) lv.push_back({d_ov + loff[k], lc[k], lr[k], 0, 0, 0});
  lv.push_back({(const float *)din, cols, rows, 0, 0, 0});
  for (Lvl &l : lv) {
    l.nx = (l.c + ts - 1) / ts;
    l.ny = (l.r + ts - 1) / ts;
    l.nt = l.nx * l.ny;
    if (l.nt > 0xFFFFFFFFull) return set_error(ctx, SD_ERR_INVALID_ARGUMENT, "raster has too many tiles");
  }
  const bool big = rows * cols * 4ull > 0xFFFFFFFFull;  // the reference's estimate (export.rs:465)
  const uint64_t n_entries = 17, ifd_bytes = big ? 8 + 17 * 20 + 8 : 2 + 17 * 12 + 4, arr = big ? 8 : 4;
  const uint64_t tile_bytes = ts * ts * 4;
  uint64_t off = big ? 16 : 8;
  std::vector<uint64_t> ifd_at(lv.size()), toff_at(lv.size()), tbc_at(lv.size()), data_at(lv.size());
  for (size_t k = 0; k < lv.size(); ++k) {
    ifd_at[k] = off;
    off += ifd_bytes;
    toff_at[k] = off;
    off += lv[k].nt * arr;
    tbc_at[k] = off;
    off += lv[k].nt * arr;
  }
  const uint64_t scale_at = off, tie_at = off + 24, keys_at = off + 72;
  off = keys_at + keys.size() * 2;
  for (size_t k = 0; k < lv.size(); ++k) {
    data_at[k] = off;
    off += lv[k].nt * tile_bytes;
  }
  Bytes h;
  h.b.reserve((size_t)data_at[0]);
  h.put<uint8_t>('I');
  h.put<uint8_t>('I');
  if (big) {
    h.put<uint16_t>(43);
    h.put<uint16_t>(8);
    h.put<uint16_t>(0);
    h.put<uint64_t>(ifd_at[0]);
  } else {
    h.put<uint16_t>(42);
    h.put<uint32_t>((uint32_t)ifd_at[0]);
  }
  for (size_t k = 0; k < lv.size(); ++k) {
    auto tag = [&](uint16_t t, uint16_t typ, uint64_t count, uint64_t val) {
      h.put<uint16_t>(t);
      h.put<uint16_t>(typ);
      if (big) {
        h.put<uint64_t>(count);
        h.put<uint64_t>(val);
      } else {
        h.put<uint32_t>((uint32_t)count);
        h.put<uint32_t>((uint32_t)val);
      }
    };
    if (big) h.put<uint64_t>(n_entries);
    else h.put<uint16_t>((uint16_t)n_entries);
    tag(256, 4, 1, lv[k].c);
    tag(257, 4, 1, lv[k].r);
    tag(258, 3, 1, 32);
    tag(259, 3, 1, 1);
    tag(262, 3, 1, 1);
    tag(277, 3, 1, 1);
    tag(282, big ? 5 : 4, 1, big ? ((1ull << 32) | 72ull) : 72);  // XResolution
    tag(283, big ? 5 : 4, 1, big ? ((1ull << 32) | 72ull) : 72);  // YResolution
    tag(296, 3, 1, 1);
    tag(322, 4, 1, ts);
    tag(323, 4, 1, ts);
    tag(324, big ? 16 : 4, lv[k].nt, toff_at[k]);
    tag(325, big ? 16 : 4, lv[k].nt, tbc_at[k]);
    tag(339, 3, 1, 3);
    tag(33550, 12, 3, scale_at);
    tag(33922, 12, 6, tie_at);
    tag(34735, 3, keys.size(), keys_at);
    const uint64_t next = k + 1 < lv.size() ? ifd_at[k + 1] : 0;
    if (big) h.put<uint64_t>(next);
    else h.put<uint32_t>((uint32_t)next);
    for (uint64_t t = 0; t < lv[k].nt; ++t) {
      if (big) h.put<uint64_t>(data_at[k] + t * tile_bytes);
      else h.put<uint32_t>((uint32_t)(data_at[k] + t * tile_bytes));
    }
    for (uint64_t t = 0; t < lv[k].nt; ++t) {
      if (big) h.put<uint64_t>(tile_bytes);
      else h.put<uint32_t>((uint32_t)tile_bytes);
    }
  }
  for (double v : {gt[1], -gt[5], 0.0, 0.0, 0.0, 0.0, gt[0], gt[3], 0.0}) h.put<double>(v);
  for (uint16_t k : keys) h.put<uint16_t>(k);

  FileCloser fc;
  fc.f = std::fopen(path, "wb");
  if (!fc.f) return set_error(ctx, SD_ERR_EXPORT_IO, "I/O error writing GeoTIFF: cannot create %s", path);
  if (std::fwrite(h.b.data(), 1, h.b.size(), fc.f) != h.b.size())
    return set_error(ctx, SD_ERR_EXPORT_IO, "I/O error writing GeoTIFF: short write to %s", path);

  // ── tiles: packed on the device in chunks, copied through two pinned
  // buffers while the host writes the previous chunk ──
  const uint64_t chunk_tiles = std::max<uint64_t>(1, (64ull << 20) / tile_bytes);
  const uint64_t chunk_bytes = chunk_tiles * tile_bytes;
  float *d_pack[2];
  SD_TRY(scratch_t(ctx, "cog.pack0", chunk_tiles * ts * ts, &d_pack[0]));
  SD_TRY(scratch_t(ctx, "cog.pack1", chunk_tiles * ts * ts, &d_pack[1]));
  PinnedBufs pb;
  for (int k = 0; k < 2; ++k) {
    SD_CUDA(ctx, cudaHostAlloc(&pb.p[k], chunk_bytes, cudaHostAllocDefault));
    SD_CUDA(ctx, cudaEventCreateWithFlags(&pb.ev[k], cudaEventDisableTiming));
  }
  struct Job {
    int buf;
    uint64_t bytes;
  };
  std::vector<Job> pending;  // at most one chunk in flight besides the one being written
  int cur = 0;
  auto drain = [&](const Job &j) -> int {
    SD_CUDA(ctx, cudaEventSynchronize(pb.ev[j.buf]));
    if (std::fwrite(pb.p[j.buf], 1, j.bytes, fc.f) != j.bytes)
      return set_error(ctx, SD_ERR_EXPORT_IO, "I/O error writing GeoTIFF: short write to %s", path);
    return SD_OK;
  };
  for (const Lvl &l : lv) {
    for (uint64_t t0 = 0; t0 < l.nt; t0 += chunk_tiles) {
      const uint64_t nt = std::min(chunk_tiles, l.nt - t0);
      if (pending.size() == 2) {  // both buffers busy: write the older one out
        SD_TRY(drain(pending.front()));
        pending.erase(pending.begin());
      }
      SD_TIMED_BEGIN(ctx, "k_tile_pack");
      k_tile_pack<<<grid_of(nt * ts * ts / 4, 256), 256, 0, s>>>(l.src, l.c, l.r, lts, (uint32_t)l.nx,
                                                                  (uint32_t)t0, (uint32_t)nt, (float4 *)d_pack[cur]);
      SD_LAUNCHED(ctx);
      SD_CUDA(ctx, cudaMemcpyAsync(pb.p[cur], d_pack[cur], nt * tile_bytes, cudaMemcpyDeviceToHost, s));
      SD_CUDA(ctx, cudaEventRecord(pb.ev[cur], s));
      pending.push_back({cur, nt * tile_bytes});
      cur ^= 1;
    }
  }
  for (const Job &j : pending) SD_TRY(drain(j));
  SD_TRY(sync(ctx));
  FILE *f = fc.f;
  fc.f = nullptr;
  if (std::fclose(f) != 0) return set_error(ctx, SD_ERR_EXPORT_IO, "I/O error writing GeoTIFF: closing %s", path);
  return SD_OK;
}
