// speckle.cu — the five SpeckleKernel filters on sm_100a.
//
// Replaces apply_speckle_filter / SpeckleKernel::apply (sardine/src/speckle.rs:
// 131-180, 218-569, 586-603).  One thread per output pixel; the block's
// window footprint (tile + halo) is staged once in shared memory, out-of-image
// cells stored as NaN so the reference's "in bounds and finite" filter is a
// single isfinite test.  Window sums are accumulated in f64 in the
// reference's row-major tap order and cast to f32 exactly as speckle.rs:
// 226-240 does, so the f32 filter arithmetic sees the same inputs.
#include <cmath>

#include "geo.cuh"
#include "runtime.cuh"
#include "tiles.cuh"

namespace sd {
namespace {

constexpr int TX = 32, TY = 8;

// Refined Lee directional masks (speckle.rs:432-457) as row-major tap lists.
struct RlMasks {
  int8_t n[8];
  int8_t dy[8][24];
  int8_t dx[8][24];
};
__constant__ RlMasks c_rl;

bool rl_in_mask(int dir, int dy, int dx) {
  if (dy == 0 && dx == 0) return false;
  switch (dir) {
    case 0: return dy >= 1 && dy <= 3;
    case 1: return dy >= -3 && dy <= -1;
    case 2: return dx >= 1 && dx <= 3;
    case 3: return dx >= -3 && dx <= -1;
    case 4: return std::abs(dy - dx) <= 1 && (dy + dx) >= 1;
    case 5: return std::abs(dy - dx) <= 1 && (dy + dx) <= -1;
    case 6: return std::abs(dy + dx) <= 1 && (dx - dy) >= 1;
    case 7: return std::abs(dy + dx) <= 1 && (dx - dy) <= -1;
  }
  return false;
}

RlMasks make_masks() {
  RlMasks m{};
  for (int d = 0; d < 8; ++d) {
    int k = 0;
    for (int dy = -3; dy <= 3; ++dy)
      for (int dx = -3; dx <= 3; ++dx)
        if (rl_in_mask(d, dy, dx)) {
          m.dy[d][k] = (int8_t)dy;
          m.dx[d][k] = (int8_t)dx;
          ++k;
        }
    m.n[d] = (int8_t)k;
  }
  return m;
}

struct SpParams {
  const float *in;
  float *out;
  int64_t cols, rows;
  int half;
  int kind;
  float enl, damping, cv_n_sq, cv_max_sq;
};

__device__ __forceinline__ bool finitef(float v) { return isfinite(v); }

struct SpCoef {
  float enl, damping, cv_n_sq, cv_max_sq;
};

// One output pixel of filter KIND from the staged window: `tile` holds the
// footprint with row stride tw, the pixel sits at (lx, ly), h = half window.
template <int KIND>
__device__ float speckle_px(const float *tile, int tw, int lx, int ly, int h, const SpCoef &p) {
  const float centre = tile[ly * tw + lx];
  float o = NAN;
  if (!finitef(centre)) return o;
  if (KIND == SD_SPECKLE_REFINED_LEE) {
    float best_cv = INFINITY, best_mean = centre, best_var = 0.0f;
    for (int d = 0; d < 8; ++d) {
      double sum = 0.0, sum_sq = 0.0;
      int n = 0;
      const int nt = c_rl.n[d];
      for (int k = 0; k < nt; ++k) {
        float v = tile[(ly + c_rl.dy[d][k]) * tw + lx + c_rl.dx[d][k]];
        if (!finitef(v)) continue;
        double vd = (double)v;
        sum += vd;
        sum_sq += vd * vd;
        ++n;
      }
      if (n == 0) continue;
      double md = sum / (double)n;
      double vard = maxd_nan(sum_sq / (double)n - md * md, 0.0);
      float mean = (float)md, var = (float)vard;
      if (!(mean > 0.0f)) continue;
      float cv = var / (mean * mean);
      if (cv < best_cv) {
        best_cv = cv;
        best_mean = mean;
        best_var = var;
      }
    }
    if (!isfinite(best_cv)) {
      o = centre;
    } else {
      float noise_var = best_mean * best_mean * p.cv_n_sq;
      float signal_var = maxf_nan(best_var - noise_var, 0.0f);
      float denom = signal_var + noise_var;
      float k = denom > 0.0f ? signal_var / denom : 0.0f;
      o = best_mean + k * (centre - best_mean);
    }
    return o;
  }
  double sum = 0.0, sum_sq = 0.0;
  int n = 0;
  for (int dy = -h; dy <= h; ++dy) {
    const float *row = tile + (ly + dy) * tw + lx;
    for (int dx = -h; dx <= h; ++dx) {
      float v = row[dx];
      if (!finitef(v)) continue;
      double vd = (double)v;
      sum += vd;
      sum_sq += vd * vd;
      ++n;
    }
  }
  if (n == 0) return o;
  double md = sum / (double)n;
  double vard = maxd_nan(sum_sq / (double)n - md * md, 0.0);
  float mean = (float)md, var = (float)vard;
  if (KIND == SD_SPECKLE_BOXCAR) {
    o = mean;
  } else if (KIND == SD_SPECKLE_LEE) {
    float noise_var = mean * mean * p.cv_n_sq;
    float signal_var = maxf_nan(var - noise_var, 0.0f);
    float denom = signal_var + noise_var;
    float k = denom > 0.0f ? signal_var / denom : 0.0f;
    o = mean + k * (centre - mean);
  } else if (KIND == SD_SPECKLE_FROST) {
    float cv_sq = mean > 0.0f ? var / (mean * mean) : 0.0f;
    float alpha = p.damping * cv_sq;
    double wsum = 0.0, vwsum = 0.0;
    for (int dy = -h; dy <= h; ++dy) {
      const float *row = tile + (ly + dy) * tw + lx;
      for (int dx = -h; dx <= h; ++dx) {
        float v = row[dx];
        if (!finitef(v)) continue;
        float dd = (float)(abs(dy) + abs(dx));
        double w = (double)expf(-alpha * dd);
        wsum += w;
        vwsum += w * (double)v;
      }
    }
    if (wsum > 0.0) o = (float)(vwsum / wsum);
  } else {  // Gamma-MAP (speckle.rs:348-411)
    float cv_sq = mean > 0.0f ? var / (mean * mean) : 0.0f;
    if (cv_sq <= p.cv_n_sq) {
      o = mean;
    } else if (cv_sq >= p.cv_max_sq) {
      o = centre;
    } else {
      float alpha = (1.0f + p.cv_n_sq) / (cv_sq - p.cv_n_sq);
      float b = (alpha - p.enl - 1.0f) * mean;
      float disc = b * b + 4.0f * alpha * p.enl * mean * centre;
      o = disc >= 0.0f ? ((p.enl - alpha + 1.0f) * mean + sqrtf(disc)) / (2.0f * p.enl) : mean;
    }
  }
  return o;
}

template <int KIND>
__global__ void __launch_bounds__(TX *TY) k_speckle(SpParams p) {
  extern __shared__ float tile[];
  const int h = p.half;
  const int tw = TX + 2 * h, th = TY + 2 * h;
  const int64_t c0 = (int64_t)blockIdx.x * TX - h, r0 = (int64_t)blockIdx.y * TY - h;
  for (int k = threadIdx.y * TX + threadIdx.x; k < tw * th; k += TX * TY) {
    int ty = k / tw, tx = k % tw;
    int64_t rr = r0 + ty, cc = c0 + tx;
    float v = NAN;
    if (rr >= 0 && cc >= 0 && rr < p.rows && cc < p.cols) v = __ldg(p.in + rr * p.cols + cc);
    tile[k] = v;
  }
  __syncthreads();
  const int64_t c = (int64_t)blockIdx.x * TX + threadIdx.x, r = (int64_t)blockIdx.y * TY + threadIdx.y;
  if (c >= p.cols || r >= p.rows) return;
  const SpCoef cf{p.enl, p.damping, p.cv_n_sq, p.cv_max_sq};
  p.out[r * p.cols + c] = speckle_px<KIND>(tile, tw, threadIdx.x + h, threadIdx.y + h, h, cf);
}

// ── batched form: many tiles, each a halo'd geocoded raster ──────────────────
// Item = one tx x ty block (the launch's block shape, chosen by the tile
// autotuner) of one tile's output.  The block stages its window from the
// tile's halo'd raster (cells outside it are NaN, which the filters skip like
// out-of-image cells), filters the data plane with the tile's kind (or
// copies it when kind < 0) and crops cos(LIA) and the mask.
__global__ void __launch_bounds__(1024) k_speckle_tiles(const SpWork *__restrict__ wp) {
  extern __shared__ float tile[];
  const SpWork w = *wp;
  const int bx = (int)blockDim.x, by = (int)blockDim.y, nt = bx * by;
  const int tid = threadIdx.y * bx + threadIdx.x;
  const uint64_t total = w.pre[w.n_jobs];
  for (uint64_t item = blockIdx.x; item < total; item += gridDim.x) {
    int lo = 0, hi = w.n_jobs;
    while (hi - lo > 1) {
      const int mid = (lo + hi) >> 1;
      if (w.pre[mid] <= item) lo = mid;
      else hi = mid;
    }
    const SpJob &jb = w.jobs[lo];
    const uint64_t li = item - w.pre[lo];
    const int64_t nbx = (jb.cols + bx - 1) / bx;
    const int64_t tr = (int64_t)li / nbx, tc = (int64_t)li % nbx;
    const int h = jb.kind >= 0 ? jb.half : 0;
    const int tw = bx + 2 * h, th = by + 2 * h;
    const int64_t in_cols = jb.cols + 2 * jb.halo, in_rows = jb.rows + 2 * jb.halo;
    // output (r, c) is input (r + halo, c + halo)
    const int64_t c0 = tc * bx + jb.halo - h, r0 = tr * by + jb.halo - h;
    __syncthreads();
    for (int k = tid; k < tw * th; k += nt) {
      const int ty = k / tw, tx = k % tw;
      const int64_t rr = r0 + ty, cc = c0 + tx;
      float v = NAN;
      if (rr >= 0 && cc >= 0 && rr < in_rows && cc < in_cols) v = __ldg(jb.in + rr * in_cols + cc);
      tile[k] = v;
    }
    __syncthreads();
    const int64_t c = tc * bx + threadIdx.x, r = tr * by + threadIdx.y;
    if (c < jb.cols && r < jb.rows) {
      const SpCoef cf{jb.enl, jb.damping, jb.cv_n_sq, jb.cv_max_sq};
      const int lx = threadIdx.x + h, ly = threadIdx.y + h;
      float o;
      switch (jb.kind) {
        case SD_SPECKLE_BOXCAR: o = speckle_px<SD_SPECKLE_BOXCAR>(tile, tw, lx, ly, h, cf); break;
        case SD_SPECKLE_LEE: o = speckle_px<SD_SPECKLE_LEE>(tile, tw, lx, ly, h, cf); break;
        case SD_SPECKLE_FROST: o = speckle_px<SD_SPECKLE_FROST>(tile, tw, lx, ly, h, cf); break;
        case SD_SPECKLE_GAMMA_MAP: o = speckle_px<SD_SPECKLE_GAMMA_MAP>(tile, tw, lx, ly, h, cf); break;
        case SD_SPECKLE_REFINED_LEE: o = speckle_px<SD_SPECKLE_REFINED_LEE>(tile, tw, lx, ly, h, cf); break;
        default: o = tile[ly * tw + lx];
      }
      const int64_t oi = r * jb.cols + c, ii = (r + jb.halo) * in_cols + (c + jb.halo);
      jb.out[oi] = o;
      if (jb.cos_out) jb.cos_out[oi] = __ldg(jb.cos_in + ii);
      if (jb.mask_out) jb.mask_out[oi] = __ldg(jb.mask_in + ii);
    }
  }
}

bool g_masks_uploaded[64] = {false};

}  // namespace

int speckle_masks(sd_ctx *ctx) {
  if (!g_masks_uploaded[ctx->device & 63]) {
    RlMasks m = make_masks();
    SD_CUDA(ctx, cudaMemcpyToSymbol(c_rl, &m, sizeof m));
    g_masks_uploaded[ctx->device & 63] = true;
  }
  return SD_OK;
}

void speckle_coefs(int kind, uint64_t window, float enl, float damping, SpJob *j) {
  const uint64_t win = kind == SD_SPECKLE_REFINED_LEE ? 7 : window;
  j->kind = kind;
  j->half = kind >= 0 ? (int)(win / 2) : 0;
  j->enl = enl;
  j->damping = damping;
  j->cv_n_sq = kind >= 0 ? 1.0f / enl : 0.0f;
  j->cv_max_sq = j->cv_n_sq < 1.0f ? 2.0f * j->cv_n_sq / (1.0f - j->cv_n_sq) : INFINITY;
}

bool speckle_shape_ok(int tx, int ty) {
  return tx >= 8 && ty >= 1 && tx <= 256 && tx * ty <= 1024 && (tx * ty) % 32 == 0;
}

int speckle_tiles_launch(sd_ctx *ctx, const SpWork *d_work, uint64_t total, bool full_grid, int tx, int ty) {
  SD_TRY(speckle_masks(ctx));
  const size_t smem = (size_t)(tx + 2 * SP_MAX_HALF) * (ty + 2 * SP_MAX_HALF) * sizeof(float);
  const unsigned g = persistent_grid(k_speckle_tiles, tx * ty, smem, full_grid ? ~0ull : total);
  SD_TIMED_BEGIN(ctx, "k_speckle_tiles");
  k_speckle_tiles<<<g, dim3(tx, ty), smem, ctx->stream>>>(d_work);
  SD_LAUNCHED(ctx);
  return SD_OK;
}

uint64_t speckle_tile_items(const SpJob &j, int tx, int ty) {
  return (uint64_t)((j.cols + tx - 1) / tx) * (uint64_t)((j.rows + ty - 1) / ty);
}

// Validation in the reference's order (speckle.rs:137-178).
int speckle_validate(uint64_t len, uint64_t cols, uint64_t rows, int kind, uint64_t window, float enl,
                     float damping) {
  if (cols != 0 && rows > UINT64_MAX / cols) return SD_ERR_SPECKLE_DIMENSION_MISMATCH;
  if (len != cols * rows) return SD_ERR_SPECKLE_DIMENSION_MISMATCH;
  if (kind < SD_SPECKLE_BOXCAR || kind > SD_SPECKLE_REFINED_LEE) return SD_ERR_INVALID_ARGUMENT;
  uint64_t win = kind == SD_SPECKLE_REFINED_LEE ? 7 : window;
  if (win < 3 || win % 2 == 0) return SD_ERR_SPECKLE_BAD_WINDOW;
  if (kind == SD_SPECKLE_LEE || kind == SD_SPECKLE_GAMMA_MAP || kind == SD_SPECKLE_REFINED_LEE)
    if (!(enl > 0.0f) || !std::isfinite(enl)) return SD_ERR_SPECKLE_BAD_ENL;
  if (kind == SD_SPECKLE_FROST)
    if (!std::isfinite(damping) || damping < 0.0f) return SD_ERR_SPECKLE_BAD_DAMPING;
  return SD_OK;
}

// Launch on device buffers (shared with the tile path).
int speckle_launch(sd_ctx *ctx, const float *d_in, float *d_out, uint64_t cols, uint64_t rows,
                   int kind, uint64_t window, float enl, float damping, cudaStream_t st) {
  if (cols == 0 || rows == 0) return SD_OK;
  SD_TRY(speckle_masks(ctx));
  uint64_t win = kind == SD_SPECKLE_REFINED_LEE ? 7 : window;
  SpParams p;
  p.in = d_in;
  p.out = d_out;
  p.cols = (int64_t)cols;
  p.rows = (int64_t)rows;
  p.half = (int)(win / 2);
  p.kind = kind;
  p.enl = enl;
  p.damping = damping;
  p.cv_n_sq = 1.0f / enl;
  p.cv_max_sq = p.cv_n_sq < 1.0f ? 2.0f * p.cv_n_sq / (1.0f - p.cv_n_sq) : INFINITY;
  const int h = p.half;
  size_t smem = (size_t)(TX + 2 * h) * (TY + 2 * h) * sizeof(float);
  if (smem > 200 * 1024)
    return set_error(ctx, SD_ERR_INVALID_ARGUMENT, "speckle window %llu too large", (unsigned long long)win);
  dim3 grid((unsigned)((cols + TX - 1) / TX), (unsigned)((rows + TY - 1) / TY));
  dim3 block(TX, TY);
  switch (kind) {
#define SD_LAUNCH_SPECKLE(K)                                                                 \
  case K:                                                                                    \
    if (smem > 48 * 1024)                                                                    \
      SD_CUDA(ctx, cudaFuncSetAttribute(k_speckle<K>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem)); \
    SD_TIMED_BEGIN(ctx, "k_speckle_" #K);                                               \
    k_speckle<K><<<grid, block, smem, st>>>(p);                                             \
    break;
    SD_LAUNCH_SPECKLE(SD_SPECKLE_BOXCAR)
    SD_LAUNCH_SPECKLE(SD_SPECKLE_LEE)
    SD_LAUNCH_SPECKLE(SD_SPECKLE_FROST)
    SD_LAUNCH_SPECKLE(SD_SPECKLE_GAMMA_MAP)
    SD_LAUNCH_SPECKLE(SD_SPECKLE_REFINED_LEE)
#undef SD_LAUNCH_SPECKLE
  }
  SD_LAUNCHED(ctx);
  return SD_OK;
}

}  // namespace sd

using namespace sd;

extern "C" int sd_speckle(sd_ctx *ctx, const float *data, uint64_t data_len, uint64_t cols,
                          uint64_t rows, int32_t kind, uint64_t window, float enl, float damping,
                          float *out) {
  if (!ctx) return SD_ERR_INVALID_ARGUMENT;
  int rc = speckle_validate(data_len, cols, rows, kind, window, enl, damping);
  if (rc != SD_OK) {
    switch (rc) {
      case SD_ERR_SPECKLE_DIMENSION_MISMATCH:
        return set_error(ctx, rc, "data length %llu does not match cols×rows = %llu",
                         (unsigned long long)data_len, (unsigned long long)(cols * rows));
      case SD_ERR_SPECKLE_BAD_WINDOW:
        return set_error(ctx, rc, "window size %llu must be an odd integer ≥ 3",
                         (unsigned long long)(kind == SD_SPECKLE_REFINED_LEE ? 7 : window));
      case SD_ERR_SPECKLE_BAD_ENL:
        return set_error(ctx, rc, "ENL must be > 0; got %g", (double)enl);
      case SD_ERR_SPECKLE_BAD_DAMPING:
        return set_error(ctx, rc, "Frost damping factor must be ≥ 0 and finite; got %g", (double)damping);
      default:
        return set_error(ctx, rc, "invalid speckle filter kind %d", kind);
    }
  }
  if (data_len == 0) return SD_OK;
  if (!data || !out) return set_error(ctx, SD_ERR_INVALID_ARGUMENT, "null buffer");
  SD_CUDA(ctx, cudaSetDevice(ctx->device));
  const void *d_in;
  void *d_out;
  SD_TRY(stage_in(ctx, "sp.in", data, data_len * sizeof(float), &d_in));
  SD_TRY(stage_out(ctx, "sp.out", out, data_len * sizeof(float), &d_out));
  SD_TRY(speckle_launch(ctx, (const float *)d_in, (float *)d_out, cols, rows, kind, window, enl,
                        damping, ctx->stream));
  SD_TRY(finish_out(ctx, out, d_out, data_len * sizeof(float)));
  return sync(ctx);
}
