// speckle.cu — the five SpeckleKernel filters on sm_100a.
//
// Replaces apply_speckle_filter / SpeckleKernel::apply (sardine/src/speckle.rs:
// 131-180, 218-569, 586-603).  A thread owns SP_ROWS outputs of one column;
// the block's window footprint (tile + halo) is staged once in shared memory,
// out-of-image cells stored as NaN so the reference's "in bounds and finite"
// filter is a single isfinite test.  Window sums are accumulated in f64 in
// the reference's row-major tap order (each tap converted once and added to
// every output of the thread whose window holds it) and cast to f32 exactly
// as speckle.rs:226-240 does, so the f32 filter arithmetic sees the same
// inputs.  The sums are sequential per output, so neither a sliding window
// nor a shuffle tree (which re-associates the adds) would reproduce them.
#include <cuda.h>
#include <cudaTypedefs.h>

#include <cmath>
#include <cstdlib>

#include "geo.cuh"
#include "runtime.cuh"
#include "tiles.cuh"

namespace sd {
namespace {

constexpr int TX = 32, TY = 8;

struct SpParams {
  const float *in;
  float *out;
  int64_t cols, rows;
  int half;
  int kind;
  float enl, damping, cv_n_sq, cv_max_sq;
  int db;                    // write the filtered value in dB (to_db_inplace)
  float db_floor;
  unsigned long long *dbc;   // db: converted, noise-masked counts
  int *err;                  // set when a staging wait timed out (k_speckle_tma)
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
  static_assert(KIND != SD_SPECKLE_REFINED_LEE, "Refined Lee: rl_rows");
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

// ── several outputs per thread ────────────────────────────────────────────────
// A thread owns SP_ROWS outputs of one column.  Each staged tap is converted
// to f64 (and squared) once and added to every one of those outputs whose
// window holds it; an output still receives its taps in the reference's
// row-major order.  A tap the reference skips (outside the image, or not
// finite) adds -0.0, which leaves every IEEE sum unchanged (x + -0.0 == x,
// also for x == +0.0), so the sums are bit-identical to the filtered loop
// while the add sequence stays the same for every lane.
constexpr int SP_ROWS = 2;
// slots of the context's device counters that hold sd_speckle's dB counts
constexpr int SP_DB_COUNTERS = 48;
// slot of the context's device error words for a timed-out staging wait
constexpr int SP_ERR_FLAG = 40;
// largest tile-batch block (Refined Lee holds 2 x 8 directional sums per thread)
constexpr int SP_MAX_THREADS = 512;

template <int R>
struct WinAcc {
  double s[R], q[R];
  int n[R];
};

__device__ __forceinline__ void tap_f64(float v, bool &f, double &d, double &q) {
  f = isfinite(v);
  d = f ? (double)v : -0.0;
  q = f ? d * d : -0.0;
}

// the w taps of one window row into outputs LO..HI
template <int R, int LO, int HI>
__device__ __forceinline__ void win_row(WinAcc<R> &a, const float *row, int w) {
  int nf = 0;
  for (int x = 0; x < w; ++x) {
    bool f;
    double d, q;
    tap_f64(row[x], f, d, q);
    nf += f;
#pragma unroll
    for (int r = LO; r <= HI; ++r) {
      a.s[r] += d;
      a.q[r] += q;
    }
  }
#pragma unroll
  for (int r = LO; r <= HI; ++r) a.n[r] += nf;
}

// outputs lo..hi with a runtime range (predicated adds; ranges strictly
// inside 0..R-1 only, which windows smaller than the thread's rows produce)
template <int R>
__device__ __forceinline__ void win_row_any(int lo, int hi, WinAcc<R> &a, const float *row, int w) {
  int nf = 0;
  for (int x = 0; x < w; ++x) {
    bool f;
    double d, q;
    tap_f64(row[x], f, d, q);
    nf += f;
#pragma unroll
    for (int r = 0; r < R; ++r)
      if (r >= lo && r <= hi) {
        a.s[r] += d;
        a.q[r] += q;
      }
  }
#pragma unroll
  for (int r = 0; r < R; ++r)
    if (r >= lo && r <= hi) a.n[r] += nf;
}

template <int R, int K = 0>
__device__ __forceinline__ void win_prefix(int hi, WinAcc<R> &a, const float *row, int w) {
  if (hi == K) return win_row<R, 0, K>(a, row, w);
  if constexpr (K + 1 < R) win_prefix<R, K + 1>(hi, a, row, w);
}
template <int R, int K = 1>
__device__ __forceinline__ void win_suffix(int lo, WinAcc<R> &a, const float *row, int w) {
  if constexpr (K < R) {
    if (lo == K) return win_row<R, K, R - 1>(a, row, w);
    win_suffix<R, K + 1>(lo, a, row, w);
  }
}

// Window sums of outputs (ly0 + r, lx), r < R, over a (2h+1)^2 window of
// the staged tile (row stride tw).  Window row k (tile row ly0 - h + k)
// feeds outputs max(0, k - 2h) .. min(R - 1, k).
template <int R>
__device__ __forceinline__ void win_stats(const float *tile, int tw, int lx, int ly0, int h, WinAcc<R> &a) {
#pragma unroll
  for (int r = 0; r < R; ++r) a.s[r] = a.q[r] = 0.0, a.n[r] = 0;
  const int w = 2 * h + 1;
  for (int k = 0; k < R + 2 * h; ++k) {
    const int lo = k - 2 * h > 0 ? k - 2 * h : 0, hi = k < R - 1 ? k : R - 1;
    const float *row = tile + (ly0 - h + k) * tw + lx - h;
    if (lo == 0) win_prefix<R>(hi, a, row, w);
    else if (hi == R - 1) win_suffix<R>(lo, a, row, w);
    else win_row_any<R>(lo, hi, a, row, w);
  }
}

// The filter of KIND (not Refined Lee, not Frost) from one output's window
// sums, as speckle_px forms it.
template <int KIND>
__device__ __forceinline__ float filt_stats(float centre, double sum, double sum_sq, int n, const SpCoef &p) {
  if (!finitef(centre) || n == 0) return NAN;
  const double md = sum / (double)n;
  const double vard = maxd_nan(sum_sq / (double)n - md * md, 0.0);
  const float mean = (float)md, var = (float)vard;
  if (KIND == SD_SPECKLE_BOXCAR) return mean;
  if (KIND == SD_SPECKLE_LEE) {
    const float noise_var = mean * mean * p.cv_n_sq;
    const float signal_var = maxf_nan(var - noise_var, 0.0f);
    const float denom = signal_var + noise_var;
    const float k = denom > 0.0f ? signal_var / denom : 0.0f;
    return mean + k * (centre - mean);
  }
  // Gamma-MAP (speckle.rs:348-411)
  const float cv_sq = mean > 0.0f ? var / (mean * mean) : 0.0f;
  if (cv_sq <= p.cv_n_sq) return mean;
  if (cv_sq >= p.cv_max_sq) return centre;
  const float alpha = (1.0f + p.cv_n_sq) / (cv_sq - p.cv_n_sq);
  const float b = (alpha - p.enl - 1.0f) * mean;
  const float disc = b * b + 4.0f * alpha * p.enl * mean * centre;
  return disc >= 0.0f ? ((p.enl - alpha + 1.0f) * mean + sqrtf(disc)) / (2.0f * p.enl) : mean;
}

// Refined Lee masks (speckle.rs:432-457) at compile time.
__host__ __device__ constexpr bool rl_mask(int d, int dy, int dx) {
  if (dy == 0 && dx == 0) return false;
  const int a = dy - dx < 0 ? dx - dy : dy - dx, b = dy + dx < 0 ? -(dy + dx) : dy + dx;
  switch (d) {
    case 0: return dy >= 1 && dy <= 3;
    case 1: return dy >= -3 && dy <= -1;
    case 2: return dx >= 1 && dx <= 3;
    case 3: return dx >= -3 && dx <= -1;
    case 4: return a <= 1 && (dy + dx) >= 1;
    case 5: return a <= 1 && (dy + dx) <= -1;
    case 6: return b <= 1 && (dx - dy) >= 1;
    case 7: return b <= 1 && (dx - dy) <= -1;
  }
  return false;
}
// bit x (dx = x - 3) of window row dy in direction d
__host__ __device__ constexpr uint32_t rl_rowbits(int d, int dy) {
  uint32_t m = 0;
  for (int x = 0; x < 7; ++x)
    if (rl_mask(d, dy, x - 3)) m |= 1u << x;
  return m;
}

// Refined Lee for outputs (ly0 + r, lx), r < R: the 8 directional sums of
// every output in one pass over the R + 6 staged rows (all membership tests
// resolved at compile time), the counts from per-row finite bits.
template <int R>
__device__ __forceinline__ void rl_rows(const float *tile, int tw, int lx, int ly0, const SpCoef &p, float *o) {
  double s[R][8], q[R][8];
  uint32_t fin[R + 6];
#pragma unroll
  for (int r = 0; r < R; ++r)
#pragma unroll
    for (int d = 0; d < 8; ++d) s[r][d] = q[r][d] = 0.0;
#pragma unroll
  for (int k = 0; k < R + 6; ++k) {
    const float *row = tile + (ly0 - 3 + k) * tw + lx - 3;
    uint32_t bits = 0;
#pragma unroll
    for (int x = 0; x < 7; ++x) {
      bool f;
      double dv, qv;
      tap_f64(row[x], f, dv, qv);
      bits |= (uint32_t)f << x;
#pragma unroll
      for (int r = 0; r < R; ++r) {
        const int dy = k - 3 - r;
        if (dy < -3 || dy > 3) continue;
#pragma unroll
        for (int d = 0; d < 8; ++d)
          if (rl_mask(d, dy, x - 3)) {
            s[r][d] += dv;
            q[r][d] += qv;
          }
      }
    }
    fin[k] = bits;
  }
#pragma unroll
  for (int r = 0; r < R; ++r) {
    const float centre = tile[(ly0 + r) * tw + lx];
    if (!finitef(centre)) {
      o[r] = NAN;
      continue;
    }
    float best_cv = INFINITY, best_mean = centre, best_var = 0.0f;
#pragma unroll
    for (int d = 0; d < 8; ++d) {
      int n = 0;
#pragma unroll
      for (int dy = -3; dy <= 3; ++dy) n += __popc(fin[r + 3 + dy] & rl_rowbits(d, dy));
      if (n == 0) continue;
      const double md = s[r][d] / (double)n;
      const double vard = maxd_nan(q[r][d] / (double)n - md * md, 0.0);
      const float mean = (float)md, var = (float)vard;
      if (!(mean > 0.0f)) continue;
      const float cv = var / (mean * mean);
      if (cv < best_cv) {
        best_cv = cv;
        best_mean = mean;
        best_var = var;
      }
    }
    if (!isfinite(best_cv)) {
      o[r] = centre;
    } else {
      const float noise_var = best_mean * best_mean * p.cv_n_sq;
      const float signal_var = maxf_nan(best_var - noise_var, 0.0f);
      const float denom = signal_var + noise_var;
      const float k = denom > 0.0f ? signal_var / denom : 0.0f;
      o[r] = best_mean + k * (centre - best_mean);
    }
  }
}

// SP_ROWS outputs (ly0 + r, lx) of filter KIND from the staged tile.
template <int KIND>
__device__ __forceinline__ void speckle_rows(const float *tile, int tw, int lx, int ly0, int h, const SpCoef &p,
                                             float *o) {
  if (KIND == SD_SPECKLE_REFINED_LEE) {
    rl_rows<SP_ROWS>(tile, tw, lx, ly0, p, o);
  } else if (KIND == SD_SPECKLE_FROST) {  // per-output weights: one output at a time
#pragma unroll
    for (int r = 0; r < SP_ROWS; ++r) o[r] = speckle_px<SD_SPECKLE_FROST>(tile, tw, lx, ly0 + r, h, p);
  } else {
    WinAcc<SP_ROWS> a;
    win_stats<SP_ROWS>(tile, tw, lx, ly0, h, a);
#pragma unroll
    for (int r = 0; r < SP_ROWS; ++r) o[r] = filt_stats<KIND>(tile[(ly0 + r) * tw + lx], a.s[r], a.q[r], a.n[r], p);
  }
}

template <int KIND>
__global__ void __launch_bounds__(TX *TY) k_speckle(SpParams p) {
  extern __shared__ float tile[];
  const int h = p.half;
  const int tw = TX + 2 * h, th = TY * SP_ROWS + 2 * h;
  const int64_t c0 = (int64_t)blockIdx.x * TX - h, r0 = (int64_t)blockIdx.y * (TY * SP_ROWS) - h;
  for (int k = threadIdx.y * TX + threadIdx.x; k < tw * th; k += TX * TY) {
    int ty = k / tw, tx = k % tw;
    int64_t rr = r0 + ty, cc = c0 + tx;
    float v = NAN;
    if (rr >= 0 && cc >= 0 && rr < p.rows && cc < p.cols) v = __ldg(p.in + rr * p.cols + cc);
    tile[k] = v;
  }
  __syncthreads();
  // this thread: column c, rows r .. r + SP_ROWS - 1 (threads past the
  // raster's edge stay for the block's count reduction)
  const int64_t c = (int64_t)blockIdx.x * TX + threadIdx.x;
  const int64_t r = (int64_t)blockIdx.y * (TY * SP_ROWS) + threadIdx.y * SP_ROWS;
  unsigned ncv = 0, nnm = 0;
  if (c < p.cols && r < p.rows) {
    const SpCoef cf{p.enl, p.damping, p.cv_n_sq, p.cv_max_sq};
    float o[SP_ROWS];
    speckle_rows<KIND>(tile, tw, threadIdx.x + h, threadIdx.y * SP_ROWS + h, h, cf, o);
#pragma unroll
    for (int k = 0; k < SP_ROWS; ++k)
      if (r + k < p.rows) {
        float v = o[k];
        if (p.db) {  // the dB conversion of the filtered raster, in this epilogue
          int dc;
          v = db_value(v, p.db_floor, &dc);
          ncv += dc == 0;
          nnm += dc == 1;
        }
        p.out[(r + k) * p.cols + c] = v;
      }
  }
  if (p.db) {  // the block's counts: warp sums, then one global atomic per block
    __shared__ unsigned s_db[2];
    const int tid = threadIdx.y * TX + threadIdx.x;
    if (tid == 0) s_db[0] = s_db[1] = 0;
    __syncthreads();
    ncv = __reduce_add_sync(0xffffffffu, ncv);
    nnm = __reduce_add_sync(0xffffffffu, nnm);
    if ((tid & 31) == 0) {
      atomicAdd(&s_db[0], ncv);
      atomicAdd(&s_db[1], nnm);
    }
    __syncthreads();
    if (tid == 0) {
      if (s_db[0]) atomicAdd(p.dbc, (unsigned long long)s_db[0]);
      if (s_db[1]) atomicAdd(p.dbc + 1, (unsigned long long)s_db[1]);
    }
  }
}

// ── the same filter with the window staged by the tensor-memory accelerator ─
// For rasters whose rows are 16-byte aligned (cols % 4 == 0, base 16-byte
// aligned) one 2-D `cp.async.bulk.tensor` load stages the block's window.
// The window's first column is rounded down to a multiple of 4 floats (the
// copy's x coordinate must be a 16-byte multiple) and the box is widened to
// bw columns to cover the remainder; cells outside the raster arrive as NaN
// (the tensor map's fill mode), exactly the "outside the image" cell the
// filters skip.  The copy completes on a shared-memory mbarrier; the wait is
// bounded and reports a timeout in *p.err instead of spinning forever.

// true once phase `phase` of the mbarrier at shared address `bar` has
// completed, false after `limit` polls
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t phase, uint32_t limit) {
  for (uint32_t it = 0; it < limit; ++it) {
    uint32_t done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(bar), "r"(phase)
        : "memory");
    if (done) return true;
    if (it > 32) __nanosleep(256);
  }
  return false;
}

template <int KIND>
__global__ void __launch_bounds__(TX *TY) k_speckle_tma(SpParams p, const __grid_constant__ CUtensorMap tm, int bw) {
  extern __shared__ __align__(128) float tile[];
  __shared__ __align__(8) unsigned long long mbar;
  const int h = p.half, th = TY * SP_ROWS + 2 * h;
  const int tid = threadIdx.y * TX + threadIdx.x;
  const int x = (int)blockIdx.x * TX - h;          // the window's first column (may be negative)
  const int x0 = x - (((x % 4) + 4) % 4);          // rounded down to 4 floats
  const int y0 = (int)blockIdx.y * (TY * SP_ROWS) - h;
  const uint32_t bar = (uint32_t)__cvta_generic_to_shared(&mbar);
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(bar), "r"(1) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  __syncthreads();
  if (tid == 0) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(bar), "r"(bw * th * 4)
                 : "memory");
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];\n" ::
            "r"((uint32_t)__cvta_generic_to_shared(tile)),
        "l"(reinterpret_cast<uint64_t>(&tm)), "r"(x0), "r"(y0), "r"(bar)
        : "memory");
  }
  if (!mbar_wait(bar, 0, 1u << 22)) {  // never expected: the copy is a few KB
    if (tid == 0) atomicExch(p.err, 1);
    return;
  }
  // this thread: column c, rows r .. r + SP_ROWS - 1
  const int64_t c = (int64_t)blockIdx.x * TX + threadIdx.x;
  const int64_t r = (int64_t)blockIdx.y * (TY * SP_ROWS) + threadIdx.y * SP_ROWS;
  unsigned ncv = 0, nnm = 0;
  if (c < p.cols && r < p.rows) {
    const SpCoef cf{p.enl, p.damping, p.cv_n_sq, p.cv_max_sq};
    float o[SP_ROWS];
    speckle_rows<KIND>(tile, bw, threadIdx.x + h + (x - x0), threadIdx.y * SP_ROWS + h, h, cf, o);
#pragma unroll
    for (int k = 0; k < SP_ROWS; ++k)
      if (r + k < p.rows) {
        float v = o[k];
        if (p.db) {
          int dc;
          v = db_value(v, p.db_floor, &dc);
          ncv += dc == 0;
          nnm += dc == 1;
        }
        p.out[(r + k) * p.cols + c] = v;
      }
  }
  if (p.db) {  // the block's counts, as k_speckle forms them
    __shared__ unsigned s_db[2];
    if (tid == 0) s_db[0] = s_db[1] = 0;
    __syncthreads();
    ncv = __reduce_add_sync(0xffffffffu, ncv);
    nnm = __reduce_add_sync(0xffffffffu, nnm);
    if ((tid & 31) == 0) {
      atomicAdd(&s_db[0], ncv);
      atomicAdd(&s_db[1], nnm);
    }
    __syncthreads();
    if (tid == 0) {
      if (s_db[0]) atomicAdd(p.dbc, (unsigned long long)s_db[0]);
      if (s_db[1]) atomicAdd(p.dbc + 1, (unsigned long long)s_db[1]);
    }
  }
}

// ── batched form: many tiles, each a halo'd geocoded raster ──────────────────
// Item = one tx x ty block (the launch's block shape, chosen by the tile
// autotuner) of one tile's output.  The block stages its window from the
// tile's halo'd raster (cells outside it are NaN, which the filters skip like
// out-of-image cells), filters the data plane with the tile's kind (or
// copies it when kind < 0) and crops cos(LIA) and the mask.
// Where one work item's window sits: its job, block position and the
// staged footprint (rows r0.., columns c0.. of the job's halo'd raster).
struct SpItem {
  const SpJob *jb;
  int64_t tr, tc, r0, c0, in_cols, in_rows;
  int h, tw, th;
};

__device__ __forceinline__ SpItem sp_item(const SpWork &w, uint64_t item, int bx, int by) {
  int lo = 0, hi = w.n_jobs;
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (w.pre[mid] <= item) lo = mid;
    else hi = mid;
  }
  SpItem it;
  it.jb = &w.jobs[lo];
  const SpJob &jb = *it.jb;
  const uint64_t li = item - w.pre[lo];
  const int64_t nbx = (jb.cols + bx - 1) / bx;
  it.tr = (int64_t)li / nbx;
  it.tc = (int64_t)li % nbx;
  it.h = jb.kind >= 0 ? jb.half : 0;
  it.tw = bx + 2 * it.h;
  it.th = by * SP_ROWS + 2 * it.h;
  it.in_cols = jb.cols + 2 * jb.halo;
  it.in_rows = jb.rows + 2 * jb.halo;
  // output (r, c) is input (r + halo, c + halo); the block covers bx
  // columns and by * SP_ROWS rows
  it.c0 = it.tc * bx + jb.halo - it.h;
  it.r0 = it.tr * by * SP_ROWS + jb.halo - it.h;
  return it;
}

// Issues the item's window into buf: asynchronous 4-byte copies
// (cp.async, completed by the caller's wait) for cells inside the raster,
// plain NaN stores for the rest.
__device__ __forceinline__ void sp_stage_async(const SpItem &it, float *buf, int tid, int nt) {
  const float *in = it.jb->in;
  for (int k = tid; k < it.tw * it.th; k += nt) {
    const int ty = k / it.tw, tx = k % it.tw;
    const int64_t rr = it.r0 + ty, cc = it.c0 + tx;
    if (rr >= 0 && cc >= 0 && rr < it.in_rows && cc < it.in_cols) {
      const unsigned sa = (unsigned)__cvta_generic_to_shared(buf + k);
      asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(sa), "l"(in + rr * it.in_cols + cc)
                   : "memory");
    } else {
      buf[k] = NAN;
    }
  }
}

// Items are strided over a persistent grid; each block double-buffers its
// window: the next item's copies are in flight while the current item is
// filtered.
__global__ void __launch_bounds__(SP_MAX_THREADS) k_speckle_tiles(const SpWork *__restrict__ wp) {
  extern __shared__ float smem[];
  const SpWork w = *wp;
  const int bx = (int)blockDim.x, by = (int)blockDim.y, nt = bx * by;
  const int tid = threadIdx.y * bx + threadIdx.x;
  const int buf_floats = (bx + 2 * SP_MAX_HALF) * (by * SP_ROWS + 2 * SP_MAX_HALF);
  const uint64_t total = w.pre[w.n_jobs];
  uint64_t item = blockIdx.x;
  if (item < total) sp_stage_async(sp_item(w, item, bx, by), smem, tid, nt);
  asm volatile("cp.async.commit_group;\n" ::: "memory");
  for (int b = 0; item < total; item += gridDim.x, b ^= 1) {
    const SpItem it = sp_item(w, item, bx, by);
    const uint64_t next = item + gridDim.x;
    if (next < total) sp_stage_async(sp_item(w, next, bx, by), smem + (b ^ 1) * buf_floats, tid, nt);
    asm volatile("cp.async.commit_group;\n" ::: "memory");
    asm volatile("cp.async.wait_group 1;\n" ::: "memory");  // this item's copies have landed
    __syncthreads();
    const float *tile = smem + b * buf_floats;
    const SpJob &jb = *it.jb;
    const int h = it.h, tw = it.tw;
    // this thread: column c, rows r .. r + SP_ROWS - 1
    const int64_t c = it.tc * bx + threadIdx.x, r = (it.tr * by + threadIdx.y) * SP_ROWS;
    if (c < jb.cols && r < jb.rows) {
      // the cropped cos(LIA) and mask travel while the filter computes
      float cz[SP_ROWS];
      uint8_t mz[SP_ROWS];
#pragma unroll
      for (int k = 0; k < SP_ROWS; ++k) {
        const int64_t ii = (r + k + jb.halo) * it.in_cols + (c + jb.halo);
        const bool in = r + k < jb.rows;
        cz[k] = in && jb.cos_out ? __ldg(jb.cos_in + ii) : 0.0f;
        mz[k] = in && jb.mask_out ? __ldg(jb.mask_in + ii) : 0;
      }
      const SpCoef cf{jb.enl, jb.damping, jb.cv_n_sq, jb.cv_max_sq};
      const int lx = threadIdx.x + h, ly = threadIdx.y * SP_ROWS + h;
      float o[SP_ROWS];
      switch (jb.kind) {
        case SD_SPECKLE_BOXCAR: speckle_rows<SD_SPECKLE_BOXCAR>(tile, tw, lx, ly, h, cf, o); break;
        case SD_SPECKLE_LEE: speckle_rows<SD_SPECKLE_LEE>(tile, tw, lx, ly, h, cf, o); break;
        case SD_SPECKLE_FROST: speckle_rows<SD_SPECKLE_FROST>(tile, tw, lx, ly, h, cf, o); break;
        case SD_SPECKLE_GAMMA_MAP: speckle_rows<SD_SPECKLE_GAMMA_MAP>(tile, tw, lx, ly, h, cf, o); break;
        case SD_SPECKLE_REFINED_LEE: speckle_rows<SD_SPECKLE_REFINED_LEE>(tile, tw, lx, ly, h, cf, o); break;
        default:
#pragma unroll
          for (int k = 0; k < SP_ROWS; ++k) o[k] = tile[(ly + k) * tw + lx];
      }
#pragma unroll
      for (int k = 0; k < SP_ROWS; ++k) {
        if (r + k >= jb.rows) break;
        const int64_t oi = (r + k) * jb.cols + c;
        jb.out[oi] = o[k];
        if (jb.cos_out) jb.cos_out[oi] = cz[k];
        if (jb.mask_out) jb.mask_out[oi] = mz[k];
      }
    }
    __syncthreads();  // every thread is done with this buffer before it is refilled
  }
  asm volatile("cp.async.wait_group 0;\n" ::: "memory");
}

}  // namespace

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
  return tx >= 8 && ty >= 1 && tx <= 256 && tx * ty <= SP_MAX_THREADS && (tx * ty) % 32 == 0;
}

int speckle_tiles_launch(sd_ctx *ctx, const SpWork *d_work, uint64_t total, bool full_grid, int tx, int ty) {
  // two window buffers (double-buffered staging)
  const size_t smem = 2 * (size_t)(tx + 2 * SP_MAX_HALF) * (ty * SP_ROWS + 2 * SP_MAX_HALF) * sizeof(float);
  const unsigned g = persistent_grid(k_speckle_tiles, tx * ty, smem, full_grid ? ~0ull : total);
  SD_TIMED_BEGIN(ctx, "k_speckle_tiles");
  k_speckle_tiles<<<g, dim3(tx, ty), smem, ctx->stream>>>(d_work);
  SD_LAUNCHED(ctx);
  return SD_OK;
}

uint64_t speckle_tile_items(const SpJob &j, int tx, int ty) {
  return (uint64_t)((j.cols + tx - 1) / tx) * (uint64_t)((j.rows + ty * SP_ROWS - 1) / (ty * SP_ROWS));
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
// The driver's tensor-map encoder, looked up once through the runtime (no
// link against libcuda).
PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = [] {
    void *f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      f = nullptr;
    return reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(f);
  }();
  return fn;
}

// SARDINE_B200_SPECKLE_TMA=0 keeps every call on the scalar staging.
bool tma_enabled() {
  static const bool on = [] {
    const char *e = std::getenv("SARDINE_B200_SPECKLE_TMA");
    return !(e && e[0] == '0');
  }();
  return on;
}

// A 2-D map of the f32 raster (cols x rows, row pitch cols floats) with a
// bw x th box, cells outside the raster filled with NaN.
bool encode_window_map(CUtensorMap *tm, const float *d, uint64_t cols, uint64_t rows, int bw, int th) {
  const PFN_cuTensorMapEncodeTiled_v12000 enc = tensor_map_encoder();
  if (!enc) return false;
  const cuuint64_t dims[2] = {cols, rows};
  const cuuint64_t strides[1] = {cols * sizeof(float)};
  const cuuint32_t box[2] = {(cuuint32_t)bw, (cuuint32_t)th};
  const cuuint32_t estr[2] = {1, 1};
  return enc(tm, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<float *>(d), dims, strides, box, estr,
             CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
             CU_TENSOR_MAP_FLOAT_OOB_FILL_NAN_REQUEST_ZERO_FMA) == CUDA_SUCCESS;
}

int speckle_launch(sd_ctx *ctx, const float *d_in, float *d_out, uint64_t cols, uint64_t rows,
                   int kind, uint64_t window, float enl, float damping, cudaStream_t st) {
  if (cols == 0 || rows == 0) return SD_OK;
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
  p.db = ctx->db_out;
  p.db_floor = ctx->db_floor;
  p.dbc = ctx->d_counters + SP_DB_COUNTERS;
  if (p.db) SD_CUDA(ctx, cudaMemsetAsync(p.dbc, 0, 2 * sizeof(unsigned long long), st));
  p.err = ctx->d_flags + SP_ERR_FLAG;
  SD_CUDA(ctx, cudaMemsetAsync(p.err, 0, sizeof(int), st));
  const int h = p.half;
  size_t smem = (size_t)(TX + 2 * h) * (TY * SP_ROWS + 2 * h) * sizeof(float);
  if (smem > 200 * 1024)
    return set_error(ctx, SD_ERR_INVALID_ARGUMENT, "speckle window %llu too large", (unsigned long long)win);
  dim3 grid((unsigned)((cols + TX - 1) / TX), (unsigned)((rows + TY * SP_ROWS - 1) / (TY * SP_ROWS)));
  dim3 block(TX, TY);
  // the TMA-staged form where the raster's rows are 16-byte aligned and the
  // widened window fits one box (at most 256 per dimension)
  const int bw = (TX + 2 * h + 3 + 3) & ~3, th = TY * SP_ROWS + 2 * h;
  CUtensorMap tm;
  if (tma_enabled() && cols % 4 == 0 && (reinterpret_cast<uintptr_t>(d_in) & 15) == 0 && bw <= 256 && th <= 256 &&
      cols < (1ull << 32) && rows < (1ull << 31) && encode_window_map(&tm, d_in, cols, rows, bw, th)) {
    const size_t tsmem = (size_t)bw * th * sizeof(float);
    switch (kind) {
#define SD_LAUNCH_SPECKLE_TMA(K)                                                              \
  case K:                                                                                     \
    if (tsmem > 48 * 1024)                                                                    \
      SD_CUDA(ctx, cudaFuncSetAttribute(k_speckle_tma<K>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)tsmem)); \
    SD_TIMED_BEGIN(ctx, "k_speckle_tma_" #K);                                            \
    k_speckle_tma<K><<<grid, block, tsmem, st>>>(p, tm, bw);                                  \
    break;
      SD_LAUNCH_SPECKLE_TMA(SD_SPECKLE_BOXCAR)
      SD_LAUNCH_SPECKLE_TMA(SD_SPECKLE_LEE)
      SD_LAUNCH_SPECKLE_TMA(SD_SPECKLE_FROST)
      SD_LAUNCH_SPECKLE_TMA(SD_SPECKLE_GAMMA_MAP)
      SD_LAUNCH_SPECKLE_TMA(SD_SPECKLE_REFINED_LEE)
#undef SD_LAUNCH_SPECKLE_TMA
    }
    SD_LAUNCHED(ctx);
    return SD_OK;
  }
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
  SD_STAGE("speckle");
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
  if (ctx->db_out) {
    unsigned long long c[2];
    SD_CUDA(ctx, cudaMemcpyAsync(c, ctx->d_counters + SP_DB_COUNTERS, sizeof c, cudaMemcpyDeviceToHost,
                                 ctx->stream));
    SD_TRY(sync(ctx));
    SD_TRY(db_finish(ctx, (const float *)d_out, data_len, c[0], c[1]));
  }
  SD_TRY(finish_out(ctx, out, d_out, data_len * sizeof(float)));
  int err = 0;
  SD_CUDA(ctx, cudaMemcpyAsync(&err, ctx->d_flags + SP_ERR_FLAG, sizeof err, cudaMemcpyDeviceToHost, ctx->stream));
  SD_TRY(sync(ctx));
  if (err) return set_error(ctx, SD_ERR_TIMEOUT, "speckle: a window's staging copy did not complete");
  return SD_OK;
}
