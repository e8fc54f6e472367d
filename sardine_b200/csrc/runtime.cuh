// runtime.cuh — context, scratch memory and host/device staging shared by the
// entry points of libsardine_b200.
#pragma once

#include <cuda_runtime.h>

#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>
#include <unordered_map>
#include <vector>

#include "../../include/sardine_b200.h"

// Streams the per-tile launches of a batch spread over (tiles largest first,
// each to the least loaded stream), so that small tiles run side by side.
// 8 measured the same as 4 on the served and tile-batch workloads.
#ifndef SD_SIDE_STREAMS
#define SD_SIDE_STREAMS 4
#endif

struct sd_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  std::string last_error;
  uint64_t launches = 0;
  struct Buf {
    void *p = nullptr;
    size_t bytes = 0;
  };
  std::unordered_map<std::string, Buf> scratch;  // grow-only named device buffers
  std::vector<void *> pinned;                    // grow-only pinned staging buffers
  int *d_flags = nullptr;                        // device-side error words
  // optional per-kernel timing: events recorded around every launch
  bool timing = false;
  struct KTime {
    std::string name;
    cudaEvent_t a, b;
  };
  std::vector<KTime> pending;
  std::unordered_map<std::string, std::pair<double, uint64_t>> ktimes;  // ms, launches
  unsigned long long *d_counters = nullptr;      // device-side counters (64 slots)
  // batched tiles (sd_tc_tiles_*): the last launch's results land here
  cudaEvent_t tiles_done = nullptr;
  unsigned long long *h_tile_counters = nullptr;  // pinned, tile_cap x 32
  int *h_tile_flags = nullptr;                    // pinned, tile_cap x 8
  uint64_t tile_cap = 0, tile_n = 0;
  std::vector<sd_geocoded_info> tile_info;
  bool tiles_pending = false;
  // launch shapes of the tile stages (set by the tile autotuner)
  int sp_tx = 32, sp_ty = 8;  // speckle/crop block
  int main_cps = 0;           // k_main_batch CTAs per SM (0: as many as fit; -1: per-tile
                              // parameter launches over the side streams)
  cudaStream_t side[SD_SIDE_STREAMS] = {};
  cudaEvent_t ev_fork = nullptr, ev_join[SD_SIDE_STREAMS] = {};
  // CUDA graphs of the tile stages (persistent kernels over fixed work tables)
  bool graphs = false;
  struct GraphRec {
    cudaGraphExec_t exec;
    const void *tag;    // address of the work table the graph reads
    uint64_t launches;  // kernels per replay
  };
  std::unordered_map<int, GraphRec> graph_exec;
  // dB output fused into the producing kernels (sd_ctx_set_db_output): the
  // terrain correction and the speckle filter write 10 log10 v, and the
  // counts and statistics of the last such call are kept for sd_ctx_db_result
  bool db_out = false;
  float db_floor = 0.0f;
  bool db_valid = false;
  uint64_t db_counts[2] = {0, 0};  // converted, noise-masked
  float db_stats[4] = {0.0f, 0.0f, 0.0f, 0.0f};
};

namespace sd {

int set_error(sd_ctx *ctx, int code, const char *fmt, ...);

// One call of an entry point as a stage of the reference's pipeline, under
// the reference's [timing] stage name (run.rs:54-60, scene_prep.rs:680-700):
// an NVTX range for profilers (nvtx3 is header-only and costs nothing when
// no tool is attached) and, when SARDINE_B200_TIMING=1 is set, the
// reference's "[timing] <stage> = <s> s" line on stderr when the call
// returns (wall clock; the entry points synchronise before returning).
struct StageScope {
  const char *name;
  double t0;
  bool log;
  explicit StageScope(const char *stage);
  ~StageScope();
};
// The reference's Newton histogram line (run.rs:319-339), when logging.
void log_newton_hist(const unsigned long long *hist, int n);

// ── debug bounds checks ─────────────────────────────────────────────────────
// Built with -DSD_BOUNDS_CHECK=1, every gather of the radar image and the
// DEM in the terrain-correction kernels tests its index against the
// buffer's extent.  The first violation in a translation unit is recorded
// in that unit's error word {site, index, extent} and the access is skipped
// (the value reads as NaN): a faulty index shows up as a status the host
// reads (sd_debug_bounds), never as a memory fault.  Default builds compile
// the checks out.
#ifndef SD_BOUNDS_CHECK
#define SD_BOUNDS_CHECK 0
#endif
enum BoundsSite : int { BS_IMAGE = 1, BS_DEM = 2 };
#if SD_BOUNDS_CHECK
static __device__ unsigned long long sd_bounds_word[3];
__device__ __noinline__ static bool sd_bounds_fail(int site, unsigned long long i, unsigned long long n) {
  if (atomicCAS(&sd_bounds_word[0], 0ull, (unsigned long long)site) == 0ull) {
    sd_bounds_word[1] = i;
    sd_bounds_word[2] = n;
  }
  return false;
}
#define SD_IN_BOUNDS(site, i, n) \
  ((unsigned long long)(i) < (unsigned long long)(n) || ::sd::sd_bounds_fail((site), (i), (n)))
// the unit's word, read and cleared by the host (one per checked unit)
#define SD_BOUNDS_ACCESSOR(fn)                                                  \
  int fn(unsigned long long out[3]) {                                           \
    if (cudaMemcpyFromSymbol(out, sd_bounds_word, 3 * sizeof(unsigned long long)) != cudaSuccess) return -1; \
    const unsigned long long z[3] = {0, 0, 0};                                  \
    return cudaMemcpyToSymbol(sd_bounds_word, z, sizeof z) == cudaSuccess ? 0 : -1; \
  }
#else
#define SD_IN_BOUNDS(site, i, n) true
#define SD_BOUNDS_ACCESSOR(fn) \
  int fn(unsigned long long out[3]) { \
    out[0] = out[1] = out[2] = 0;     \
    return 0;                         \
  }
#endif
int bounds_read_tc(unsigned long long out[3]);
int bounds_read_tiles(unsigned long long out[3]);

// to_db_inplace (export.rs:80-90) on one value: NaN stays NaN (*cls -1);
// v <= floor_lin becomes NaN (*cls 1, noise-masked); anything else becomes
// 10 log10 v (*cls 0, converted).
__device__ __forceinline__ float db_value(float v, float floor_lin, int *cls) {
  if (v != v) {
    *cls = -1;
    return v;
  }
  if (v <= floor_lin) {
    *cls = 1;
    return __int_as_float(0x7fc00000);
  }
  *cls = 0;
  return 10.0f * log10f(v);
}

// compute_db_stats (run.rs:63-97) of the device raster d[0..n) into st:
// {min, max, mean, median}, NaN when no value is finite (export.cu).
int db_stats_device(sd_ctx *ctx, const float *d, uint64_t n, float st[4]);
// After a producing call that wrote dB values: the counts (from the
// kernels' counters) and the statistics of the device raster d_out.
int db_finish(sd_ctx *ctx, const float *d_out, uint64_t n, uint64_t converted, uint64_t masked);
#define SD_STAGE(stage) ::sd::StageScope sd_stage_scope__(stage)

#define SD_CUDA(ctx, call)                                                               \
  do {                                                                                   \
    cudaError_t e__ = (call);                                                            \
    if (e__ != cudaSuccess)                                                              \
      return ::sd::set_error((ctx), e__ == cudaErrorMemoryAllocation ? SD_ERR_OUT_OF_MEMORY \
                                                                     : SD_ERR_CUDA,      \
                             "%s failed: %s (%s:%d)", #call, cudaGetErrorString(e__),    \
                             __FILE__, __LINE__);                                        \
  } while (0)

// Bracket a launch with SD_TIMED_BEGIN(ctx, "name") ... SD_LAUNCHED(ctx).
#define SD_TIMED_BEGIN(ctx, nm) ::sd::timing_begin((ctx), (nm))

#define SD_LAUNCHED(ctx)                                                                  \
  do {                                                                                   \
    (ctx)->launches++;                                                                   \
    ::sd::timing_end(ctx);                                                               \
    cudaError_t e__ = cudaGetLastError();                                                \
    if (e__ != cudaSuccess)                                                              \
      return ::sd::set_error((ctx), SD_ERR_CUDA, "kernel launch failed: %s (%s:%d)",     \
                             cudaGetErrorString(e__), __FILE__, __LINE__);               \
  } while (0)

#define SD_TRY(expr)            \
  do {                          \
    int r__ = (expr);           \
    if (r__ != SD_OK) return r__; \
  } while (0)

// Named grow-only device scratch buffer.
int scratch(sd_ctx *ctx, const char *name, size_t bytes, void **out);
template <class T>
int scratch_t(sd_ctx *ctx, const char *name, size_t count, T **out) {
  void *p = nullptr;
  int rc = scratch(ctx, name, count * sizeof(T), &p);
  *out = (T *)p;
  return rc;
}

// True when `p` is device (or managed) memory usable by kernels on ctx->device.
bool is_device_ptr(const void *p);

// Input view: device pointer to `bytes` of data, staged through scratch
// `name` when the caller passed host memory.
int stage_in(sd_ctx *ctx, const char *name, const void *p, size_t bytes, const void **dev);
// Output view: a device buffer for `bytes`; after the kernels run call
// finish_out to copy back when the caller passed host memory.
int stage_out(sd_ctx *ctx, const char *name, void *p, size_t bytes, void **dev);
int finish_out(sd_ctx *ctx, void *user, const void *dev, size_t bytes);
int sync(sd_ctx *ctx);
void timing_begin(sd_ctx *ctx, const char *name);
void timing_end(sd_ctx *ctx);
void timing_collect(sd_ctx *ctx);

inline unsigned grid_for(size_t n, unsigned block) {
  size_t g = (n + block - 1) / block;
  return (unsigned)(g == 0 ? 1 : g);
}

// Grid of a persistent kernel: the CTAs the current device keeps resident
// at once (occupancy x SMs), or fewer when there are fewer work blocks.
template <class K>
unsigned persistent_grid(K kernel, int threads, size_t smem, uint64_t blocks) {
  int dev = 0, sms = 1, occ = 1;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kernel, threads, smem) != cudaSuccess || occ < 1)
    occ = 1;
  uint64_t g = (uint64_t)occ * (uint64_t)(sms < 1 ? 1 : sms);
  if (blocks < g) g = blocks;
  return (unsigned)(g == 0 ? 1 : g);
}

}  // namespace sd
