// runtime.cu — context lifecycle, error reporting and staging.
#include "runtime.cuh"

#include <nvtx3/nvToolsExt.h>

#include <chrono>
#include <cstdlib>

namespace sd {

namespace {
bool timing_log_on() {
  static const bool on = [] {
    const char *e = std::getenv("SARDINE_B200_TIMING");
    return e && e[0] == '1';
  }();
  return on;
}
double now_s() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}
}  // namespace

StageScope::StageScope(const char *stage) : name(stage), t0(0.0), log(timing_log_on()) {
  nvtxRangePushA(stage);
  if (log) t0 = now_s();
}

StageScope::~StageScope() {
  nvtxRangePop();
  if (log) std::fprintf(stderr, "[timing] %s = %.3f s\n", name, now_s() - t0);
}

void log_newton_hist(const unsigned long long *hist, int n) {
  if (!timing_log_on() || !hist) return;
  unsigned long long total = 0;
  for (int i = 0; i < n; ++i) total += hist[i];
  if (total == 0) return;
  std::string parts;
  for (int i = 1; i < n; ++i)
    if (hist[i]) parts += (parts.empty() ? "" : " ") + std::to_string(i) + "=" + std::to_string(hist[i]);
  std::fprintf(stderr, "[timing] newton_iter_hist (total=%llu): %s\n", total, parts.c_str());
}

int set_error(sd_ctx *ctx, int code, const char *fmt, ...) {
  if (ctx) {
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    ctx->last_error = buf;
  }
  return code;
}

int scratch(sd_ctx *ctx, const char *name, size_t bytes, void **out) {
  if (bytes == 0) bytes = 16;
  auto &b = ctx->scratch[name];
  if (b.bytes < bytes) {
    if (b.p) {
      cudaStreamSynchronize(ctx->stream);
      cudaFree(b.p);
      b.p = nullptr;
      b.bytes = 0;
    }
    cudaError_t e = cudaMalloc(&b.p, bytes);
    if (e != cudaSuccess) {
      cudaGetLastError();
      b.p = nullptr;
      return set_error(ctx, SD_ERR_OUT_OF_MEMORY, "scratch '%s': cudaMalloc(%zu) failed: %s",
                       name, bytes, cudaGetErrorString(e));
    }
    b.bytes = bytes;
  }
  *out = b.p;
  return SD_OK;
}

bool is_device_ptr(const void *p) {
  if (!p) return false;
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

int stage_in(sd_ctx *ctx, const char *name, const void *p, size_t bytes, const void **dev) {
  if (!p) {
    *dev = nullptr;
    return SD_OK;
  }
  if (is_device_ptr(p)) {
    *dev = p;
    return SD_OK;
  }
  void *d = nullptr;
  SD_TRY(scratch(ctx, name, bytes, &d));
  SD_CUDA(ctx, cudaMemcpyAsync(d, p, bytes, cudaMemcpyHostToDevice, ctx->stream));
  *dev = d;
  return SD_OK;
}

int stage_out(sd_ctx *ctx, const char *name, void *p, size_t bytes, void **dev) {
  if (!p) {
    *dev = nullptr;
    return SD_OK;
  }
  if (is_device_ptr(p)) {
    *dev = p;
    return SD_OK;
  }
  return scratch(ctx, name, bytes, dev);
}

int finish_out(sd_ctx *ctx, void *user, const void *dev, size_t bytes) {
  if (!user || user == dev || bytes == 0) return SD_OK;
  SD_CUDA(ctx, cudaMemcpyAsync(user, dev, bytes, cudaMemcpyDeviceToHost, ctx->stream));
  return SD_OK;
}

int sync(sd_ctx *ctx) {
  SD_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  timing_collect(ctx);
  return SD_OK;
}

static thread_local const char *t_pending_name = nullptr;

void timing_begin(sd_ctx *ctx, const char *name) {
  if (!ctx->timing) return;
  sd_ctx::KTime k;
  k.name = name;
  cudaEventCreate(&k.a);
  cudaEventCreate(&k.b);
  cudaEventRecord(k.a, ctx->stream);
  ctx->pending.push_back(k);
  t_pending_name = name;
}

void timing_end(sd_ctx *ctx) {
  if (!ctx->timing || !t_pending_name || ctx->pending.empty()) return;
  cudaEventRecord(ctx->pending.back().b, ctx->stream);
  t_pending_name = nullptr;
}

void timing_collect(sd_ctx *ctx) {
  for (auto &k : ctx->pending) {
    float ms = 0.0f;
    if (cudaEventSynchronize(k.b) == cudaSuccess && cudaEventElapsedTime(&ms, k.a, k.b) == cudaSuccess) {
      auto &acc = ctx->ktimes[k.name];
      acc.first += ms;
      acc.second += 1;
    }
    cudaEventDestroy(k.a);
    cudaEventDestroy(k.b);
  }
  cudaGetLastError();
  ctx->pending.clear();
}

}  // namespace sd

extern "C" {

int sd_abi_version(void) { return SD_ABI_VERSION; }

int sd_ctx_create(int device, sd_ctx **out) {
  if (!out) return SD_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  int n = 0;
  cudaError_t e = cudaGetDeviceCount(&n);
  if (e != cudaSuccess || n == 0) {
    cudaGetLastError();
    return SD_ERR_CUDA;
  }
  if (device < 0 || device >= n) return SD_ERR_INVALID_ARGUMENT;
  if (cudaSetDevice(device) != cudaSuccess) return SD_ERR_CUDA;
  sd_ctx *c = new sd_ctx();
  c->device = device;
  if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreate(&c->ev0) != cudaSuccess || cudaEventCreate(&c->ev1) != cudaSuccess ||
      cudaMalloc(&c->d_flags, 64 * sizeof(int)) != cudaSuccess ||
      cudaMalloc(&c->d_counters, 64 * sizeof(unsigned long long)) != cudaSuccess) {
    cudaGetLastError();
    sd_ctx_destroy(c);
    return SD_ERR_CUDA;
  }
  *out = c;
  return SD_OK;
}

void sd_ctx_destroy(sd_ctx *ctx) {
  if (!ctx) return;
  cudaSetDevice(ctx->device);
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  for (auto &kv : ctx->scratch)
    if (kv.second.p) cudaFree(kv.second.p);
  for (void *p : ctx->pinned) cudaFreeHost(p);
  if (ctx->d_flags) cudaFree(ctx->d_flags);
  if (ctx->d_counters) cudaFree(ctx->d_counters);
  for (auto &kv : ctx->graph_exec) cudaGraphExecDestroy(kv.second.exec);
  if (ctx->tiles_done) cudaEventDestroy(ctx->tiles_done);
  for (int k = 0; k < SD_SIDE_STREAMS; ++k) {
    if (ctx->side[k]) cudaStreamDestroy(ctx->side[k]);
    if (ctx->ev_join[k]) cudaEventDestroy(ctx->ev_join[k]);
  }
  if (ctx->ev_fork) cudaEventDestroy(ctx->ev_fork);
  if (ctx->h_tile_counters) cudaFreeHost(ctx->h_tile_counters);
  if (ctx->h_tile_flags) cudaFreeHost(ctx->h_tile_flags);
  if (ctx->ev0) cudaEventDestroy(ctx->ev0);
  if (ctx->ev1) cudaEventDestroy(ctx->ev1);
  if (ctx->stream) cudaStreamDestroy(ctx->stream);
  delete ctx;
}

const char *sd_last_error(const sd_ctx *ctx) { return ctx ? ctx->last_error.c_str() : ""; }

uint64_t sd_kernel_launches(const sd_ctx *ctx) { return ctx ? ctx->launches : 0; }

void *sd_ctx_stream(sd_ctx *ctx) { return ctx ? (void *)ctx->stream : nullptr; }

int sd_ctx_set_timing(sd_ctx *ctx, int on) {
  if (!ctx) return SD_ERR_INVALID_ARGUMENT;
  cudaStreamSynchronize(ctx->stream);
  sd::timing_collect(ctx);
  ctx->timing = on != 0;
  if (on) ctx->ktimes.clear();
  return SD_OK;
}

int sd_ctx_kernel_times(sd_ctx *ctx, char *names, uint64_t names_len, double *ms, uint64_t *counts,
                        uint64_t max_entries, uint64_t *n_out) {
  if (!ctx || !n_out) return SD_ERR_INVALID_ARGUMENT;
  cudaStreamSynchronize(ctx->stream);
  sd::timing_collect(ctx);
  uint64_t i = 0;
  std::string all;
  for (auto &kv : ctx->ktimes) {
    if (i < max_entries) {
      if (ms) ms[i] = kv.second.first;
      if (counts) counts[i] = kv.second.second;
      all += kv.first;
      all += '\n';
    }
    ++i;
  }
  *n_out = i;
  if (names && names_len > 0) {
    size_t n = std::min<size_t>(all.size(), names_len - 1);
    memcpy(names, all.data(), n);
    names[n] = 0;
  }
  return SD_OK;
}

}  // extern "C"

// The first out-of-bounds gather the checked kernels recorded since the last
// call: word = {site (1 radar image, 2 DEM; 0 none), index, extent, checks
// compiled in (1) or not (0)}; the words are cleared.
extern "C" int sd_debug_bounds(sd_ctx *ctx, uint64_t *word) {
  if (!ctx || !word) return SD_ERR_INVALID_ARGUMENT;
  unsigned long long a[3], b[3];
  if (cudaSetDevice(ctx->device) != cudaSuccess || sd::bounds_read_tc(a) != 0 || sd::bounds_read_tiles(b) != 0)
    return sd::set_error(ctx, SD_ERR_CUDA, "reading the bounds-check words failed");
  const unsigned long long *w = a[0] ? a : b;
  word[0] = w[0];
  word[1] = w[1];
  word[2] = w[2];
  word[3] = SD_BOUNDS_CHECK ? 1 : 0;
  return SD_OK;
}
