// Pre-TC multilook (apply_multilook, scene_prep.rs:1060-1160): the NaN-aware
// A x R boxcar of sigma0 and NESZ, one thread per output pixel.  HBM-bound:
// every input pixel is read once (8 B: sigma0 + NESZ), every output written
// once (8 B).  Sums are f64 in the reference's order (azimuth outer, range
// inner), so the output equals a sequential evaluation bit for bit.  The
// geometry updates (spacing, near range, azimuth start) are host arithmetic
// (sardine_b200.apply_multilook).
#include "runtime.cuh"

namespace sd {
namespace {

__global__ void k_multilook(const float *__restrict__ d, const float *__restrict__ nz, uint64_t in_s,
                            uint32_t rl, uint32_t al, float *__restrict__ od, float *__restrict__ onz,
                            uint64_t out_l, uint64_t out_s) {
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= out_l * out_s) return;
  const uint64_t ol = i / out_s, os = i - ol * out_s;
  double sum = 0.0, sum_n = 0.0;
  uint32_t cnt = 0;
  for (uint32_t da = 0; da < al; ++da) {
    const uint64_t row = (ol * al + da) * in_s + os * rl;
    for (uint32_t dr = 0; dr < rl; ++dr) {
      const float v = __ldg(d + row + dr);
      if (v == v) {
        sum += (double)v;
        if (nz) sum_n += (double)__ldg(nz + row + dr);
        ++cnt;
      }
    }
  }
  od[i] = cnt ? (float)(sum / (double)cnt) : NAN;
  if (onz) onz[i] = cnt ? (float)(sum_n / (double)cnt) : NAN;
}

}  // namespace
}  // namespace sd

using namespace sd;

extern "C" int sd_multilook(sd_ctx *ctx, const float *data, const float *nesz, uint64_t lines, uint64_t samples,
                            uint32_t range_looks, uint32_t azimuth_looks, float *out_data, float *out_nesz) {
  SD_STAGE("multilook");
  if (!ctx) return SD_ERR_INVALID_ARGUMENT;
  if (range_looks == 0 || azimuth_looks == 0)
    return set_error(ctx, SD_ERR_INVALID_ARGUMENT, "multilook factors must be >= 1 (range=%u, azimuth=%u)",
                     range_looks, azimuth_looks);
  const uint64_t ol = lines / azimuth_looks, os = samples / range_looks;
  if (ol == 0 || os == 0)
    return set_error(ctx, SD_ERR_INVALID_ARGUMENT,
                     "multilook (%ux%u) is larger than image dimensions (%llu samples x %llu lines)", range_looks,
                     azimuth_looks, (unsigned long long)samples, (unsigned long long)lines);
  if (!data || !out_data || (nesz && !out_nesz)) return set_error(ctx, SD_ERR_INVALID_ARGUMENT, "null buffer");
  SD_CUDA(ctx, cudaSetDevice(ctx->device));
  const void *dd, *dn = nullptr;
  void *od, *on = nullptr;
  SD_TRY(stage_in(ctx, "ml.data", data, lines * samples * 4, &dd));
  if (nesz) SD_TRY(stage_in(ctx, "ml.nesz", nesz, lines * samples * 4, &dn));
  SD_TRY(stage_out(ctx, "ml.out", out_data, ol * os * 4, &od));
  if (nesz) SD_TRY(stage_out(ctx, "ml.onz", out_nesz, ol * os * 4, &on));
  SD_TIMED_BEGIN(ctx, "k_multilook");
  k_multilook<<<(unsigned)((ol * os + 255) / 256), 256, 0, ctx->stream>>>(
      (const float *)dd, (const float *)dn, samples, range_looks, azimuth_looks, (float *)od, (float *)on, ol, os);
  SD_LAUNCHED(ctx);
  SD_TRY(finish_out(ctx, out_data, od, ol * os * 4));
  if (nesz) SD_TRY(finish_out(ctx, out_nesz, on, ol * os * 4));
  return sync(ctx);
}
