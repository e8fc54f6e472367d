// diag.cu — FP64 / FP32 FMA-chain throughput probes.  The roofline of the
// terrain correction is the FP64 pipe, whose peak is not among the measured
// HBM / tensor figures; this measures it on the device at run time.
#include "crmath.cuh"
#include "runtime.cuh"

namespace sd {
namespace {

template <class T>
__global__ void k_fma_chain(T *out, int iters, T a, T b) {
  // 8 independent chains per thread keep the FMA pipe busy.
  T x0 = (T)threadIdx.x, x1 = x0 + (T)1, x2 = x0 + (T)2, x3 = x0 + (T)3;
  T x4 = x0 + (T)4, x5 = x0 + (T)5, x6 = x0 + (T)6, x7 = x0 + (T)7;
  for (int i = 0; i < iters; ++i) {
    x0 = fma(x0, a, b); x1 = fma(x1, a, b); x2 = fma(x2, a, b); x3 = fma(x3, a, b);
    x4 = fma(x4, a, b); x5 = fma(x5, a, b); x6 = fma(x6, a, b); x7 = fma(x7, a, b);
  }
  T s = x0 + x1 + x2 + x3 + x4 + x5 + x6 + x7;
  if (s == (T)-12345.0) out[0] = s;  // keeps the chains live
}

template <class T>
int measure(sd_ctx *ctx, int iters, double *tflops) {
  SD_CUDA(ctx, cudaSetDevice(ctx->device));
  int sms = 0;
  SD_CUDA(ctx, cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx->device));
  T *d;
  SD_TRY(scratch_t(ctx, "diag.out", 16, &d));
  const int block = 256, grid = sms * 8;
  SD_TIMED_BEGIN(ctx, "k_fma_chain<T>");
  k_fma_chain<T><<<grid, block, 0, ctx->stream>>>(d, 64, (T)0.999999, (T)1e-7);  // warm-up
  SD_LAUNCHED(ctx);
  SD_CUDA(ctx, cudaEventRecord(ctx->ev0, ctx->stream));
  SD_TIMED_BEGIN(ctx, "k_fma_chain<T>");
  k_fma_chain<T><<<grid, block, 0, ctx->stream>>>(d, iters, (T)0.999999, (T)1e-7);
  SD_LAUNCHED(ctx);
  SD_CUDA(ctx, cudaEventRecord(ctx->ev1, ctx->stream));
  SD_CUDA(ctx, cudaEventSynchronize(ctx->ev1));
  float ms = 0;
  SD_CUDA(ctx, cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1));
  double flops = 2.0 * 8.0 * (double)iters * (double)grid * (double)block;
  *tflops = flops / (ms * 1e-3) / 1e12;
  return SD_OK;
}

__global__ void k_cr_sincos(const double *x, uint64_t n, double *s, double *c) {
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) crm::sincos(x[i], s + i, c + i);
}

}  // namespace
}  // namespace sd

extern "C" int sd_cr_sincos(sd_ctx *ctx, const double *x, uint64_t n, double *s, double *c) {
  if (!ctx || (n && (!x || !s || !c))) return SD_ERR_INVALID_ARGUMENT;
  if (n == 0) return SD_OK;
  if (!sd::is_device_ptr(x) || !sd::is_device_ptr(s) || !sd::is_device_ptr(c))
    return sd::set_error(ctx, SD_ERR_INVALID_ARGUMENT, "sd_cr_sincos needs device buffers");
  SD_CUDA(ctx, cudaSetDevice(ctx->device));
  SD_TIMED_BEGIN(ctx, "k_cr_sincos");
  sd::k_cr_sincos<<<sd::grid_for(n, 256), 256, 0, ctx->stream>>>(x, n, s, c);
  SD_LAUNCHED(ctx);
  return SD_OK;
}

extern "C" int sd_measure_fp64_peak(sd_ctx *ctx, int32_t iters, double *tflops) {
  if (!ctx || !tflops || iters <= 0) return SD_ERR_INVALID_ARGUMENT;
  return sd::measure<double>(ctx, iters, tflops);
}

extern "C" int sd_measure_fp32_peak(sd_ctx *ctx, int32_t iters, double *tflops) {
  if (!ctx || !tflops || iters <= 0) return SD_ERR_INVALID_ARGUMENT;
  return sd::measure<float>(ctx, iters, tflops);
}
