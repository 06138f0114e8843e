// Arithmetic-throughput probes for the compute side of the rooflines the
// benchmark reports: FP64 FMA (the FP64 stencils) and packed FP32 FMA (the
// FP32 Chebyshev stencil).  Every thread runs 8 independent FMA chains so
// that issue, not latency, bounds the rate; the results are written out so
// the chains are not eliminated.
#include <cuda_runtime.h>

#include "../../include/nrqcd_b200.h"
#include "nrq_internal.h"

namespace {
constexpr int kChains = 8;

__global__ void __launch_bounds__(256) k_probe_dfma(int iters, double seed, double *out) {
  double a[kChains];
#pragma unroll
  for (int k = 0; k < kChains; ++k) a[k] = seed + 1e-3 * (threadIdx.x + k);
  const double m = 0.999999, c = 1e-9;
  for (int i = 0; i < iters; ++i)
#pragma unroll
    for (int k = 0; k < kChains; ++k) a[k] = fma(a[k], m, c);
  double s = 0.0;
#pragma unroll
  for (int k = 0; k < kChains; ++k) s += a[k];
  out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

__global__ void __launch_bounds__(256) k_probe_ffma2(int iters, float seed, float *out) {
  float2 a[kChains];
#pragma unroll
  for (int k = 0; k < kChains; ++k) a[k] = make_float2(seed + 1e-3f * (threadIdx.x + k), seed - 1e-3f * k);
  const float2 m = make_float2(0.999999f, 0.999998f), c = make_float2(1e-9f, 2e-9f);
  for (int i = 0; i < iters; ++i)
#pragma unroll
    for (int k = 0; k < kChains; ++k) a[k] = __ffma2_rn(a[k], m, c);
  float s = 0.f;
#pragma unroll
  for (int k = 0; k < kChains; ++k) s += a[k].x + a[k].y;
  out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}
}  // namespace

extern "C" int nrq_measure_peaks(nrq_ctx *ctx, double *fp64_tflops, double *fp32_tflops) {
  if (!ctx) return NRQ_ERR_BAD_ARG;
  int rc = nrqh::set_device(ctx);
  if (rc) return rc;
  const int blocks = ctx->sm_count * 8, threads = 256, iters = 4096;
  void *out = nullptr;
  NRQ_CUDA_TRY(ctx, cudaMalloc(&out, sizeof(double) * blocks * threads));
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  auto timed = [&](bool fp64) {
    float best = 1e30f;
    for (int r = 0; r < 4; ++r) {  // first repetition warms up
      cudaEventRecord(e0, ctx->stream);
      if (fp64)
        k_probe_dfma<<<blocks, threads, 0, ctx->stream>>>(iters, 1.0, (double *)out);
      else
        k_probe_ffma2<<<blocks, threads, 0, ctx->stream>>>(iters, 1.0f, (float *)out);
      cudaEventRecord(e1, ctx->stream);
      cudaEventSynchronize(e1);
      float ms = 0.f;
      cudaEventElapsedTime(&ms, e0, e1);
      if (r > 0 && ms < best) best = ms;
    }
    return best;
  };
  const double fmas = (double)blocks * threads * iters * kChains;
  const float ms64 = timed(true), ms32 = timed(false);
  rc = nrqh::check_launch(ctx, "peak probes");
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(out);
  if (rc) return rc;
  if (fp64_tflops) *fp64_tflops = 2.0 * fmas / (ms64 * 1e-3) / 1e12;
  if (fp32_tflops) *fp32_tflops = 2.0 * 2.0 * fmas / (ms32 * 1e-3) / 1e12;  // two lanes per packed FMA
  return NRQ_OK;
}
