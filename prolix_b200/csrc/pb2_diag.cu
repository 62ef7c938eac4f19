// Diagnostics: measured FP32 FMA throughput of this GPU, the denominator of
// the pair kernels' roofline (they are bound by FP32/MUFU issue, not HBM).
#include "pb2_common.cuh"
#include "pb2_internal.h"

namespace pb2 {

// Eight independent FMA chains per thread keep the FMA pipe full; the
// result is written only when it is (never) negative so the work is kept.
__global__ void fma_peak_kernel(float *sink, int iters, float a, float b) {
  float v[8];
#pragma unroll
  for (int c = 0; c < 8; ++c) v[c] = (threadIdx.x + c) * 1e-3f;
  for (int it = 0; it < iters; ++it) {
#pragma unroll
    for (int c = 0; c < 8; ++c) v[c] = fmaf(v[c], a, b);
  }
  float s = 0.f;
#pragma unroll
  for (int c = 0; c < 8; ++c) s += v[c];
  if (s < -1e30f) sink[blockIdx.x] = s;
}

}  // namespace pb2

extern "C" int pb2_fp32_peak(pb2_ctx *ctx, double *tflops) {
  if (!ctx || !tflops) return PB2_EINVAL;
  CUDA_TRY(ctx, cudaSetDevice(ctx->device));
  float *sink = nullptr;
  CUDA_TRY(ctx, cudaMalloc(&sink, 65536 * sizeof(float)));
  const int blocks = ctx->sm_count * 8, threads = 256, iters = 1 << 14;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  double best = 0.0;
  for (int rep = 0; rep < 4; ++rep) {
    cudaEventRecord(e0);
    fma_peak_kernel<<<blocks, threads>>>(sink, iters, 0.9999f, 1e-6f);
    cudaEventRecord(e1);
    cudaEventSynchronize(e1);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    const double flops = 2.0 * 8.0 * iters * (double)blocks * threads;
    if (ms > 0) best = std::max(best, flops / (ms * 1e-3) / 1e12);
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  const cudaError_t e = cudaGetLastError();
  cudaFree(sink);
  if (e != cudaSuccess) return fail(ctx, PB2_ECUDA, cudaGetErrorString(e));
  *tflops = best;
  return PB2_OK;
}
