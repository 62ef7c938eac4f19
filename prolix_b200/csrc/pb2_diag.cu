// Diagnostics: measured FP32 FMA throughput of this GPU, the denominator of
// the pair kernels' roofline (they are bound by FP32/MUFU issue, not HBM).
#include "pb2_common.cuh"
#include "pb2_divide.cuh"
#include "pb2_internal.h"

namespace pb2 {

__device__ __forceinline__ unsigned long long splitmix64(unsigned long long z) {
  z += 0x9e3779b97f4a7c15ull;
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
  return z ^ (z >> 31);
}

// div_by against the correctly rounded division on n seeded (p, m) pairs:
// p of any sign with exponents -40..40, m with exponents -1..8 (masses
// 0.5-512 amu), and every 16 samples a mass with an all-ones and one with
// an all-zeros significand, an exact multiple, a zero and a subnormal-range
// quotient.  Counts the pairs whose bits differ; the first one found is
// recorded.
__global__ void div_check_kernel(unsigned long long seed, long long n, unsigned long long *bad, double *example) {
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += stride) {
    const unsigned long long h1 = splitmix64(seed ^ (2ull * (unsigned long long)i));
    const unsigned long long h2 = splitmix64(seed ^ (2ull * (unsigned long long)i + 1ull));
    const int ep = (int)((h1 >> 52) % 81ull) - 40;
    const unsigned long long frac = 0x000fffffffffffffull;
    double p = __longlong_as_double((long long)((h1 & frac) | ((unsigned long long)(1023 + ep) << 52) |
                                                (h2 & 0x8000000000000000ull)));
    const int em = (int)((h2 >> 52) % 10ull) - 1;
    unsigned long long mm = h2 & frac;
    const int kind = (int)(i & 15);
    if (kind == 1) mm = frac;
    if (kind == 2) mm = 0;
    const double m = __longlong_as_double((long long)(mm | ((unsigned long long)(1023 + em) << 52)));
    if (kind == 3) p = m * (double)(h1 & 0xffff);
    if (kind == 4) p = (h1 & 1) ? -0.0 : 0.0;
    if (kind == 5) p = __longlong_as_double((long long)((h1 & frac) | (20ull << 52)));
    const double q = div_by(p, m, __drcp_rn(m));
    const double r = __ddiv_rn(p, m);
    if (__double_as_longlong(q) != __double_as_longlong(r)) {
      if (atomicAdd(bad, 1ull) == 0ull) {
        example[0] = p;
        example[1] = m;
      }
    }
  }
}

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

extern "C" int pb2_diag_div_check(pb2_ctx *ctx, long long n, unsigned long long seed, long long *mismatches,
                                  double *example) {
  if (!ctx || !mismatches || n < 0) return PB2_EINVAL;
  CUDA_TRY(ctx, cudaSetDevice(ctx->device));
  unsigned long long *bad = nullptr;
  double *ex = nullptr;
  CUDA_TRY(ctx, cudaMalloc(&bad, sizeof(unsigned long long)));
  CUDA_TRY(ctx, cudaMalloc(&ex, 2 * sizeof(double)));
  cudaMemset(bad, 0, sizeof(unsigned long long));
  cudaMemset(ex, 0, 2 * sizeof(double));
  pb2::div_check_kernel<<<ctx->sm_count * 8, 256>>>(seed, n, bad, ex);
  unsigned long long h = 0;
  double hx[2] = {0.0, 0.0};
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaMemcpy(&h, bad, sizeof h, cudaMemcpyDeviceToHost);
  if (e == cudaSuccess) e = cudaMemcpy(hx, ex, sizeof hx, cudaMemcpyDeviceToHost);
  cudaFree(bad);
  cudaFree(ex);
  if (e != cudaSuccess) return fail(ctx, PB2_ECUDA, cudaGetErrorString(e));
  *mismatches = (long long)h;
  if (example) {
    example[0] = hx[0];
    example[1] = hx[1];
  }
  return PB2_OK;
}
