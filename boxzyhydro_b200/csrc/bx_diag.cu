// bx_diag.cu -- FP64 FMA throughput probe (include/boxzy_diag.h).
#include <cuda_runtime.h>

#include "../../include/boxzy_diag.h"

namespace {
constexpr int kChains = 8;
constexpr int kIters = 2048;

__global__ void __launch_bounds__(256) k_dfma(double* out, double seed) {
  double a[kChains];
  const double b = 1.0 + 1e-9 * threadIdx.x, c = 1e-12 * blockIdx.x;
#pragma unroll
  for (int k = 0; k < kChains; ++k) a[k] = seed + k;
  for (int it = 0; it < kIters; ++it) {
#pragma unroll
    for (int k = 0; k < kChains; ++k) a[k] = fma(a[k], b, c);
  }
  double s = 0.0;
#pragma unroll
  for (int k = 0; k < kChains; ++k) s += a[k];
  if (s == 1234.5678) out[0] = s;  // keeps the chains live
}
}  // namespace

extern "C" int bx_fp64_peak(double* tflops, double* ms_out) {
  int dev = 0, sms = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return 2;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  double* out = nullptr;
  if (cudaMalloc(&out, sizeof(double)) != cudaSuccess) return 5;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  const int blocks = sms * 8, threads = 256;
  for (int w = 0; w < 3; ++w) k_dfma<<<blocks, threads>>>(out, 1.0);
  float best = 1e30f;
  for (int r = 0; r < 5; ++r) {
    cudaEventRecord(e0);
    k_dfma<<<blocks, threads>>>(out, 1.0);
    cudaEventRecord(e1);
    cudaEventSynchronize(e1);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    if (ms < best) best = ms;
  }
  const double flops = 2.0 * kChains * (double)kIters * blocks * threads;
  if (tflops) *tflops = flops / (best * 1e-3) / 1e12;
  if (ms_out) *ms_out = best;
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(out);
  return cudaGetLastError() == cudaSuccess ? 0 : 2;
}
