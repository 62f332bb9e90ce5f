// Benchmark-only library (libegpu_bench.so, not part of libelemgpu.so): the
// FP64 roofline denominator of this GPU.  The FP64 tensor path on sm_100a is
// warp-level DMMA (mma.sync m16n8k8 f64; tcgen05 has no f64 kind), so the
// peak is an in-register m16n8k8 loop with no memory traffic, 8 CTAs of 256
// threads per SM.  bench.py --case peaks loads this library by itself.
#include <cuda_runtime.h>

#include <algorithm>

#include "../csrc/common.cuh"

namespace {

__global__ void __launch_bounds__(256) dmma_peak_kernel(double* sink, int iters) {
  double a[4] = {threadIdx.x * 1e-3, 2e-3, 3e-3, 4e-3};
  double b[2] = {1e-3, 5e-3};
  double c[4][4];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) c[i][j] = 0.0;
  for (int it = 0; it < iters; ++it) {
#pragma unroll
    for (int i = 0; i < 4; ++i) egpu::dmma_16x8x8(c[i], a, b);
  }
  double r = 0.0;
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) r += c[i][j];
  sink[blockIdx.x * blockDim.x + threadIdx.x] = r;
}

}  // namespace

// DMMA throughput of the current device in TFLOP/s (best of two timed
// launches after one warm-up).  Returns 0, or the failing cudaError_t.
extern "C" __attribute__((visibility("default"))) int egpu_bench_fp64_peak(double* tflops) {
  if (!tflops) return (int)cudaErrorInvalidValue;
  int dev = 0, sms = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int blocks = sms * 8, threads = 256, iters = 2000;
  double* sink = nullptr;
  cudaError_t e = cudaMalloc(&sink, sizeof(double) * blocks * threads);
  if (e != cudaSuccess) return (int)e;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  float best = 1e30f;
  for (int rep = 0; rep < 3; ++rep) {
    cudaEventRecord(e0);
    dmma_peak_kernel<<<blocks, threads>>>(sink, iters);
    cudaEventRecord(e1);
    cudaEventSynchronize(e1);
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    if (rep > 0) best = std::min(best, ms);
  }
  e = cudaGetLastError();
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(sink);
  if (e != cudaSuccess) return (int)e;
  // per warp per iteration: 4 MMAs of 16 x 8 x 8 = 4 * 2 * 1024 flops
  const double flops = 4.0 * 2.0 * 16 * 8 * 8 * (double)iters * blocks * (threads / 32);
  *tflops = flops / (best * 1e-3) / 1e12;
  return 0;
}
