// Roofline denominator: FP64 tensor-core (DMMA) throughput of this GPU,
// measured with an in-register mma.sync m16n8k8 loop (no memory traffic).
#include "internal.h"

namespace egpu {

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
    for (int i = 0; i < 4; ++i) dmma_16x8x8(c[i], a, b);
  }
  double r = 0.0;
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) r += c[i][j];
  sink[blockIdx.x * blockDim.x + threadIdx.x] = r;
}

}  // namespace egpu

using namespace egpu;

extern "C" int egpu_measure_fp64_peak(egpu_handle h, double* tflops) {
  if (!h || !tflops) return EGPU_ERR_ARG;
  int dev = 0, sms = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int blocks = sms * 8, threads = 256, iters = 2000;
  double* sink = nullptr;
  EGPU_CUDA_TRY(cudaMalloc(&sink, sizeof(double) * blocks * threads));
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
  cudaError_t e = cudaGetLastError();
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(sink);
  if (e != cudaSuccess) {
    set_last_error(e, "dmma_peak", __FILE__, __LINE__);
    return EGPU_ERR_CUDA;
  }
  // per warp per iteration: 4 MMAs of 16x8x8 = 4 * 2 * 1024 flops
  const double flops = 4.0 * 2.0 * 16 * 8 * 8 * (double)iters * blocks * (threads / 32);
  *tflops = flops / (best * 1e-3) / 1e12;
  return EGPU_OK;
}
