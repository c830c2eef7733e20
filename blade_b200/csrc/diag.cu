// FP32 issue-rate microbenchmark: the roofline denominator of the pair kernel.
//
// The direct-space pair kernel runs on the FP32/MUFU pipes, not on tensor
// cores or HBM, so neither a copy bandwidth nor a BF16 GEMM rate bounds it.
// This kernel measures the FP32 FMA throughput of the
// device with 8 independent dependency chains per thread and a grid of
// 8 CTAs x 256 threads per SM, timed with CUDA events.
#include <cuda_runtime.h>

#include "bnb.h"

namespace {

__global__ void k_fma_chains(float *out, int iters, float a, float b) {
  float x0 = threadIdx.x * 1e-3f, x1 = x0 + 1.f, x2 = x0 + 2.f, x3 = x0 + 3.f;
  float x4 = x0 + 4.f, x5 = x0 + 5.f, x6 = x0 + 6.f, x7 = x0 + 7.f;
  for (int i = 0; i < iters; i++) {
#pragma unroll
    for (int k = 0; k < 8; k++) {
      x0 = fmaf(x0, a, b); x1 = fmaf(x1, a, b); x2 = fmaf(x2, a, b); x3 = fmaf(x3, a, b);
      x4 = fmaf(x4, a, b); x5 = fmaf(x5, a, b); x6 = fmaf(x6, a, b); x7 = fmaf(x7, a, b);
    }
  }
  float s = x0 + x1 + x2 + x3 + x4 + x5 + x6 + x7;
  if (s == 1234.5f) out[blockIdx.x] = s;  // never true in practice; keeps the chains live
}

}  // namespace

extern "C" int bnb_fp32_peak(void *stream, double *flopsPerSecond) {
  if (!flopsPerSecond) return BNB_ERR_ARG;
  cudaStream_t s = (cudaStream_t)stream;
  int dev = 0, sms = 0;
  if (cudaGetDevice(&dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
    return BNB_ERR_CUDA;
  const int grid = sms * 8, threads = 256, iters = 4096;
  float *out = nullptr;
  if (cudaMallocAsync(&out, sizeof(float) * grid, s) != cudaSuccess) return BNB_ERR_CUDA;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  k_fma_chains<<<grid, threads, 0, s>>>(out, iters, 0.9999999f, 1e-7f);  // warm-up
  float best = 1e30f;
  for (int rep = 0; rep < 5; rep++) {
    cudaEventRecord(e0, s);
    k_fma_chains<<<grid, threads, 0, s>>>(out, iters, 0.9999999f, 1e-7f);
    cudaEventRecord(e1, s);
    cudaEventSynchronize(e1);
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    if (ms < best) best = ms;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFreeAsync(out, s);
  if (cudaStreamSynchronize(s) != cudaSuccess) return BNB_ERR_CUDA;
  double flops = 2.0 * 64.0 * iters * (double)grid * threads;
  *flopsPerSecond = flops / (best * 1e-3);
  return BNB_OK;
}
