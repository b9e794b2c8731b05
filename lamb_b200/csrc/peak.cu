// FP64 tensor-pipe throughput probe (declared in include/lamb_probe.h).
#include "common.cuh"
#include "lamb_probe.h"

namespace {

__global__ void k_dmma_peak(double* out, int iters) {
  const double a = 1e-3 * (threadIdx.x & 7), b = 1e-3;
  double c[8];
#pragma unroll
  for (int j = 0; j < 8; ++j) c[j] = 0.0;
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int j = 0; j < 4; ++j)
      asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
                   : "+d"(c[2 * j]), "+d"(c[2 * j + 1])
                   : "d"(a), "d"(b));
  }
  double s = 0.0;
#pragma unroll
  for (int j = 0; j < 8; ++j) s += c[j];
  out[(size_t)blockIdx.x * blockDim.x + threadIdx.x] = s;
}

}  // namespace

extern "C" int32_t lamb_probe_fp64_tflops(int32_t device, int32_t reps, double* tflops) {
  if (!tflops) return lamb::make_status(LAMB_LEVEL_FAILURE, LAMB_TYPE_WRONG_ARGS);
  if (cudaSetDevice(device) != cudaSuccess) return lamb::make_status(LAMB_LEVEL_FAILURE, LAMB_TYPE_EXTERNAL_ERROR);
  int sms = 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  const int threads = 256, blocks = sms * 8, iters = 20000;
  double* out = nullptr;
  if (cudaMalloc(&out, sizeof(double) * (size_t)threads * blocks) != cudaSuccess)
    return lamb::make_status(LAMB_LEVEL_MEMORY, LAMB_TYPE_EXTERNAL_ERROR);
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  k_dmma_peak<<<blocks, threads>>>(out, iters / 10);
  float best = 1e30f;
  for (int r = 0; r < (reps > 0 ? reps : 3); ++r) {
    cudaEventRecord(e0);
    k_dmma_peak<<<blocks, threads>>>(out, iters);
    cudaEventRecord(e1);
    cudaEventSynchronize(e1);
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    best = ms < best ? ms : best;
  }
  cudaError_t e = cudaGetLastError();
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(out);
  if (e != cudaSuccess) return lamb::make_status(LAMB_LEVEL_FAILURE, LAMB_TYPE_EXTERNAL_ERROR);
  const double flops = 512.0 * 4 * iters * ((double)blocks * threads / 32);
  *tflops = flops / (best * 1e-3) / 1e12;
  return LAMB_GPU_OK;
}
