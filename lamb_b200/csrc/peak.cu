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

// Integer tensor pipe through mma.sync (the instruction of the int8-slice
// kernel): independent m16n8k32 s8 products, 8192 integer ops each.
__global__ void k_imma_peak(int* out, int iters) {
  const int a = 0x01010101 * (threadIdx.x & 3), b = 0x01010101;
  int c[8][4];
#pragma unroll
  for (int j = 0; j < 8; ++j)
#pragma unroll
    for (int h = 0; h < 4; ++h) c[j][h] = 0;
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int j = 0; j < 8; ++j)
      asm volatile(
          "mma.sync.aligned.m16n8k32.row.col.s32.s8.s8.s32 {%0,%1,%2,%3}, {%4,%4,%4,%4}, {%5,%5}, {%0,%1,%2,%3};"
          : "+r"(c[j][0]), "+r"(c[j][1]), "+r"(c[j][2]), "+r"(c[j][3])
          : "r"(a), "r"(b));
  }
  int s = 0;
#pragma unroll
  for (int j = 0; j < 8; ++j) s += c[j][0] + c[j][1] + c[j][2] + c[j][3];
  out[(size_t)blockIdx.x * blockDim.x + threadIdx.x] = s;
}

}  // namespace

extern "C" int32_t lamb_probe_int8_tops(int32_t device, int32_t reps, double* tops) {
  if (!tops) return lamb::make_status(LAMB_LEVEL_FAILURE, LAMB_TYPE_WRONG_ARGS);
  if (cudaSetDevice(device) != cudaSuccess) return lamb::make_status(LAMB_LEVEL_FAILURE, LAMB_TYPE_EXTERNAL_ERROR);
  int sms = 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  const int threads = 256, blocks = sms * 4, iters = 20000;
  int* out = nullptr;
  if (cudaMalloc(&out, sizeof(int) * (size_t)threads * blocks) != cudaSuccess)
    return lamb::make_status(LAMB_LEVEL_MEMORY, LAMB_TYPE_EXTERNAL_ERROR);
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  k_imma_peak<<<blocks, threads>>>(out, iters / 10);
  float best = 1e30f;
  for (int r = 0; r < (reps > 0 ? reps : 3); ++r) {
    cudaEventRecord(e0);
    k_imma_peak<<<blocks, threads>>>(out, iters);
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
  const double ops = 8192.0 * 8 * iters * ((double)blocks * threads / 32);
  *tops = ops / (best * 1e-3) / 1e12;
  return LAMB_GPU_OK;
}

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
