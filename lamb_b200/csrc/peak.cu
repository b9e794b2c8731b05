// Tensor-pipe throughput probes: FP64, int8 and bf16 through mma.sync
// (declared in include/lamb_probe.h).
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

// bf16 tensor pipe through mma.sync with FP32 accumulation (the instruction a
// bf16-slice kernel would use): independent m16n8k16 products, 4096 flops each.
__global__ void k_hmma_peak(float* out, int iters) {
  const unsigned a = 0x3f803f80u * (threadIdx.x & 1), b = 0x3f803f80u;  // bf16 pairs (1, 1)
  float c[8][4];
#pragma unroll
  for (int j = 0; j < 8; ++j)
#pragma unroll
    for (int h = 0; h < 4; ++h) c[j][h] = 0.f;
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int j = 0; j < 8; ++j)
      asm volatile(
          "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%4,%4,%4}, {%5,%5}, "
          "{%0,%1,%2,%3};"
          : "+f"(c[j][0]), "+f"(c[j][1]), "+f"(c[j][2]), "+f"(c[j][3])
          : "r"(a), "r"(b));
  }
  float s = 0.f;
#pragma unroll
  for (int j = 0; j < 8; ++j) s += c[j][0] + c[j][1] + c[j][2] + c[j][3];
  out[(size_t)blockIdx.x * blockDim.x + threadIdx.x] = s;
}

}  // namespace

// Best of `reps` timed launches of kern (per_sm CTAs of 256 threads on every
// SM, `iters` loop iterations) after one short warm-up launch; writes
// ops_per_warp_iter x iterations x warps / time in units of 1e12 per second.
template <typename T>
static int32_t time_probe(int32_t device, int32_t reps, int per_sm, void (*kern)(T*, int), double ops_per_warp_iter,
                          double* rate) {
  if (!rate) return lamb::make_status(LAMB_LEVEL_FAILURE, LAMB_TYPE_WRONG_ARGS);
  if (cudaSetDevice(device) != cudaSuccess) return lamb::make_status(LAMB_LEVEL_FAILURE, LAMB_TYPE_EXTERNAL_ERROR);
  int sms = 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  const int threads = 256, blocks = sms * per_sm, iters = 20000;
  T* out = nullptr;
  if (cudaMalloc(&out, sizeof(T) * (size_t)threads * blocks) != cudaSuccess)
    return lamb::make_status(LAMB_LEVEL_MEMORY, LAMB_TYPE_EXTERNAL_ERROR);
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  kern<<<blocks, threads>>>(out, iters / 10);
  float best = 1e30f;
  for (int r = 0; r < (reps > 0 ? reps : 3); ++r) {
    cudaEventRecord(e0);
    kern<<<blocks, threads>>>(out, iters);
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
  *rate = ops_per_warp_iter * iters * ((double)blocks * threads / 32) / (best * 1e-3) / 1e12;
  return LAMB_GPU_OK;
}

extern "C" int32_t lamb_probe_fp64_tflops(int32_t device, int32_t reps, double* tflops) {
  return time_probe<double>(device, reps, 8, k_dmma_peak, 512.0 * 4, tflops);
}

extern "C" int32_t lamb_probe_int8_tops(int32_t device, int32_t reps, double* tops) {
  return time_probe<int>(device, reps, 4, k_imma_peak, 8192.0 * 8, tops);
}

extern "C" int32_t lamb_probe_bf16_tflops(int32_t device, int32_t reps, double* tflops) {
  return time_probe<float>(device, reps, 4, k_hmma_peak, 4096.0 * 8, tflops);
}
