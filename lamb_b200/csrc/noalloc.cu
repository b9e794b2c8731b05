// Tr(X.Y) without any device allocation: lamb_gpu_trace_product_noalloc
// (declared in include/lamb_gpu.h, where its callers and limits are described).
// Working storage is the file-scope array below; host code uses its device
// address, looked up once per device.
#include <mutex>

#include "common.cuh"

namespace {

constexpr int kMaxBlocks = LAMB_GPU_NOALLOC_MAX_BLOCKS;
constexpr int kMaxDevices = 64;

// One partial sum per block of X, then the total (slot kMaxBlocks) and a
// blocking-mismatch flag (slot kSlotBad, cleared by every call).
constexpr int kSlotBad = kMaxBlocks + 1;
static __device__ __align__(256) double g_trace_scratch[kMaxBlocks + 2];

std::mutex g_mu;
double* g_scratch_ptr[kMaxDevices] = {};

// Device address of g_trace_scratch on the current device (set up once).
int32_t scratch_for_device(int dev, double** out) {
  if (dev < 0 || dev >= kMaxDevices) return lamb::make_status(LAMB_LEVEL_FAILURE, LAMB_TYPE_UNIMPLEMENTED);
  std::lock_guard<std::mutex> lock(g_mu);
  if (!g_scratch_ptr[dev]) {
    double* p = nullptr;
    if (cudaGetSymbolAddress((void**)&p, g_trace_scratch) != cudaSuccess || !p)
      return lamb::make_status(LAMB_LEVEL_FAILURE, LAMB_TYPE_EXTERNAL_ERROR);
    g_scratch_ptr[dev] = p;
  }
  *out = g_scratch_ptr[dev];
  return LAMB_GPU_OK;
}

// Partial of X block u: <X_ij, Y_ji^T>, Y_ji found by binary search.  A Y
// block whose shape is not X_ij's transpose (the two matrices' blockings
// differ) is skipped and reported through scratch[kSlotBad].
__global__ void k_noalloc_partials(lamb_gpu_dcsr x, lamb_gpu_dcsr y, double* __restrict__ scratch) {
  const int lane = threadIdx.x & 31;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t r = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; r < x.n_rows; r += nw) {
    const int bi = x.row_bs[r];
    for (int64_t u = x.row_p[r]; u < x.row_p[r + 1]; ++u) {
      const int j = x.col[u], bj = x.col_bs[j];
      int64_t yb = -1;
      if (y.nnz > 0) {
        int64_t lo = y.row_p[j], hi = y.row_p[j + 1] - 1;
        while (lo <= hi) {
          const int64_t mid = (lo + hi) >> 1;
          const int c = y.col[mid];
          if (c == r) { yb = mid; break; }
          if (c < r) lo = mid + 1; else hi = mid - 1;
        }
      }
      if (yb >= 0 && (y.row_bs[j] != bj || y.col_bs[r] != bi)) {
        if (lane == 0) scratch[kSlotBad] = 1.0;
        yb = -1;
      }
      double s = 0.0;
      if (yb >= 0) {
        const double* xp = x.data + x.off[u];
        const double* yp = y.data + y.off[yb];
        for (int e = lane; e < bi * bj; e += 32) {
          const int p = e % bi, q = e / bi;
          s = __fma_rn(xp[e], yp[q + (int64_t)p * bj], s);
        }
      }
      s = lamb::warp_sum(s);
      if (lane == 0) scratch[u] = s;
    }
  }
}

// Fixed-order sum of scratch[0..n) into scratch[kMaxBlocks] (one CTA).
__global__ void k_noalloc_total(int64_t n, double* __restrict__ scratch) {
  __shared__ double part[256];
  double s = 0.0;
  for (int64_t i = threadIdx.x; i < n; i += blockDim.x) s += scratch[i];
  part[threadIdx.x] = s;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w) part[threadIdx.x] += part[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) scratch[kMaxBlocks] = part[0];
}

}  // namespace

extern "C" int32_t lamb_gpu_trace_product_noalloc(const lamb_gpu_dcsr* x, const lamb_gpu_dcsr* y, void* stream,
                                                  double* result) {
  using lamb::make_status;
  if (!x || !y || !result) return make_status(LAMB_LEVEL_FAILURE, LAMB_TYPE_WRONG_ARGS);
  if (x->nnz < 0 || x->nnz > kMaxBlocks || x->n_rows < 0) return make_status(LAMB_LEVEL_FAILURE, LAMB_TYPE_WRONG_ARGS);
  if (x->n_rows != y->n_cols || x->n_cols != y->n_rows || y->nnz < 0)
    return make_status(LAMB_LEVEL_FAILURE, LAMB_TYPE_WRONG_ARGS);
  if (x->nnz > 0 && (!x->row_bs || !x->col_bs || !x->row_p || !x->col || !x->off || !x->data))
    return make_status(LAMB_LEVEL_FAILURE, LAMB_TYPE_WRONG_ARGS);
  // An empty Y (no blocks) may come with null arrays: the trace is then 0.
  if (x->nnz > 0 && y->nnz > 0 && (!y->row_bs || !y->col_bs || !y->row_p || !y->col || !y->off || !y->data))
    return make_status(LAMB_LEVEL_FAILURE, LAMB_TYPE_WRONG_ARGS);
  // A CUDA error left pending by earlier, unrelated work is not this call's:
  // report it without launching (and without clearing it).
  if (cudaPeekAtLastError() != cudaSuccess) return make_status(LAMB_LEVEL_FAILURE, LAMB_TYPE_EXTERNAL_ERROR);
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return make_status(LAMB_LEVEL_FAILURE, LAMB_TYPE_EXTERNAL_ERROR);
  double* scratch = nullptr;
  int32_t st = scratch_for_device(dev, &scratch);
  if (st != LAMB_GPU_OK) return st;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  if (cudaMemsetAsync(scratch + kSlotBad, 0, sizeof(double), s) != cudaSuccess)
    return make_status(LAMB_LEVEL_FAILURE, LAMB_TYPE_EXTERNAL_ERROR);
  if (x->nnz > 0 && x->n_rows > 0) {
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int64_t warps = x->n_rows;
    const int grid = (int)std::min<int64_t>((warps + 7) / 8, (int64_t)sms * 16);
    k_noalloc_partials<<<grid, 256, 0, s>>>(*x, *y, scratch);
  }
  k_noalloc_total<<<1, 256, 0, s>>>(x->nnz, scratch);
  // Nothing was pending before the launches, so an error now is theirs.
  if (cudaGetLastError() != cudaSuccess) return make_status(LAMB_LEVEL_FAILURE, LAMB_TYPE_EXTERNAL_ERROR);
  double back[2] = {0.0, 0.0};  // total, mismatch flag (adjacent slots)
  if (cudaMemcpyAsync(back, scratch + kMaxBlocks, sizeof(back), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
      cudaStreamSynchronize(s) != cudaSuccess)
    return make_status(LAMB_LEVEL_FAILURE, LAMB_TYPE_EXTERNAL_ERROR);
  if (back[1] != 0.0) return make_status(LAMB_LEVEL_FAILURE, LAMB_TYPE_WRONG_ARGS);
  *result = back[0];
  return LAMB_GPU_OK;
}
