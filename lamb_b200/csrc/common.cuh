// Shared definitions of the B200 sector-multiply library (liblamb_b200.so).
#pragma once

#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <string>
#include <vector>

#include "lamb_gpu.h"

namespace lamb {

// ---- status codes (level/type pairs of src/lamb_error.F90:120-159) -------
inline int32_t make_status(int level, int type) { return level * 100000 + (type + 50000); }

// ---- device matrix ------------------------------------------------------------
// Every device matrix is one block-CSR over "sector order": the atoms of
// subset 1 first (in local order), then subset 2, ... along rows and columns.
// A global row is a local row of one row subset; its blocks are sorted by
// global column, so the blocks of sector (m,n) are a contiguous run of the row.
// Block data live in one buffer, sector-major: all blocks of sector (m,n)
// inside [sec_base[s], sec_base[s] + sec_dlen[s]), s = (m-1)*n_csub + (n-1).
// Inside a sector the caller's layout (uploads) or CSR order (results) is kept.
struct DevMatrix {
  int32_t n_rsub = 0, n_csub = 0;
  std::vector<int32_t> rsub_cnt, csub_cnt;    // atoms per subset
  std::vector<int32_t> rsub_base, csub_base;  // first sector-order index of each subset (+ total)
  std::vector<int8_t> h_row_bs, h_col_bs;     // block sizes (host copies)
  int32_t n_rows = 0, n_cols = 0;
  int64_t nnz = 0, data_len = 0;
  std::vector<int64_t> sec_base, sec_dlen, sec_nblk;  // per sector (m,n)
  int8_t* row_bs = nullptr;    // [n_rows]
  int8_t* col_bs = nullptr;    // [n_cols]
  int64_t* row_p = nullptr;    // [n_rows+1]
  int32_t* col = nullptr;      // [nnz]
  int64_t* off = nullptr;      // [nnz], 0-based data offset of each block
  double* data = nullptr;      // [data_len]
  int64_t data_cap = 0;        // elements of data a later multiply into this matrix may reuse (0: none)
  double* norms = nullptr;     // [nnz] Frobenius norms, valid when norms_valid
  bool norms_valid = false;
  // Locality: optional row-atom coordinates (sector order) and the processing
  // order of rows derived from them (Morton) or from the pattern (Cuthill-McKee).
  std::vector<float> h_pos;    // 3*n_rows, empty when not given
  float box[3] = {0, 0, 0};
  std::vector<int32_t> h_order;  // row processing order, empty until computed
  int32_t* order = nullptr;      // device copy of h_order
  // Result of a multiply computed in row chunks: the data of chunk p in
  // sector s is [chunk_rng[2*(p*S_all+s)], chunk_rng[2*(p*S_all+s)+1]) relative
  // to the sector's base; chunk p is complete when the context's chunk_ev[p]
  // fires (valid while the context's chunk_m points here).
  int n_chunks = 0;
  std::vector<int64_t> chunk_rng;
  const double* chunk_data = nullptr;  // data buffer the ranges refer to
  // Layout generation: a process-wide unique value renewed (touch()) whenever
  // the device buffers or the block layout are replaced, so that holders of
  // raw device pointers (batches) can detect a stale view.
  uint64_t gen = 0;
};

// Gives m a new layout generation.
void touch(DevMatrix* m);

// Row chunks of a multiply's numeric phase: at most kMaxChunks, at least
// kMinChunks when C has enough blocks (downloads overlap the later chunks).
constexpr int kMaxChunks = 64;
constexpr int kMinChunks = 8;

// Roles of the context's grow-only scratch buffers (multiply temporaries).
enum ScratchSlot : int { kScrEnt = 0, kScrWork, kScrWorkC, kScrPlaneA, kScrPlaneB, kScrSlots };

struct Ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  std::string last_error;
  std::map<int64_t, std::unique_ptr<DevMatrix>> mats;
  int64_t next_handle = 1;
  lamb_gpu_mult_stats last_stats{};
  int64_t launches = 0;  // kernels of this library launched on the context
  cudaEvent_t ev[8] = {};
  bool trace = false;     // LAMB_GPU_TRACE=1 at creation: phase timings on stderr
  bool trace_host = false; // LAMB_GPU_TRACE=2: host time between marks, no synchronisation
  double trace_t = 0.0;   // host time of the previous trace mark (ms)
  // Multiply temporaries of several GB (stacks, work items, digit planes) are
  // kept between calls: releasing and re-reserving them fragments the
  // stream-ordered pool, which then maps fresh memory at up to a second a call.
  void* scr[kScrSlots] = {};
  size_t scr_bytes[kScrSlots] = {};
  // Result filter whose host metadata is still on its way (LAMB_GPU_ASYNC):
  // per-sector kept block counts land in pend_h (pinned) when pend_ev fires.
  DevMatrix* pend_m = nullptr;
  int64_t* pend_h = nullptr;
  size_t pend_cap = 0;
  cudaEvent_t pend_ev = nullptr;
  // Chunked numeric phase of the last multiply (downloads overlap it).
  DevMatrix* chunk_m = nullptr;
  cudaEvent_t chunk_ev[kMaxChunks] = {};
  // timing events around each row chunk's product-kernel launch (FP64 path)
  cudaEvent_t kern_ev[2][kMaxChunks] = {};
  int kern_chunks = 0;
  cudaStream_t copy_stream = nullptr;
};

// Completes a pending result filter (waits for its counts and updates the
// matrix's host metadata).  Every entry point reaches it through get_matrix.
int32_t settle(Ctx* ctx);

// With tracing on, waits for the stream (not with LAMB_GPU_TRACE=2) and
// prints the host time since the previous mark; otherwise does nothing.
void trace_mark(Ctx* ctx, const char* what);

// Error helpers: set the message, return the encoded status.
int32_t fail(Ctx* ctx, int level, int type, const std::string& msg);
#define LAMB_CUDA(ctx, call)                                                                             \
  do {                                                                                                   \
    cudaError_t e_ = (call);                                                                             \
    if (e_ != cudaSuccess)                                                                               \
      return ::lamb::fail((ctx), LAMB_LEVEL_FAILURE, LAMB_TYPE_EXTERNAL_ERROR,                           \
                          std::string(#call) + ": " + cudaGetErrorString(e_) + " (" + __FILE__ + ":" +   \
                              std::to_string(__LINE__) + ")");                                           \
  } while (0)
#define LAMB_TRY(x)                   \
  do {                                \
    int32_t st_ = (x);                \
    if (st_ != LAMB_GPU_OK) return st_; \
  } while (0)

// Stream-ordered allocation on the context's stream.  When the pool cannot
// satisfy a request, unused pool memory is returned to the device once and the
// allocation retried.
int32_t dalloc_bytes(Ctx* ctx, void** p, size_t bytes);
template <typename T>
int32_t dalloc(Ctx* ctx, T** p, int64_t n) {
  *p = nullptr;
  if (n <= 0) return LAMB_GPU_OK;
  return dalloc_bytes(ctx, reinterpret_cast<void**>(p), sizeof(T) * (size_t)n);
}

// Grow-only scratch buffer of the context for one role; the contents do not
// survive the next call that uses the same role.
int32_t scratch_bytes(Ctx* ctx, int slot, size_t bytes, void** p);
template <typename T>
int32_t scratch(Ctx* ctx, int slot, int64_t n, T** p) {
  return scratch_bytes(ctx, slot, sizeof(T) * (size_t)std::max<int64_t>(n, 1), reinterpret_cast<void**>(p));
}
void release_scratch(Ctx* ctx);

template <typename T>
void dfree(Ctx* ctx, T*& p) {
  if (p) cudaFreeAsync((void*)p, ctx->stream);
  p = nullptr;
}

DevMatrix* get_matrix(Ctx* ctx, lamb_gpu_matrix h);  // settles a pending result filter first
DevMatrix* find_matrix(Ctx* ctx, lamb_gpu_matrix h); // no settle
void free_matrix_buffers(Ctx* ctx, DevMatrix* m);
int32_t register_matrix(Ctx* ctx, std::unique_ptr<DevMatrix> m, lamb_gpu_matrix* h);
int32_t ensure_norms(Ctx* ctx, DevMatrix* m);
// Row processing order of m (computed once, cached): Morton order of the row
// coordinates when given, else Cuthill-McKee order of m's block pattern.
int32_t ensure_row_order(Ctx* ctx, DevMatrix* m);
// Copies the row locality data (coordinates and order) of src to dst.
int32_t inherit_row_locality(Ctx* ctx, DevMatrix* dst, const DevMatrix* src);
// Copies the subset structure (not the blocks) of rows of `r` and columns of `c`.
void copy_structure(DevMatrix* dst, const DevMatrix* r_src, bool rows_from_rows, const DevMatrix* c_src,
                    bool cols_from_cols);
int32_t upload_block_sizes(Ctx* ctx, DevMatrix* m);
// Sector-major layout for a pattern already in m (row_p/col set): fills off,
// sec_base/sec_dlen/sec_nblk, data_len.  row_of (optional, [nnz]) gets each block's row.
// by_order: inside a sector, rows' blocks follow m's processing order (h_order)
// instead of the local row order; h_base (optional) gets the data offset of
// every (row subset, column subset, local rank) run, indexed
// rsub_base[a]*S + n*rsub_cnt[a] + rank.
int32_t layout_sector_major(Ctx* ctx, DevMatrix* m, int32_t* row_of, bool by_order = false,
                            std::vector<int64_t>* h_base = nullptr);
// Per-sector download index of m on the device: for sector s (query order)
// its blocks occupy [first_s, first_s + sec_nblk[s]) of col16 (1-based int16
// columns) and ext (1-based inclusive extents into the sector's data); h_bcnt
// (filled once the stream reaches it) holds the run length of every
// (row subset a, column subset n, local row l) at rsub_base[a]*S + n*rsub_cnt[a] + l.
struct SectorIndex {
  int16_t* col16 = nullptr;
  int64_t* ext = nullptr;
  std::vector<int64_t> h_bcnt;
};
int32_t build_sector_index(Ctx* ctx, const DevMatrix* m, SectorIndex* si);
void free_sector_index(Ctx* ctx, SectorIndex* si);
// Exclusive scan of int64 (in place allowed), via CUB with stream-ordered scratch.
int32_t exclusive_scan_i64(Ctx* ctx, const int64_t* in, int64_t* out, int64_t n);
int32_t inclusive_scan_i64(Ctx* ctx, const int64_t* in, int64_t* out, int64_t n);
int32_t sum_i64(Ctx* ctx, const int64_t* in, int64_t n, int64_t* host_out);
// Largest of n int64 (waits for the stream); 0 when n == 0.
int32_t max_i64(Ctx* ctx, const int64_t* in, int64_t n, int64_t* host_out);
// Smallest of n doubles (waits for the stream); 0 when n == 0.
int32_t min_f64(Ctx* ctx, const double* in, int64_t n, double* host_out);

// ---- device helpers -------------------------------------------------------------
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ int warp_incl_scan(int v, int lane) {
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    int t = __shfl_up_sync(0xffffffffu, v, o);
    if (lane >= o) v += t;
  }
  return v;
}
__device__ __forceinline__ long long warp_incl_scan_ll(long long v, int lane) {
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    long long t = __shfl_up_sync(0xffffffffu, v, o);
    if (lane >= o) v += t;
  }
  return v;
}
__device__ __forceinline__ long long warp_sum_ll(long long v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
// First position in [lo, hi) whose column is >= c (columns ascending within a row).
__device__ __forceinline__ int64_t lower_col(const int32_t* __restrict__ col, int64_t lo, int64_t hi, int32_t c) {
  while (lo < hi) {
    const int64_t mid = (lo + hi) >> 1;
    if (col[mid] < c) lo = mid + 1; else hi = mid;
  }
  return lo;
}
// Row subset of row r (n_rsub is small: a linear scan).
__device__ __forceinline__ int row_subset(const int32_t* __restrict__ rsub_base, int32_t n_rsub, int64_t r) {
  int m = 0;
  while (m + 1 < n_rsub && rsub_base[m + 1] <= r) ++m;
  return m;
}
// Warp-per-row loops: global warp index and warp count of the grid.
// Step of an element walk: e -> e + 32 moves (minor, major) of a block whose
// minor extent is d by (32 % d, 32 / d) with a carry; the start (lane % d,
// lane / d) and the steps come from one float quotient, exact for the
// block sizes 1 <= d <= 127 because (lane + 0.5) / d lies at least 0.5 / d
// from an integer.
struct Walk {
  int minor, major, step_minor, step_major, d;
  __device__ __forceinline__ Walk(int d_, int lane) : d(d_) {
    const float rcp = __frcp_rn((float)d_);
    major = (int)(((float)lane + 0.5f) * rcp);
    minor = lane - major * d_;
    step_major = (int)(32.5f * rcp);
    step_minor = 32 - step_major * d_;
  }
  __device__ __forceinline__ void next() {
    minor += step_minor;
    major += step_major;
    if (minor >= d) {
      minor -= d;
      ++major;
    }
  }
};

__device__ __forceinline__ int64_t global_warp() { return ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; }
__device__ __forceinline__ int64_t grid_warps() { return ((int64_t)gridDim.x * blockDim.x) >> 5; }

// Fixed-order block norm: sequential fma over the block in storage order.
// The CPU oracle uses the same expression, so the filter decisions agree bit for bit.
__device__ __forceinline__ double block_norm_seq(const double* __restrict__ x, int64_t n) {
  double s = 0.0;
  for (int64_t e = 0; e < n; ++e) s = __fma_rn(x[e], x[e], s);
  return __dsqrt_rn(s);
}

constexpr int kThreads = 256;
// Counts a launch of one of this library's kernels and checks it.
#define LAMB_LAUNCHED(ctx) do { ++(ctx)->launches; LAMB_CUDA((ctx), cudaGetLastError()); } while (0)
inline int grid_for(int64_t n, int threads = kThreads, int cap = 148 * 64) {
  int64_t g = (n + threads - 1) / threads;
  if (g < 1) g = 1;
  if (g > cap) g = cap;
  return (int)g;
}

}  // namespace lamb
