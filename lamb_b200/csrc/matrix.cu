// Context, device matrices (upload / query / download / copy) and shared
// device utilities of liblamb_b200.so.
//
// The device matrix replaces the reference's per-sector storage
// (lamb_sector_X_type + lamb_index_type + lamb_data_X_type,
// src/lamb_sector_X_types.F90:79-87, src/lamb_index_types.F90:86-105,
// src/lamb_data_X_types.F90:77-83) with one block-CSR per matrix in sector
// order; see DevMatrix in common.cuh.
#include <cub/cub.cuh>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cstdio>
#include <cstdlib>

#include "common.cuh"

namespace lamb {

int32_t fail(Ctx* ctx, int level, int type, const std::string& msg) {
  if (ctx) ctx->last_error = msg;
  return make_status(level, type);
}

int32_t dalloc_bytes(Ctx* ctx, void** p, size_t bytes) {
  *p = nullptr;
  cudaError_t e = cudaMallocAsync(p, bytes, ctx->stream);
  if (e == cudaErrorMemoryAllocation) {
    cudaGetLastError();
    cudaMemPool_t pool;
    if (cudaStreamSynchronize(ctx->stream) == cudaSuccess && cudaDeviceGetDefaultMemPool(&pool, ctx->device) == cudaSuccess &&
        cudaMemPoolTrimTo(pool, 0) == cudaSuccess)
      e = cudaMallocAsync(p, bytes, ctx->stream);
  }
  if (e != cudaSuccess) {
    cudaGetLastError();
    *p = nullptr;
    return fail(ctx, LAMB_LEVEL_MEMORY, LAMB_TYPE_EXTERNAL_ERROR,
                "device allocation of " + std::to_string(bytes) + " bytes failed: " + cudaGetErrorString(e));
  }
  return LAMB_GPU_OK;
}

int32_t scratch_bytes(Ctx* ctx, int slot, size_t bytes, void** p) {
  if (bytes > ctx->scr_bytes[slot]) {
    if (ctx->scr[slot]) cudaFreeAsync(ctx->scr[slot], ctx->stream);
    ctx->scr[slot] = nullptr;
    ctx->scr_bytes[slot] = 0;
    const size_t mib2 = size_t(2) << 20;
    size_t want = ((bytes + bytes / 16) + mib2 - 1) / mib2 * mib2;  // headroom for the next, slightly larger call
    if (dalloc_bytes(ctx, &ctx->scr[slot], want) != LAMB_GPU_OK) {
      want = bytes;
      LAMB_TRY(dalloc_bytes(ctx, &ctx->scr[slot], want));
    }
    ctx->scr_bytes[slot] = want;
  }
  *p = ctx->scr[slot];
  return LAMB_GPU_OK;
}

void release_scratch(Ctx* ctx) {
  for (int i = 0; i < kScrSlots; ++i) {
    if (ctx->scr[i]) cudaFreeAsync(ctx->scr[i], ctx->stream);
    ctx->scr[i] = nullptr;
    ctx->scr_bytes[i] = 0;
  }
}

void trace_mark(Ctx* ctx, const char* what) {
  if (!ctx->trace) return;
  if (!ctx->trace_host) cudaStreamSynchronize(ctx->stream);
  const double now =
      std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now().time_since_epoch()).count();
  std::fprintf(stderr, "[lamb trace] %-28s %10.2f ms\n", what, ctx->trace_t > 0 ? now - ctx->trace_t : 0.0);
  ctx->trace_t = now;
}

int32_t settle(Ctx* ctx) {
  DevMatrix* m = ctx->pend_m;
  if (!m) return LAMB_GPU_OK;
  ctx->pend_m = nullptr;
  LAMB_CUDA(ctx, cudaEventSynchronize(ctx->pend_ev));
  const size_t n = (size_t)m->n_rsub * m->n_csub;
  m->sec_nblk.assign(ctx->pend_h, ctx->pend_h + n);
  int64_t tot = 0;
  for (int64_t x : m->sec_nblk) tot += x;
  m->nnz = tot;
  return LAMB_GPU_OK;
}

DevMatrix* find_matrix(Ctx* ctx, lamb_gpu_matrix h) {
  auto it = ctx->mats.find(h);
  return it == ctx->mats.end() ? nullptr : it->second.get();
}

DevMatrix* get_matrix(Ctx* ctx, lamb_gpu_matrix h) {
  settle(ctx);
  return find_matrix(ctx, h);
}

void touch(DevMatrix* m) {
  static std::atomic<uint64_t> g_gen{0};
  m->gen = ++g_gen;
}

void free_matrix_buffers(Ctx* ctx, DevMatrix* m) {
  touch(m);
  dfree(ctx, m->row_bs);
  dfree(ctx, m->col_bs);
  dfree(ctx, m->row_p);
  dfree(ctx, m->col);
  dfree(ctx, m->off);
  dfree(ctx, m->data);
  m->data_cap = 0;
  dfree(ctx, m->norms);
  dfree(ctx, m->order);
  m->h_order.clear();
  m->norms_valid = false;
  m->n_chunks = 0;
  m->chunk_rng.clear();
  if (ctx->chunk_m == m) ctx->chunk_m = nullptr;
}

int32_t register_matrix(Ctx* ctx, std::unique_ptr<DevMatrix> m, lamb_gpu_matrix* h) {
  *h = ctx->next_handle++;
  touch(m.get());
  ctx->mats[*h] = std::move(m);
  return LAMB_GPU_OK;
}

void copy_structure(DevMatrix* d, const DevMatrix* r, bool rows_from_rows, const DevMatrix* c, bool cols_from_cols) {
  if (rows_from_rows) {
    d->n_rsub = r->n_rsub; d->rsub_cnt = r->rsub_cnt; d->rsub_base = r->rsub_base; d->h_row_bs = r->h_row_bs;
    d->n_rows = r->n_rows;
  } else {
    d->n_rsub = r->n_csub; d->rsub_cnt = r->csub_cnt; d->rsub_base = r->csub_base; d->h_row_bs = r->h_col_bs;
    d->n_rows = r->n_cols;
  }
  if (cols_from_cols) {
    d->n_csub = c->n_csub; d->csub_cnt = c->csub_cnt; d->csub_base = c->csub_base; d->h_col_bs = c->h_col_bs;
    d->n_cols = c->n_cols;
  } else {
    d->n_csub = c->n_rsub; d->csub_cnt = c->rsub_cnt; d->csub_base = c->rsub_base; d->h_col_bs = c->h_row_bs;
    d->n_cols = c->n_rows;
  }
}

int32_t upload_block_sizes(Ctx* ctx, DevMatrix* m) {
  LAMB_TRY(dalloc(ctx, &m->row_bs, std::max(m->n_rows, 1)));
  LAMB_TRY(dalloc(ctx, &m->col_bs, std::max(m->n_cols, 1)));
  if (m->n_rows)
    LAMB_CUDA(ctx, cudaMemcpyAsync(m->row_bs, m->h_row_bs.data(), m->n_rows, cudaMemcpyHostToDevice, ctx->stream));
  if (m->n_cols)
    LAMB_CUDA(ctx, cudaMemcpyAsync(m->col_bs, m->h_col_bs.data(), m->n_cols, cudaMemcpyHostToDevice, ctx->stream));
  return LAMB_GPU_OK;
}

// ---- scans --------------------------------------------------------------------------
int32_t exclusive_scan_i64(Ctx* ctx, const int64_t* in, int64_t* out, int64_t n) {
  if (n <= 0) return LAMB_GPU_OK;
  size_t bytes = 0;
  LAMB_CUDA(ctx, cub::DeviceScan::ExclusiveSum(nullptr, bytes, in, out, n, ctx->stream));
  void* tmp = nullptr;
  LAMB_TRY(dalloc(ctx, (char**)&tmp, (int64_t)bytes + 16));
  cudaError_t e = cub::DeviceScan::ExclusiveSum(tmp, bytes, in, out, n, ctx->stream);
  cudaFreeAsync(tmp, ctx->stream);
  LAMB_CUDA(ctx, e);
  return LAMB_GPU_OK;
}

int32_t inclusive_scan_i64(Ctx* ctx, const int64_t* in, int64_t* out, int64_t n) {
  if (n <= 0) return LAMB_GPU_OK;
  size_t bytes = 0;
  LAMB_CUDA(ctx, cub::DeviceScan::InclusiveSum(nullptr, bytes, in, out, n, ctx->stream));
  void* tmp = nullptr;
  LAMB_TRY(dalloc(ctx, (char**)&tmp, (int64_t)bytes + 16));
  cudaError_t e = cub::DeviceScan::InclusiveSum(tmp, bytes, in, out, n, ctx->stream);
  cudaFreeAsync(tmp, ctx->stream);
  LAMB_CUDA(ctx, e);
  return LAMB_GPU_OK;
}

int32_t sum_i64(Ctx* ctx, const int64_t* in, int64_t n, int64_t* host_out) {
  *host_out = 0;
  if (n <= 0) return LAMB_GPU_OK;
  int64_t* d_out = nullptr;
  LAMB_TRY(dalloc(ctx, &d_out, 1));
  size_t bytes = 0;
  LAMB_CUDA(ctx, cub::DeviceReduce::Sum(nullptr, bytes, in, d_out, n, ctx->stream));
  void* tmp = nullptr;
  LAMB_TRY(dalloc(ctx, (char**)&tmp, (int64_t)bytes + 16));
  cudaError_t e = cub::DeviceReduce::Sum(tmp, bytes, in, d_out, n, ctx->stream);
  cudaFreeAsync(tmp, ctx->stream);
  LAMB_CUDA(ctx, e);
  LAMB_CUDA(ctx, cudaMemcpyAsync(host_out, d_out, sizeof(int64_t), cudaMemcpyDeviceToHost, ctx->stream));
  LAMB_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  dfree(ctx, d_out);
  return LAMB_GPU_OK;
}

int32_t max_i64(Ctx* ctx, const int64_t* in, int64_t n, int64_t* host_out) {
  *host_out = 0;
  if (n <= 0) return LAMB_GPU_OK;
  int64_t* d_out = nullptr;
  LAMB_TRY(dalloc(ctx, &d_out, 1));
  size_t bytes = 0;
  LAMB_CUDA(ctx, cub::DeviceReduce::Max(nullptr, bytes, in, d_out, n, ctx->stream));
  void* tmp = nullptr;
  LAMB_TRY(dalloc(ctx, (char**)&tmp, (int64_t)bytes + 16));
  cudaError_t e = cub::DeviceReduce::Max(tmp, bytes, in, d_out, n, ctx->stream);
  cudaFreeAsync(tmp, ctx->stream);
  LAMB_CUDA(ctx, e);
  LAMB_CUDA(ctx, cudaMemcpyAsync(host_out, d_out, sizeof(int64_t), cudaMemcpyDeviceToHost, ctx->stream));
  LAMB_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  dfree(ctx, d_out);
  return LAMB_GPU_OK;
}

int32_t min_f64(Ctx* ctx, const double* in, int64_t n, double* host_out) {
  *host_out = 0.0;
  if (n <= 0) return LAMB_GPU_OK;
  double* d_out = nullptr;
  LAMB_TRY(dalloc(ctx, &d_out, 1));
  size_t bytes = 0;
  LAMB_CUDA(ctx, cub::DeviceReduce::Min(nullptr, bytes, in, d_out, n, ctx->stream));
  void* tmp = nullptr;
  LAMB_TRY(dalloc(ctx, (char**)&tmp, (int64_t)bytes + 16));
  cudaError_t e = cub::DeviceReduce::Min(tmp, bytes, in, d_out, n, ctx->stream);
  cudaFreeAsync(tmp, ctx->stream);
  LAMB_CUDA(ctx, e);
  LAMB_CUDA(ctx, cudaMemcpyAsync(host_out, d_out, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  LAMB_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  dfree(ctx, d_out);
  return LAMB_GPU_OK;
}

// ---- block norms -----------------------------------------------------------------------
// One warp per block row; each lane sums whole blocks sequentially (fixed order).
__global__ void k_block_norms(int32_t n_rows, const int64_t* __restrict__ row_p, const int32_t* __restrict__ col,
                              const int64_t* __restrict__ off, const int8_t* __restrict__ row_bs,
                              const int8_t* __restrict__ col_bs, const double* __restrict__ data,
                              double* __restrict__ norms) {
  const int lane = threadIdx.x & 31;
  const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t r = warp; r < n_rows; r += nwarps) {
    const int bi = row_bs[r];
    for (int64_t b = row_p[r] + lane; b < row_p[r + 1]; b += 32) {
      const int64_t n = (int64_t)bi * col_bs[col[b]];
      norms[b] = block_norm_seq(data + off[b], n);
    }
  }
}

int32_t ensure_norms(Ctx* ctx, DevMatrix* m) {
  if (m->norms_valid) return LAMB_GPU_OK;
  if (!m->norms) LAMB_TRY(dalloc(ctx, &m->norms, std::max<int64_t>(m->nnz, 1)));
  if (m->nnz > 0) {
    k_block_norms<<<grid_for((int64_t)m->n_rows * 32), kThreads, 0, ctx->stream>>>(
        m->n_rows, m->row_p, m->col, m->off, m->row_bs, m->col_bs, m->data, m->norms);
    LAMB_LAUNCHED(ctx);
  }
  m->norms_valid = true;
  return LAMB_GPU_OK;
}

// ---- sector-major layout ------------------------------------------------------------
// Part sizes: for row r (subset m, local l) and column subset n, the data
// size and block count of the row's run in sector (m,n).  Stored at
// idx(m,n,l) = rsub_base[m]*S + n*cnt[m] + l so that one exclusive scan over
// the array gives sector-major offsets.
__global__ void k_part_sizes(int32_t n_rows, int32_t n_rsub, int32_t S, const int32_t* __restrict__ rsub_base,
                             const int32_t* __restrict__ csub_base, const int64_t* __restrict__ row_p,
                             const int32_t* __restrict__ col, const int8_t* __restrict__ row_bs,
                             const int8_t* __restrict__ col_bs, const int32_t* __restrict__ lrank,
                             int64_t* __restrict__ dsz, int64_t* __restrict__ bcnt) {
  const int lane = threadIdx.x & 31;
  for (int64_t r = global_warp(); r < n_rows; r += grid_warps()) {
    const int m = row_subset(rsub_base, n_rsub, r);
    const int64_t cnt = rsub_base[m + 1] - rsub_base[m];
    const int64_t l = lrank ? lrank[r] : r - rsub_base[m];
    const int64_t base = (int64_t)rsub_base[m] * S + l;
    const long long bi = row_bs[r];
    const int64_t b1 = row_p[r + 1];
    int64_t lo = row_p[r];
    for (int n = 0; n < S; ++n) {
      const int64_t hi = lower_col(col, lo, b1, csub_base[n + 1]);
      long long ds = 0;
      for (int64_t b = lo + lane; b < hi; b += 32) ds += col_bs[col[b]];
      ds = warp_sum_ll(ds) * bi;
      if (lane == 0) {
        dsz[base + n * cnt] = ds;
        bcnt[base + n * cnt] = hi - lo;
      }
      lo = hi;
    }
  }
}

__global__ void k_part_offsets(int32_t n_rows, int32_t n_rsub, int32_t S, const int32_t* __restrict__ rsub_base,
                               const int32_t* __restrict__ csub_base, const int64_t* __restrict__ row_p,
                               const int32_t* __restrict__ col, const int8_t* __restrict__ row_bs,
                               const int8_t* __restrict__ col_bs, const int64_t* __restrict__ dbase,
                               const int32_t* __restrict__ lrank, int64_t* __restrict__ off,
                               int32_t* __restrict__ row_of) {
  const int lane = threadIdx.x & 31;
  for (int64_t r = global_warp(); r < n_rows; r += grid_warps()) {
    const int m = row_subset(rsub_base, n_rsub, r);
    const int64_t cnt = rsub_base[m + 1] - rsub_base[m];
    const int64_t l = lrank ? lrank[r] : r - rsub_base[m];
    const int64_t base = (int64_t)rsub_base[m] * S + l;
    const long long bi = row_bs[r];
    const int64_t b1 = row_p[r + 1];
    int64_t lo = row_p[r];
    for (int n = 0; n < S; ++n) {
      const int64_t hi = lower_col(col, lo, b1, csub_base[n + 1]);
      long long o = dbase[base + n * cnt];
      for (int64_t b0 = lo; b0 < hi; b0 += 32) {
        const int64_t b = b0 + lane;
        const long long v = b < hi ? bi * col_bs[col[b]] : 0;
        const long long incl = warp_incl_scan_ll(v, lane);
        if (b < hi) {
          off[b] = o + incl - v;
          if (row_of) row_of[b] = (int32_t)r;
        }
        o += __shfl_sync(0xffffffffu, incl, 31);
      }
      lo = hi;
    }
  }
}

// Sector index of every block for downloads: position bpos[idx(m,n,l)] + i
// of the i-th block of local row l in sector (m,n) in an array ordered sector
// by sector; column 1-based within the column subset, extents 1-based
// inclusive within the sector's data.
__global__ void k_sector_index(int32_t n_rows, int32_t n_rsub, int32_t S, const int32_t* __restrict__ rsub_base,
                               const int32_t* __restrict__ csub_base, const int64_t* __restrict__ row_p,
                               const int32_t* __restrict__ col, const int64_t* __restrict__ off,
                               const int8_t* __restrict__ row_bs, const int8_t* __restrict__ col_bs,
                               const int64_t* __restrict__ bpos, const int64_t* __restrict__ sec_base,
                               int16_t* __restrict__ col16, int64_t* __restrict__ ext) {
  const int lane = threadIdx.x & 31;
  for (int64_t r = global_warp(); r < n_rows; r += grid_warps()) {
    const int m = row_subset(rsub_base, n_rsub, r);
    const int64_t cnt = rsub_base[m + 1] - rsub_base[m];
    const int64_t l = r - rsub_base[m];
    const int64_t base = (int64_t)rsub_base[m] * S + l;
    const int64_t bi = row_bs[r];
    const int64_t b1 = row_p[r + 1];
    int64_t lo = row_p[r];
    for (int n = 0; n < S; ++n) {
      const int64_t hi = lower_col(col, lo, b1, csub_base[n + 1]);
      const int64_t q0 = bpos[base + n * cnt] - lo, sb = sec_base[(int64_t)m * S + n];
      for (int64_t b = lo + lane; b < hi; b += 32) {
        const int c = col[b];
        const int64_t q = q0 + b, e1 = off[b] - sb + 1;
        col16[q] = (int16_t)(c - csub_base[n] + 1);
        ext[2 * q] = e1;
        ext[2 * q + 1] = e1 + bi * col_bs[c] - 1;
      }
      lo = hi;
    }
  }
}

int32_t build_sector_index(Ctx* ctx, const DevMatrix* m, SectorIndex* si) {
  const int S = m->n_csub;
  const int64_t n_seq = (int64_t)m->n_rows * S;
  si->h_bcnt.assign(std::max<int64_t>(n_seq, 1), 0);
  if (n_seq == 0 || m->nnz == 0) return LAMB_GPU_OK;
  int64_t *d_dsz = nullptr, *d_bcnt = nullptr, *d_bpos = nullptr, *d_sbase = nullptr;
  int32_t *d_rb = nullptr, *d_cb = nullptr;
  LAMB_TRY(dalloc(ctx, &si->col16, m->nnz));
  LAMB_TRY(dalloc(ctx, &si->ext, 2 * m->nnz));
  LAMB_TRY(dalloc(ctx, &d_dsz, n_seq));
  LAMB_TRY(dalloc(ctx, &d_bcnt, n_seq));
  LAMB_TRY(dalloc(ctx, &d_bpos, n_seq));
  LAMB_TRY(dalloc(ctx, &d_sbase, (int64_t)m->sec_base.size()));
  LAMB_TRY(dalloc(ctx, &d_rb, m->n_rsub + 1));
  LAMB_TRY(dalloc(ctx, &d_cb, S + 1));
  // the host vectors copied from are members of m: they outlive the copies
  LAMB_CUDA(ctx, cudaMemcpyAsync(d_sbase, m->sec_base.data(), sizeof(int64_t) * m->sec_base.size(), cudaMemcpyHostToDevice, ctx->stream));
  LAMB_CUDA(ctx, cudaMemcpyAsync(d_rb, m->rsub_base.data(), sizeof(int32_t) * (m->n_rsub + 1), cudaMemcpyHostToDevice, ctx->stream));
  LAMB_CUDA(ctx, cudaMemcpyAsync(d_cb, m->csub_base.data(), sizeof(int32_t) * (S + 1), cudaMemcpyHostToDevice, ctx->stream));
  k_part_sizes<<<grid_for(32ll * m->n_rows, 256), 256, 0, ctx->stream>>>(m->n_rows, m->n_rsub, S, d_rb, d_cb, m->row_p,
                                                                    m->col, m->row_bs, m->col_bs, nullptr, d_dsz, d_bcnt);
  LAMB_LAUNCHED(ctx);
  LAMB_TRY(exclusive_scan_i64(ctx, d_bcnt, d_bpos, n_seq));
  k_sector_index<<<grid_for(32ll * m->n_rows, 256), 256, 0, ctx->stream>>>(m->n_rows, m->n_rsub, S, d_rb, d_cb, m->row_p,
                                                                      m->col, m->off, m->row_bs, m->col_bs, d_bpos,
                                                                      d_sbase, si->col16, si->ext);
  LAMB_LAUNCHED(ctx);
  LAMB_CUDA(ctx, cudaMemcpyAsync(si->h_bcnt.data(), d_bcnt, sizeof(int64_t) * n_seq, cudaMemcpyDeviceToHost, ctx->stream));
  dfree(ctx, d_dsz); dfree(ctx, d_bcnt); dfree(ctx, d_bpos); dfree(ctx, d_sbase); dfree(ctx, d_rb); dfree(ctx, d_cb);
  return LAMB_GPU_OK;
}

void free_sector_index(Ctx* ctx, SectorIndex* si) {
  dfree(ctx, si->col16);
  dfree(ctx, si->ext);
}

int32_t layout_sector_major(Ctx* ctx, DevMatrix* m, int32_t* row_of, bool by_order, std::vector<int64_t>* h_base_out) {
  const int S = m->n_csub;
  const int64_t n_seq = (int64_t)m->n_rows * S;
  // Rank of every row among the rows of its subset, in the processing order
  // (h_order), when the rows' data should follow that order.
  std::vector<int32_t> h_rank;
  int32_t* d_rank = nullptr;
  if (by_order && (int64_t)m->h_order.size() == m->n_rows && m->n_rows > 0) {
    h_rank.resize(m->n_rows);
    std::vector<int32_t> next(m->n_rsub, 0), sub_of(m->n_rows);
    for (int a = 0; a < m->n_rsub; ++a)
      for (int r = m->rsub_base[a]; r < m->rsub_base[a + 1]; ++r) sub_of[r] = a;
    for (int32_t r : m->h_order) h_rank[r] = next[sub_of[r]]++;
  }
  m->sec_base.assign((size_t)m->n_rsub * S, 0);
  m->sec_dlen.assign((size_t)m->n_rsub * S, 0);
  m->sec_nblk.assign((size_t)m->n_rsub * S, 0);
  if (!m->off) LAMB_TRY(dalloc(ctx, &m->off, std::max<int64_t>(m->nnz, 1)));
  if (n_seq == 0) { m->data_len = 0; return LAMB_GPU_OK; }
  int32_t *d_rb = nullptr, *d_cb = nullptr;
  int64_t *dsz = nullptr, *bcnt = nullptr, *dbase = nullptr;
  LAMB_TRY(dalloc(ctx, &d_rb, m->n_rsub + 1));
  LAMB_TRY(dalloc(ctx, &d_cb, S + 1));
  LAMB_TRY(dalloc(ctx, &dsz, n_seq));
  LAMB_TRY(dalloc(ctx, &bcnt, n_seq));
  LAMB_TRY(dalloc(ctx, &dbase, n_seq));
  if (!h_rank.empty()) {
    LAMB_TRY(dalloc(ctx, &d_rank, m->n_rows));
    LAMB_CUDA(ctx, cudaMemcpyAsync(d_rank, h_rank.data(), sizeof(int32_t) * m->n_rows, cudaMemcpyHostToDevice, ctx->stream));
  }
  LAMB_CUDA(ctx, cudaMemcpyAsync(d_rb, m->rsub_base.data(), sizeof(int32_t) * (m->n_rsub + 1), cudaMemcpyHostToDevice, ctx->stream));
  LAMB_CUDA(ctx, cudaMemcpyAsync(d_cb, m->csub_base.data(), sizeof(int32_t) * (S + 1), cudaMemcpyHostToDevice, ctx->stream));
  k_part_sizes<<<grid_for(32ll * m->n_rows, 256), 256, 0, ctx->stream>>>(m->n_rows, m->n_rsub, S, d_rb, d_cb, m->row_p,
                                                                    m->col, m->row_bs, m->col_bs, d_rank, dsz, bcnt);
  LAMB_LAUNCHED(ctx);
  LAMB_TRY(exclusive_scan_i64(ctx, dsz, dbase, n_seq));
  k_part_offsets<<<grid_for(32ll * m->n_rows, 256), 256, 0, ctx->stream>>>(m->n_rows, m->n_rsub, S, d_rb, d_cb, m->row_p,
                                                                      m->col, m->row_bs, m->col_bs, dbase, d_rank,
                                                                      m->off, row_of);
  LAMB_LAUNCHED(ctx);
  std::vector<int64_t> h_dsz(n_seq), h_bcnt(n_seq), h_dbase(n_seq);
  LAMB_CUDA(ctx, cudaMemcpyAsync(h_dsz.data(), dsz, sizeof(int64_t) * n_seq, cudaMemcpyDeviceToHost, ctx->stream));
  LAMB_CUDA(ctx, cudaMemcpyAsync(h_bcnt.data(), bcnt, sizeof(int64_t) * n_seq, cudaMemcpyDeviceToHost, ctx->stream));
  LAMB_CUDA(ctx, cudaMemcpyAsync(h_dbase.data(), dbase, sizeof(int64_t) * n_seq, cudaMemcpyDeviceToHost, ctx->stream));
  LAMB_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  for (int a = 0; a < m->n_rsub; ++a)
    for (int n = 0; n < S; ++n) {
      const int64_t cnt = m->rsub_cnt[a];
      const int64_t first = (int64_t)m->rsub_base[a] * S + n * cnt;
      int64_t dl = 0, nb = 0;
      for (int64_t l = 0; l < cnt; ++l) { dl += h_dsz[first + l]; nb += h_bcnt[first + l]; }
      const size_t s = (size_t)a * S + n;
      m->sec_base[s] = cnt ? h_dbase[first] : (s ? m->sec_base[s - 1] + m->sec_dlen[s - 1] : 0);
      m->sec_dlen[s] = dl;
      m->sec_nblk[s] = nb;
    }
  m->data_len = h_dbase[n_seq - 1] + h_dsz[n_seq - 1];
  if (h_base_out) *h_base_out = std::move(h_dbase);
  dfree(ctx, d_rb); dfree(ctx, d_cb); dfree(ctx, dsz); dfree(ctx, bcnt); dfree(ctx, dbase); dfree(ctx, d_rank);
  return LAMB_GPU_OK;
}

// ---- row processing order ------------------------------------------------------------
// Morton (Z-order) key of a point in the periodic cell, 10 bits per axis.
static uint32_t morton3(float x, float y, float z, const float* box) {
  auto q = [](float v, float L) {
    float f = v / L;
    f -= floorf(f);
    int c = (int)(f * 1024.0f);
    return (uint32_t)(c < 0 ? 0 : (c > 1023 ? 1023 : c));
  };
  auto spread = [](uint32_t v) {
    v = (v | (v << 16)) & 0x030000FFu;
    v = (v | (v << 8)) & 0x0300F00Fu;
    v = (v | (v << 4)) & 0x030C30C3u;
    v = (v | (v << 2)) & 0x09249249u;
    return v;
  };
  return spread(q(x, box[0])) | (spread(q(y, box[1])) << 1) | (spread(q(z, box[2])) << 2);
}

// Cuthill-McKee: BFS from a pseudo-peripheral row, neighbours by increasing
// degree.  Uses the block pattern as a graph (columns index the same atoms as
// rows when the matrix is square in atoms).
static void cuthill_mckee(int n, const std::vector<int64_t>& rp, const std::vector<int32_t>& cl,
                          std::vector<int32_t>& order) {
  order.clear();
  order.reserve(n);
  std::vector<int32_t> deg(n), level(n, -1);
  for (int i = 0; i < n; ++i) deg[i] = (int32_t)(rp[i + 1] - rp[i]);
  auto bfs_last = [&](int s) {
    std::vector<int32_t> q{s};
    std::fill(level.begin(), level.end(), -1);
    level[s] = 0;
    for (size_t h = 0; h < q.size(); ++h)
      for (int64_t b = rp[q[h]]; b < rp[q[h] + 1]; ++b) {
        int j = cl[b];
        if (j < n && level[j] < 0) { level[j] = level[q[h]] + 1; q.push_back(j); }
      }
    return q.back();
  };
  std::vector<char> seen(n, 0);
  std::vector<int32_t> nb;
  for (int start = 0; start < n; ++start) {
    if (seen[start]) continue;
    int s = bfs_last(bfs_last(start));
    if (seen[s]) s = start;
    size_t h = order.size();
    order.push_back(s);
    seen[s] = 1;
    for (; h < order.size(); ++h) {
      nb.clear();
      for (int64_t b = rp[order[h]]; b < rp[order[h] + 1]; ++b) {
        int j = cl[b];
        if (j < n && !seen[j]) { seen[j] = 1; nb.push_back(j); }
      }
      std::sort(nb.begin(), nb.end(), [&](int x, int y) { return deg[x] < deg[y] || (deg[x] == deg[y] && x < y); });
      order.insert(order.end(), nb.begin(), nb.end());
    }
  }
}

int32_t ensure_row_order(Ctx* ctx, DevMatrix* m) {
  if (!m->h_order.empty() || m->n_rows == 0) {
    if (m->n_rows && !m->order) {
      LAMB_TRY(dalloc(ctx, &m->order, m->n_rows));
      LAMB_CUDA(ctx, cudaMemcpyAsync(m->order, m->h_order.data(), sizeof(int32_t) * m->n_rows,
                                     cudaMemcpyHostToDevice, ctx->stream));
    }
    return LAMB_GPU_OK;
  }
  const int n = m->n_rows;
  std::vector<int32_t> ord(n);
  if ((int64_t)m->h_pos.size() == 3ll * n) {
    std::vector<std::pair<uint32_t, int32_t>> key(n);
    for (int i = 0; i < n; ++i) key[i] = {morton3(m->h_pos[3 * i], m->h_pos[3 * i + 1], m->h_pos[3 * i + 2], m->box), i};
    std::sort(key.begin(), key.end());
    for (int i = 0; i < n; ++i) ord[i] = key[i].second;
  } else if (m->n_cols == m->n_rows && m->nnz > 0) {
    std::vector<int64_t> rp(n + 1);
    std::vector<int32_t> cl(m->nnz);
    LAMB_CUDA(ctx, cudaMemcpyAsync(rp.data(), m->row_p, sizeof(int64_t) * (n + 1), cudaMemcpyDeviceToHost, ctx->stream));
    LAMB_CUDA(ctx, cudaMemcpyAsync(cl.data(), m->col, sizeof(int32_t) * m->nnz, cudaMemcpyDeviceToHost, ctx->stream));
    LAMB_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    cuthill_mckee(n, rp, cl, ord);
  } else {
    for (int i = 0; i < n; ++i) ord[i] = i;
  }
  m->h_order.swap(ord);
  dfree(ctx, m->order);
  return ensure_row_order(ctx, m);
}

int32_t inherit_row_locality(Ctx* ctx, DevMatrix* dst, const DevMatrix* src) {
  if (dst->n_rows != src->n_rows) return LAMB_GPU_OK;
  dst->h_pos = src->h_pos;
  memcpy(dst->box, src->box, sizeof(dst->box));
  dst->h_order = src->h_order;
  dfree(ctx, dst->order);
  return LAMB_GPU_OK;
}

// ---- sector structure validation ------------------------------------------------
static int32_t check_sector(Ctx* ctx, const lamb_c_sector& s, int idx) {
  auto bad = [&](const std::string& w) {
    return fail(ctx, LAMB_LEVEL_FAILURE, LAMB_TYPE_WRONG_ARGS, "sector " + std::to_string(idx) + ": " + w);
  };
  if (s.subset_row < 1 || s.subset_col < 1) return bad("subset positions must be >= 1");
  if (s.n_rows < 0 || s.n_cols < 0 || s.n_blks < 0 || s.data_len < 0) return bad("negative size");
  if (s.n_cols > 32767 || s.n_rows > 32767) return bad("more than 32767 atoms in a subset (int16 local index)");
  if (!s.row_p) return bad("row_p is NULL");
  if (s.n_rows && (!s.row_blk_sizes)) return bad("row_blk_sizes is NULL");
  if (s.n_cols && (!s.col_blk_sizes)) return bad("col_blk_sizes is NULL");
  if (s.n_blks && (!s.col_i || !s.extents)) return bad("col_i/extents is NULL");
  if (s.data_len && !s.data) return bad("data is NULL");
  if (s.row_p[0] != 0) return bad("row_p[0] must be 0");
  if (s.row_p[s.n_rows] != s.n_blks) return bad("row_p[n_rows] must equal n_blks");
  for (int32_t r = 0; r < s.n_rows; ++r) {
    if (s.row_blk_sizes[r] < 0) return bad("negative block size");
    if (s.row_p[r + 1] < s.row_p[r]) return bad("row_p must be non-decreasing");
    int prev = 0;
    for (int64_t b = s.row_p[r]; b < s.row_p[r + 1]; ++b) {
      const int c = s.col_i[b];
      if (c < 1 || c > s.n_cols) return bad("col_i out of range at block " + std::to_string(b));
      if (c <= prev) return bad("col_i not strictly increasing in row " + std::to_string(r + 1));
      prev = c;
      const int64_t sz = (int64_t)s.row_blk_sizes[r] * s.col_blk_sizes[c - 1];
      const int64_t f = s.extents[2 * b], l = s.extents[2 * b + 1];
      if (l - f + 1 != sz) return bad("extent length does not match block size at block " + std::to_string(b));
      if (sz > 0 && (f < 1 || l > s.data_len)) return bad("extent outside data at block " + std::to_string(b));
    }
  }
  for (int32_t c = 0; c < s.n_cols; ++c)
    if (s.col_blk_sizes[c] < 0) return bad("negative block size");
  return LAMB_GPU_OK;
}

}  // namespace lamb

using namespace lamb;

// ============================== C ABI ========================================
extern "C" {

int32_t lamb_gpu_status_level(int32_t status) { return status == 0 ? 0 : status / 100000; }
int32_t lamb_gpu_status_type(int32_t status) { return status == 0 ? 0 : status % 100000 - 50000; }

int32_t lamb_gpu_ctx_create(int32_t device, lamb_gpu_ctx** out) {
  if (!out) return make_status(LAMB_LEVEL_FAILURE, LAMB_TYPE_WRONG_ARGS);
  *out = nullptr;
  int n = 0;
  cudaError_t e = cudaGetDeviceCount(&n);
  if (e != cudaSuccess || n == 0) return make_status(LAMB_LEVEL_FAILURE, LAMB_TYPE_EXTERNAL_ERROR);
  if (device < 0 || device >= n) return make_status(LAMB_LEVEL_FAILURE, LAMB_TYPE_WRONG_ARGS);
  cudaDeviceProp p;
  if (cudaGetDeviceProperties(&p, device) != cudaSuccess || p.major < 10)
    return make_status(LAMB_LEVEL_FAILURE, LAMB_TYPE_UNIMPLEMENTED);  // built for sm_100a only
  if (cudaSetDevice(device) != cudaSuccess) return make_status(LAMB_LEVEL_FAILURE, LAMB_TYPE_EXTERNAL_ERROR);
  auto* ctx = new Ctx;
  ctx->device = device;
  if (cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) != cudaSuccess) {
    delete ctx;
    return make_status(LAMB_LEVEL_FAILURE, LAMB_TYPE_EXTERNAL_ERROR);
  }
  for (auto& ev : ctx->ev) cudaEventCreate(&ev);
  for (auto& ev : ctx->chunk_ev) cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
  for (auto& row : ctx->kern_ev)
    for (auto& ev : row) cudaEventCreate(&ev);
  cudaStreamCreateWithFlags(&ctx->copy_stream, cudaStreamNonBlocking);
  if (const char* t = std::getenv("LAMB_GPU_TRACE")) {
    ctx->trace = t[0] == '1' || t[0] == '2';
    ctx->trace_host = t[0] == '2';
  }
  // Keep freed stream-ordered memory in the pool between calls.
  cudaMemPool_t pool;
  if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
    uint64_t thr = UINT64_MAX;
    cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
  }
  *out = reinterpret_cast<lamb_gpu_ctx*>(ctx);
  return LAMB_GPU_OK;
}

int32_t lamb_gpu_ctx_destroy(lamb_gpu_ctx* c) {
  auto* ctx = reinterpret_cast<Ctx*>(c);
  if (!ctx) return LAMB_GPU_OK;
  cudaSetDevice(ctx->device);
  settle(ctx);
  for (auto& kv : ctx->mats) free_matrix_buffers(ctx, kv.second.get());
  ctx->mats.clear();
  release_scratch(ctx);
  cudaStreamSynchronize(ctx->stream);
  for (auto& ev : ctx->ev) cudaEventDestroy(ev);
  for (auto& ev : ctx->chunk_ev) cudaEventDestroy(ev);
  for (auto& row : ctx->kern_ev)
    for (auto& ev : row) cudaEventDestroy(ev);
  if (ctx->copy_stream) cudaStreamDestroy(ctx->copy_stream);
  if (ctx->pend_ev) cudaEventDestroy(ctx->pend_ev);
  if (ctx->pend_h) cudaFreeHost(ctx->pend_h);
  cudaStreamDestroy(ctx->stream);
  delete ctx;
  return LAMB_GPU_OK;
}

int32_t lamb_gpu_last_error(const lamb_gpu_ctx* c, char* msg, int32_t len) {
  auto* ctx = reinterpret_cast<const Ctx*>(c);
  if (!msg || len <= 0) return make_status(LAMB_LEVEL_FAILURE, LAMB_TYPE_WRONG_ARGS);
  const std::string& s = ctx ? ctx->last_error : std::string("no context");
  size_t n = std::min<size_t>(s.size(), (size_t)len - 1);
  memcpy(msg, s.data(), n);
  msg[n] = 0;
  return LAMB_GPU_OK;
}

int32_t lamb_gpu_ctx_get_stream(const lamb_gpu_ctx* c, void** stream) {
  auto* ctx = reinterpret_cast<const Ctx*>(c);
  if (!ctx || !stream) return make_status(LAMB_LEVEL_FAILURE, LAMB_TYPE_WRONG_ARGS);
  *stream = (void*)ctx->stream;
  return LAMB_GPU_OK;
}

int32_t lamb_gpu_ctx_synchronize(lamb_gpu_ctx* c) {
  auto* ctx = reinterpret_cast<Ctx*>(c);
  if (!ctx) return make_status(LAMB_LEVEL_FAILURE, LAMB_TYPE_WRONG_ARGS);
  LAMB_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return LAMB_GPU_OK;
}

int32_t lamb_gpu_matrix_upload(lamb_gpu_ctx* c, const lamb_c_sector* sec, int32_t n_sec, lamb_gpu_matrix* handle) {
  auto* ctx = reinterpret_cast<Ctx*>(c);
  if (!ctx) return make_status(LAMB_LEVEL_FAILURE, LAMB_TYPE_WRONG_ARGS);
  if (!handle || n_sec < 0 || (n_sec && !sec))
    return fail(ctx, LAMB_LEVEL_FAILURE, LAMB_TYPE_WRONG_ARGS, "upload: bad arguments");
  *handle = 0;
  cudaSetDevice(ctx->device);
  for (int i = 0; i < n_sec; ++i) LAMB_TRY(check_sector(ctx, sec[i], i));
  auto m = std::make_unique<DevMatrix>();
  for (int i = 0; i < n_sec; ++i) {
    m->n_rsub = std::max(m->n_rsub, sec[i].subset_row);
    m->n_csub = std::max(m->n_csub, sec[i].subset_col);
  }
  const int R = m->n_rsub, S = m->n_csub;
  std::vector<int> sid((size_t)R * S, -1);
  std::vector<const int8_t*> rbs(R, nullptr), cbs(S, nullptr);
  m->rsub_cnt.assign(R, -1);
  m->csub_cnt.assign(S, -1);
  for (int i = 0; i < n_sec; ++i) {
    const auto& s = sec[i];
    const size_t k = (size_t)(s.subset_row - 1) * S + (s.subset_col - 1);
    if (sid[k] >= 0) return fail(ctx, LAMB_LEVEL_FAILURE, LAMB_TYPE_WRONG_ARGS, "duplicate sector");
    sid[k] = i;
    int& rc = m->rsub_cnt[s.subset_row - 1];
    if (rc < 0) { rc = s.n_rows; rbs[s.subset_row - 1] = s.row_blk_sizes; }
    else if (rc != s.n_rows || memcmp(rbs[s.subset_row - 1], s.row_blk_sizes, s.n_rows))
      return fail(ctx, LAMB_LEVEL_FAILURE, LAMB_TYPE_WRONG_ARGS, "row subset sizes differ between sectors");
    int& cc = m->csub_cnt[s.subset_col - 1];
    if (cc < 0) { cc = s.n_cols; cbs[s.subset_col - 1] = s.col_blk_sizes; }
    else if (cc != s.n_cols || memcmp(cbs[s.subset_col - 1], s.col_blk_sizes, s.n_cols))
      return fail(ctx, LAMB_LEVEL_FAILURE, LAMB_TYPE_WRONG_ARGS, "column subset sizes differ between sectors");
  }
  for (int a = 0; a < R; ++a)
    if (m->rsub_cnt[a] < 0) return fail(ctx, LAMB_LEVEL_FAILURE, LAMB_TYPE_WRONG_ARGS, "a row subset has no sector");
  for (int a = 0; a < S; ++a)
    if (m->csub_cnt[a] < 0) return fail(ctx, LAMB_LEVEL_FAILURE, LAMB_TYPE_WRONG_ARGS, "a column subset has no sector");
  m->rsub_base.assign(R + 1, 0);
  m->csub_base.assign(S + 1, 0);
  for (int a = 0; a < R; ++a) m->rsub_base[a + 1] = m->rsub_base[a] + m->rsub_cnt[a];
  for (int a = 0; a < S; ++a) m->csub_base[a + 1] = m->csub_base[a] + m->csub_cnt[a];
  m->n_rows = m->rsub_base[R];
  m->n_cols = m->csub_base[S];
  m->h_row_bs.resize(m->n_rows);
  m->h_col_bs.resize(m->n_cols);
  for (int a = 0; a < R; ++a) if (m->rsub_cnt[a]) memcpy(&m->h_row_bs[m->rsub_base[a]], rbs[a], m->rsub_cnt[a]);
  for (int a = 0; a < S; ++a) if (m->csub_cnt[a]) memcpy(&m->h_col_bs[m->csub_base[a]], cbs[a], m->csub_cnt[a]);
  // Global CSR (host), sector-major data.
  m->sec_base.assign((size_t)R * S, 0);
  m->sec_dlen.assign((size_t)R * S, 0);
  m->sec_nblk.assign((size_t)R * S, 0);
  int64_t dpos = 0, nnz = 0;
  for (size_t k = 0; k < sid.size(); ++k) {
    m->sec_base[k] = dpos;
    if (sid[k] >= 0) {
      m->sec_dlen[k] = sec[sid[k]].data_len;
      m->sec_nblk[k] = sec[sid[k]].n_blks;
      dpos += sec[sid[k]].data_len;
      nnz += sec[sid[k]].n_blks;
    }
  }
  m->data_len = dpos;
  m->nnz = nnz;
  // Block data first: the copies run while the index is built on the host.
  LAMB_TRY(dalloc(ctx, &m->data, std::max<int64_t>(m->data_len, 1)));
  for (size_t k = 0; k < sid.size(); ++k)
    if (sid[k] >= 0 && sec[sid[k]].data_len > 0)
      LAMB_CUDA(ctx, cudaMemcpyAsync(m->data + m->sec_base[k], sec[sid[k]].data, sizeof(double) * sec[sid[k]].data_len,
                                     cudaMemcpyDefault, ctx->stream));
  std::vector<int64_t> h_row_p(m->n_rows + 1, 0), h_off(nnz);
  std::vector<int32_t> h_col(nnz);
  int64_t p = 0;
  for (int a = 0; a < R; ++a)
    for (int l = 0; l < m->rsub_cnt[a]; ++l) {
      for (int n = 0; n < S; ++n) {
        const int i = sid[(size_t)a * S + n];
        if (i < 0) continue;
        const auto& s = sec[i];
        for (int64_t b = s.row_p[l]; b < s.row_p[l + 1]; ++b) {
          h_col[p] = m->csub_base[n] + s.col_i[b] - 1;
          const int64_t sz = s.extents[2 * b + 1] - s.extents[2 * b] + 1;
          h_off[p] = m->sec_base[(size_t)a * S + n] + (sz > 0 ? s.extents[2 * b] - 1 : 0);
          ++p;
        }
      }
      h_row_p[m->rsub_base[a] + l + 1] = p;
    }
  LAMB_TRY(upload_block_sizes(ctx, m.get()));
  LAMB_TRY(dalloc(ctx, &m->row_p, m->n_rows + 1));
  LAMB_TRY(dalloc(ctx, &m->col, std::max<int64_t>(nnz, 1)));
  LAMB_TRY(dalloc(ctx, &m->off, std::max<int64_t>(nnz, 1)));
  LAMB_CUDA(ctx, cudaMemcpyAsync(m->row_p, h_row_p.data(), sizeof(int64_t) * (m->n_rows + 1), cudaMemcpyHostToDevice, ctx->stream));
  if (nnz) {
    LAMB_CUDA(ctx, cudaMemcpyAsync(m->col, h_col.data(), sizeof(int32_t) * nnz, cudaMemcpyHostToDevice, ctx->stream));
    LAMB_CUDA(ctx, cudaMemcpyAsync(m->off, h_off.data(), sizeof(int64_t) * nnz, cudaMemcpyHostToDevice, ctx->stream));
  }
  // The host vectors above die at return: wait for the copies.
  LAMB_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return register_matrix(ctx, std::move(m), handle);
}

int32_t lamb_gpu_matrix_create_like(lamb_gpu_ctx* c, lamb_gpu_matrix like, lamb_gpu_matrix* handle) {
  auto* ctx = reinterpret_cast<Ctx*>(c);
  if (!ctx || !handle) return make_status(LAMB_LEVEL_FAILURE, LAMB_TYPE_WRONG_ARGS);
  DevMatrix* src = get_matrix(ctx, like);
  if (!src) return fail(ctx, LAMB_LEVEL_FAILURE, LAMB_TYPE_WRONG_ARGS, "create_like: invalid handle");
  cudaSetDevice(ctx->device);
  auto m = std::make_unique<DevMatrix>();
  copy_structure(m.get(), src, true, src, true);
  LAMB_TRY(upload_block_sizes(ctx, m.get()));
  LAMB_TRY(dalloc(ctx, &m->row_p, m->n_rows + 1));
  LAMB_CUDA(ctx, cudaMemsetAsync(m->row_p, 0, sizeof(int64_t) * (m->n_rows + 1), ctx->stream));
  m->sec_base.assign((size_t)m->n_rsub * m->n_csub, 0);
  m->sec_dlen.assign((size_t)m->n_rsub * m->n_csub, 0);
  m->sec_nblk.assign((size_t)m->n_rsub * m->n_csub, 0);
  return register_matrix(ctx, std::move(m), handle);
}

int32_t lamb_gpu_matrix_destroy(lamb_gpu_ctx* c, lamb_gpu_matrix h) {
  auto* ctx = reinterpret_cast<Ctx*>(c);
  if (!ctx) return make_status(LAMB_LEVEL_FAILURE, LAMB_TYPE_WRONG_ARGS);
  settle(ctx);
  auto it = ctx->mats.find(h);
  if (it == ctx->mats.end()) return fail(ctx, LAMB_LEVEL_WARNING, LAMB_TYPE_WRONG_ARGS, "destroy: invalid handle");
  cudaSetDevice(ctx->device);
  free_matrix_buffers(ctx, it->second.get());
  ctx->mats.erase(it);
  return LAMB_GPU_OK;
}

int32_t lamb_gpu_matrix_set_positions(lamb_gpu_ctx* c, lamb_gpu_matrix h, const float* xyz, int32_t n_rows,
                                      const float* box) {
  auto* ctx = reinterpret_cast<Ctx*>(c);
  if (!ctx) return make_status(LAMB_LEVEL_FAILURE, LAMB_TYPE_WRONG_ARGS);
  DevMatrix* m = get_matrix(ctx, h);
  if (!m) return fail(ctx, LAMB_LEVEL_FAILURE, LAMB_TYPE_WRONG_ARGS, "set_positions: invalid handle");
  if (!xyz || !box || n_rows != m->n_rows)
    return fail(ctx, LAMB_LEVEL_FAILURE, LAMB_TYPE_WRONG_ARGS, "set_positions: need 3*n_rows coordinates and box[3]");
  for (int d = 0; d < 3; ++d)
    if (!(box[d] > 0)) return fail(ctx, LAMB_LEVEL_FAILURE, LAMB_TYPE_WRONG_ARGS, "set_positions: box must be positive");
  m->h_pos.assign(xyz, xyz + 3 * (size_t)n_rows);
  memcpy(m->box, box, sizeof(m->box));
  m->h_order.clear();
  dfree(ctx, m->order);
  return LAMB_GPU_OK;
}

int32_t lamb_gpu_matrix_n_sectors(lamb_gpu_ctx* c, lamb_gpu_matrix h, int32_t* n) {
  auto* ctx = reinterpret_cast<Ctx*>(c);
  if (!ctx || !n) return make_status(LAMB_LEVEL_FAILURE, LAMB_TYPE_WRONG_ARGS);
  DevMatrix* m = find_matrix(ctx, h);
  if (!m) return fail(ctx, LAMB_LEVEL_FAILURE, LAMB_TYPE_WRONG_ARGS, "invalid handle");
  *n = m->n_rsub * m->n_csub;
  return LAMB_GPU_OK;
}

int32_t lamb_gpu_matrix_query(lamb_gpu_ctx* c, lamb_gpu_matrix h, lamb_c_sector_sizes* sizes, int32_t n) {
  auto* ctx = reinterpret_cast<Ctx*>(c);
  if (!ctx) return make_status(LAMB_LEVEL_FAILURE, LAMB_TYPE_WRONG_ARGS);
  // No settle(): after a LAMB_GPU_ASYNC multiply the block counts are the
  // counts before the result filter (capacities that suffice for download).
  DevMatrix* m = find_matrix(ctx, h);
  if (!m) return fail(ctx, LAMB_LEVEL_FAILURE, LAMB_TYPE_WRONG_ARGS, "invalid handle");
  if (!sizes || n != m->n_rsub * m->n_csub)
    return fail(ctx, LAMB_LEVEL_FAILURE, LAMB_TYPE_WRONG_ARGS, "query: sizes array must hold n_sectors entries");
  for (int a = 0; a < m->n_rsub; ++a)
    for (int b = 0; b < m->n_csub; ++b) {
      auto& o = sizes[a * m->n_csub + b];
      o.subset_row = a + 1;
      o.subset_col = b + 1;
      o.n_rows = m->rsub_cnt[a];
      o.n_cols = m->csub_cnt[b];
      o.n_blks = m->sec_nblk[(size_t)a * m->n_csub + b];
      o.data_len = m->sec_dlen[(size_t)a * m->n_csub + b];
    }
  return LAMB_GPU_OK;
}

int32_t lamb_gpu_matrix_download(lamb_gpu_ctx* c, lamb_gpu_matrix h, lamb_c_sector_out* out, int32_t n) {
  auto* ctx = reinterpret_cast<Ctx*>(c);
  if (!ctx) return make_status(LAMB_LEVEL_FAILURE, LAMB_TYPE_WRONG_ARGS);
  // The data copies may start before a pending result filter completes (the
  // filter moves no data); settle() comes after they are queued.
  DevMatrix* m = find_matrix(ctx, h);
  if (!m) return fail(ctx, LAMB_LEVEL_FAILURE, LAMB_TYPE_WRONG_ARGS, "invalid handle");
  if (!out || n != m->n_rsub * m->n_csub)
    return fail(ctx, LAMB_LEVEL_FAILURE, LAMB_TYPE_WRONG_ARGS, "download: out array must hold n_sectors entries");
  cudaSetDevice(ctx->device);
  const int S = m->n_csub;
  for (int a = 0; a < m->n_rsub; ++a)
    for (int b = 0; b < S; ++b) {
      auto& o = out[a * S + b];
      const size_t s = (size_t)a * S + b;
      if (o.data_len < m->sec_dlen[s])
        return fail(ctx, LAMB_LEVEL_FAILURE, LAMB_TYPE_WRONG_ARGS, "download: capacity below queried size");
      if ((m->sec_dlen[s] && !o.data) || !o.row_p)
        return fail(ctx, LAMB_LEVEL_FAILURE, LAMB_TYPE_WRONG_ARGS, "download: NULL output array");
    }
  // Data first (largest copies), straight into the caller's arrays.  A
  // multiply's result computed in row chunks goes chunk by chunk on the copy
  // stream, each chunk after its event: the transfer overlaps the chunks still
  // being computed.
  const size_t n_sec = (size_t)m->n_rsub * S;
  bool chunked = ctx->chunk_m == m && m->n_chunks > 0 && m->chunk_data == m->data &&
                 m->chunk_rng.size() == 2 * (size_t)m->n_chunks * n_sec;
  for (size_t s = 0; chunked && s < n_sec; ++s)  // the chunks must tile every sector's data
    for (int p = 0; p < m->n_chunks; ++p) {
      const int64_t b0 = m->chunk_rng[2 * (p * n_sec + s)], b1 = m->chunk_rng[2 * (p * n_sec + s) + 1];
      const int64_t prev = p ? m->chunk_rng[2 * ((p - 1) * n_sec + s) + 1] : 0;
      if (b0 != prev || b1 < b0 || (p == m->n_chunks - 1 && b1 != m->sec_dlen[s])) chunked = false;
    }
  if (chunked) {
    for (int p = 0; p < m->n_chunks; ++p) {
      LAMB_CUDA(ctx, cudaStreamWaitEvent(ctx->copy_stream, ctx->chunk_ev[p], 0));
      for (size_t s = 0; s < n_sec; ++s) {
        const int64_t b0 = m->chunk_rng[2 * (p * n_sec + s)], b1 = m->chunk_rng[2 * (p * n_sec + s) + 1];
        if (b1 > b0)
          LAMB_CUDA(ctx, cudaMemcpyAsync(out[s].data + b0, m->data + m->sec_base[s] + b0, sizeof(double) * (b1 - b0),
                                         cudaMemcpyDeviceToHost, ctx->copy_stream));
      }
    }
  } else {
    for (size_t s = 0; s < n_sec; ++s)
      if (m->sec_dlen[s])
        LAMB_CUDA(ctx, cudaMemcpyAsync(out[s].data, m->data + m->sec_base[s], sizeof(double) * m->sec_dlen[s],
                                       cudaMemcpyDeviceToHost, ctx->stream));
  }
  LAMB_TRY(settle(ctx));
  for (size_t s = 0; s < n_sec; ++s) {
    if (out[s].n_blks < m->sec_nblk[s])
      return fail(ctx, LAMB_LEVEL_FAILURE, LAMB_TYPE_WRONG_ARGS, "download: capacity below queried size");
    if (m->sec_nblk[s] && (!out[s].col_i || !out[s].extents))
      return fail(ctx, LAMB_LEVEL_FAILURE, LAMB_TYPE_WRONG_ARGS, "download: NULL output array");
  }
  // Sector indices (1-based int16 columns, 1-based extents) are built on the
  // device in one array ordered sector by sector, then copied per sector.
  SectorIndex si;
  LAMB_TRY(build_sector_index(ctx, m, &si));
  {
    int64_t first = 0;
    for (size_t s = 0; s < n_sec; ++s) {
      const int64_t nb = m->sec_nblk[s];
      if (nb) {
        LAMB_CUDA(ctx, cudaMemcpyAsync(out[s].col_i, si.col16 + first, sizeof(int16_t) * nb, cudaMemcpyDeviceToHost, ctx->stream));
        LAMB_CUDA(ctx, cudaMemcpyAsync(out[s].extents, si.ext + 2 * first, sizeof(int64_t) * 2 * nb, cudaMemcpyDeviceToHost, ctx->stream));
      }
      first += nb;
    }
  }
  LAMB_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  LAMB_CUDA(ctx, cudaStreamSynchronize(ctx->copy_stream));
  free_sector_index(ctx, &si);
  for (int a = 0; a < m->n_rsub; ++a)
    for (int b = 0; b < S; ++b) {
      auto& o = out[a * S + b];
      const size_t s = (size_t)a * S + b;
      o.subset_row = a + 1;
      o.subset_col = b + 1;
      o.n_rows = m->rsub_cnt[a];
      o.n_cols = m->csub_cnt[b];
      if (o.row_blk_sizes && o.n_rows) memcpy(o.row_blk_sizes, &m->h_row_bs[m->rsub_base[a]], o.n_rows);
      if (o.col_blk_sizes && o.n_cols) memcpy(o.col_blk_sizes, &m->h_col_bs[m->csub_base[b]], o.n_cols);
      // run lengths of sector (a,b): h_bcnt[rsub_base[a]*S + b*cnt_a + l]
      const int64_t cnt = m->rsub_cnt[a];
      const int64_t base = (int64_t)m->rsub_base[a] * S + b * cnt;
      o.row_p[0] = 0;
      for (int64_t l = 0; l < cnt; ++l) o.row_p[l + 1] = o.row_p[l] + (m->nnz ? si.h_bcnt[base + l] : 0);
      o.n_blks = m->sec_nblk[s];
      o.data_len = m->sec_dlen[s];
    }
  return LAMB_GPU_OK;
}

}  // extern "C"
