// C = A.B over LAMB sectors on the GPU: symbolic phase, FP64 numeric phase,
// result filter, and the lamb_gpu_multiply / lamb_gpu_multiply_stacks entry
// points.
//
// Replaces lamb_multiply (src/lamb_multiplication.F90:116-204): its sector
// pairing "A(m,k) with B(k',n) when k == k', into C(m,n)" (:180-201) is
// realised by the sector-order block-CSR, in which A's column k and B's row k
// index the same atom, so one global product visits exactly the sector
// triples the reference pairs, with k subsets in ascending order.  The
// sector_multiply stub (:206-225) becomes the numeric kernels below.
#include <cub/cub.cuh>

#include <algorithm>
#include <cstdlib>
#include <numeric>

#include "multiply.cuh"

namespace lamb {

void free_symbolic(Ctx* ctx, Symbolic& s) {
  dfree(ctx, s.stack_p);
  if (s.use_scratch)
    s.ent = nullptr;
  else
    dfree(ctx, s.ent);
  dfree(ctx, s.ids);
  dfree(ctx, s.c_row);
}

int32_t check_compatible(Ctx* ctx, const DevMatrix* A, const DevMatrix* B) {
  if (A->n_csub != B->n_rsub || A->csub_cnt != B->rsub_cnt || A->h_col_bs != B->h_row_bs)
    return fail(ctx, LAMB_LEVEL_FAILURE, LAMB_TYPE_WRONG_ARGS,
                "A's column subsets and B's row subsets differ (A, B distributions do not match)");
  return LAMB_GPU_OK;
}

// ---- symbolic phase ----------------------------------------------------------------
// One CTA per C block row.  A bitmap over C's block columns marks the columns
// reached by surviving products A_ik.B_kj (|A_ik|*|B_kj| >= eps).
constexpr int kSymThreads = 256;

// FILT = false when no product can fall below eps: the norms are then not read.
template <bool FILT>
__device__ __forceinline__ bool keep_pair(double na, const double* __restrict__ b_nrm, int64_t bb, double eps) {
  return !FILT || !(na * b_nrm[bb] < eps);
}
// The fill always reads the norms (with eps = 0 when nothing is filtered:
// norms are >= 0 or NaN, so every pair stays); its norm-free variant measured
// 1.4 ms slower at 6,144 waters while the count kernel gains 0.8 ms.
__device__ __forceinline__ bool keep_norms(double na, double nb, double eps) { return !(na * nb < eps); }

template <bool FILT>
__global__ void __launch_bounds__(kSymThreads) k_sym_count(
    int32_t n_rows, const int64_t* __restrict__ a_row_p, const int32_t* __restrict__ a_col,
    const double* __restrict__ a_nrm, const int64_t* __restrict__ b_row_p, const int32_t* __restrict__ b_col,
    const double* __restrict__ b_nrm, const int8_t* __restrict__ row_bs, const int8_t* __restrict__ k_bs,
    const int8_t* __restrict__ col_bs, double eps, int32_t n_words, int64_t* __restrict__ c_cnt,
    int64_t* __restrict__ s_cnt, int64_t* __restrict__ p_cnt, double* __restrict__ row_flops,
    unsigned* __restrict__ max_a_len) {
  extern __shared__ uint32_t bm[];
  typedef cub::BlockReduce<int64_t, kSymThreads> RI;
  typedef cub::BlockReduce<double, kSymThreads> RD;
  __shared__ typename RI::TempStorage ti;
  __shared__ typename RD::TempStorage td;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nw = kSymThreads / 32;
  for (int64_t i = blockIdx.x; i < n_rows; i += gridDim.x) {
    for (int w = tid; w < n_words; w += kSymThreads) bm[w] = 0u;
    __syncthreads();
    int64_t kept = 0, pairs = 0;
    double fl = 0.0;
    const int bi = row_bs[i];
    for (int64_t ab = a_row_p[i] + warp; ab < a_row_p[i + 1]; ab += nw) {
      const int k = a_col[ab];
      const double na = FILT ? a_nrm[ab] : 0.0;
      const int bk = k_bs[k];
      const int64_t b1 = b_row_p[k + 1];
      for (int64_t bb = b_row_p[k] + lane; bb < b1; bb += 32) {
        ++pairs;
        if (!keep_pair<FILT>(na, b_nrm, bb, eps)) continue;
        const int j = b_col[bb];
        atomicOr(&bm[j >> 5], 1u << (j & 31));
        ++kept;
        fl += 2.0 * bi * bk * col_bs[j];
      }
    }
    __syncthreads();
    int64_t pc = 0;
    for (int w = tid; w < n_words; w += kSymThreads) pc += __popc(bm[w]);
    int64_t tot_pc = RI(ti).Sum(pc);
    __syncthreads();
    int64_t tot_kept = RI(ti).Sum(kept);
    __syncthreads();
    int64_t tot_pairs = RI(ti).Sum(pairs);
    __syncthreads();
    double tot_fl = RD(td).Sum(fl);
    if (tid == 0) {
      c_cnt[i] = tot_pc;
      s_cnt[i] = tot_kept;
      p_cnt[i] = tot_pairs;
      row_flops[i] = tot_fl;
      atomicMax(max_a_len, (unsigned)(a_row_p[i + 1] - a_row_p[i]));
    }
    __syncthreads();
  }
}

// Exclusive block scan of v[0..n) in place; returns the total.
__device__ int block_excl_scan_smem(int* v, int n) {
  typedef cub::BlockScan<int, kSymThreads> BS;
  __shared__ typename BS::TempStorage ts;
  __shared__ int total;
  const int tid = threadIdx.x;
  const int per = (n + kSymThreads - 1) / kSymThreads;
  const int lo = min(n, tid * per), hi = min(n, lo + per);
  int s = 0;
  for (int t = lo; t < hi; ++t) s += v[t];
  int ex, agg;
  BS(ts).ExclusiveSum(s, ex, agg);
  __syncthreads();
  for (int t = lo; t < hi; ++t) {
    const int x = v[t];
    v[t] = ex;
    ex += x;
  }
  if (tid == 0) total = agg;
  __syncthreads();
  return total;
}

__device__ __forceinline__ int bm_rank(const uint32_t* bm, const int* wpre, int j) {
  return wpre[j >> 5] + __popc(bm[j >> 5] & ((1u << (j & 31)) - 1u));
}

// C pattern only (no stacks), one CTA per C row: the bitmap of reached
// columns, then the row's columns in ascending order.  Used by the mixed
// tensor-core path, which needs no block-product stacks.
__global__ void __launch_bounds__(kSymThreads) k_sym_pattern(
    int32_t n_rows, const int64_t* __restrict__ a_row_p, const int32_t* __restrict__ a_col,
    const double* __restrict__ a_nrm, const int64_t* __restrict__ b_row_p, const int32_t* __restrict__ b_col,
    const double* __restrict__ b_nrm, double eps, int32_t n_words, const int64_t* __restrict__ c_row_p,
    int32_t* __restrict__ c_col) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  uint32_t* bm = reinterpret_cast<uint32_t*>(smem_raw);
  int* wpre = reinterpret_cast<int*>(bm + n_words);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nw = kSymThreads / 32;
  for (int64_t i = blockIdx.x; i < n_rows; i += gridDim.x) {
    for (int w = tid; w < n_words; w += kSymThreads) bm[w] = 0u;
    __syncthreads();
    for (int64_t ab = a_row_p[i] + warp; ab < a_row_p[i + 1]; ab += nw) {
      const int k = a_col[ab];
      const double x = a_nrm[ab];
      for (int64_t bb = b_row_p[k] + lane; bb < b_row_p[k + 1]; bb += 32)
        if (keep_norms(x, b_nrm[bb], eps)) {
          const int j = b_col[bb];
          atomicOr(&bm[j >> 5], 1u << (j & 31));
        }
    }
    __syncthreads();
    for (int w = tid; w < n_words; w += kSymThreads) wpre[w] = __popc(bm[w]);
    __syncthreads();
    block_excl_scan_smem(wpre, n_words);
    const int64_t c0 = c_row_p[i];
    for (int w = tid; w < n_words; w += kSymThreads) {
      uint32_t bits = bm[w];
      int p = wpre[w];
      while (bits) {
        const int b = __ffs(bits) - 1;
        bits &= bits - 1u;
        c_col[c0 + p++] = w * 32 + b;
      }
    }
    __syncthreads();
  }
}

// Stack fill, one CTA per C row.  The row's A blocks (column norm, operand
// word, B-row bounds) are staged in shared memory first, so the pair loops
// carry one dependent load (the B block) instead of three.  Entries are
// written one A block at a time (barrier between A blocks), so every C
// block's stack lists its products in ascending k and consecutive slots of a
// stack are written close together in time; thread t prefetches its B block
// (norm, column, data offset) of the next A block before the barrier.  The
// stack is written with evict-first stores: it streams through L2 once and
// would otherwise push out the B index the next rows read.
// Shared memory: bitmap and word ranks (n_words each), stack cursors
// (max_c + 1) and the staged A row (na_max x 32 bytes).
template <bool IDS>
__global__ void __launch_bounds__(kSymThreads) k_sym_fill(
    int32_t n_rows, const int64_t* __restrict__ a_row_p, const int32_t* __restrict__ a_col,
    const double* __restrict__ a_nrm, const int64_t* __restrict__ b_row_p, const int32_t* __restrict__ b_col,
    const double* __restrict__ b_nrm, double eps, int32_t n_words, int32_t na_max, int32_t nc_max,
    const int64_t* __restrict__ c_row_p, const int64_t* __restrict__ s_row_base, int32_t* __restrict__ c_col,
    int64_t* __restrict__ stack_p, const int64_t* __restrict__ a_offk, const int64_t* __restrict__ b_off,
    Ent* __restrict__ ent, int2* __restrict__ ids, const int32_t* __restrict__ rows, int write_cols) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double* s_anrm = reinterpret_cast<double*>(smem_raw);
  long long* s_aoff = reinterpret_cast<long long*>(s_anrm + na_max);
  int64_t* s_bbeg = reinterpret_cast<int64_t*>(s_aoff + na_max);
  int64_t* s_bend = s_bbeg + na_max;
  uint32_t* bm = reinterpret_cast<uint32_t*>(s_bend + na_max);
  int* wpre = reinterpret_cast<int*>(bm + n_words);
  int* cur = wpre + n_words;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nw = kSymThreads / 32;
  for (int64_t idx = blockIdx.x; idx < n_rows; idx += gridDim.x) {
    const int64_t i = rows ? rows[idx] : idx;  // C row; s_row_base is indexed by idx
    const int64_t a0 = a_row_p[i];
    const int na = (int)(a_row_p[i + 1] - a0);
    for (int t = tid; t < na; t += kSymThreads) {
      const int k = a_col[a0 + t];
      s_anrm[t] = a_nrm[a0 + t];
      s_aoff[t] = IDS ? 0 : a_offk[a0 + t];
      s_bbeg[t] = b_row_p[k];
      s_bend[t] = b_row_p[k + 1];
    }
    for (int w = tid; w < n_words; w += kSymThreads) bm[w] = 0u;
    __syncthreads();
    for (int a = warp; a < na; a += nw) {
      const double x = s_anrm[a];
      for (int64_t bb = s_bbeg[a] + lane; bb < s_bend[a]; bb += 32)
        if (keep_norms(x, b_nrm[bb], eps)) {
          const int j = b_col[bb];
          atomicOr(&bm[j >> 5], 1u << (j & 31));
        }
    }
    __syncthreads();
    for (int w = tid; w < n_words; w += kSymThreads) wpre[w] = __popc(bm[w]);
    __syncthreads();
    block_excl_scan_smem(wpre, n_words);
    const int64_t c0 = c_row_p[i];
    const int nc = (int)(c_row_p[i + 1] - c0);
    // C columns of the row, ascending (already written when the pattern was
    // built beforehand)
    if (write_cols)
      for (int w = tid; w < n_words; w += kSymThreads) {
        uint32_t bits = bm[w];
        int p = wpre[w];
        while (bits) {
          const int b = __ffs(bits) - 1;
          bits &= bits - 1u;
          c_col[c0 + p++] = w * 32 + b;
        }
      }
    for (int t = tid; t < nc; t += kSymThreads) cur[t] = 0;
    __syncthreads();
    for (int a = warp; a < na; a += nw) {
      const double x = s_anrm[a];
      for (int64_t bb = s_bbeg[a] + lane; bb < s_bend[a]; bb += 32)
        if (keep_norms(x, b_nrm[bb], eps)) atomicAdd(&cur[bm_rank(bm, wpre, b_col[bb])], 1);
    }
    __syncthreads();
    block_excl_scan_smem(cur, nc);
    const int64_t sb = s_row_base[idx];
    for (int t = tid; t < nc; t += kSymThreads) stack_p[c0 + t] = sb + cur[t];
    __syncthreads();
    // Entries in k order: one A block at a time; the B row's columns are
    // distinct, so each C position advances at most once per A block.
    // Thread t owns B entries t, t + 256, ... of every B row; its first one
    // of the next A block is loaded before the barrier.
    int64_t bb = na > 0 ? s_bbeg[0] + tid : 0;
    bool have = na > 0 && bb < s_bend[0];
    double nb = have ? b_nrm[bb] : 0.0;
    int jb = have ? b_col[bb] : 0;
    long long ob = (!IDS && have) ? b_off[bb] : 0;
    for (int a = 0; a < na; ++a) {
      const double x = s_anrm[a];
      const long long ak = s_aoff[a];
      const int64_t bend = s_bend[a];
      // prefetch of the next A block's first entry for this thread
      const int64_t nbb = a + 1 < na ? s_bbeg[a + 1] + tid : 0;
      const bool nhave = a + 1 < na && nbb < s_bend[a + 1];
      const double nnb = nhave ? b_nrm[nbb] : 0.0;
      const int njb = nhave ? b_col[nbb] : 0;
      const long long nob = (!IDS && nhave) ? b_off[nbb] : 0;
      while (have) {
        if (keep_norms(x, nb, eps)) {
          const int p = bm_rank(bm, wpre, jb);
          const int slot = cur[p];
          cur[p] = slot + 1;
          if (IDS)
            ids[sb + slot] = make_int2((int)(a0 + a), (int)bb);
          else
            __stcs(reinterpret_cast<longlong2*>(ent + sb + slot), make_longlong2(ak, ob));
        }
        bb += kSymThreads;
        have = bb < bend;
        if (have) { nb = b_nrm[bb]; jb = b_col[bb]; if (!IDS) ob = b_off[bb]; }
      }
      __syncthreads();
      bb = nbb; have = nhave; nb = nnb; jb = njb; ob = nob;
    }
  }
}

// Grid of a row-looping symbolic kernel: the CTAs that are resident at once
// on all SMs (at most one per row).
template <typename K>
static int32_t resident_grid(Ctx* ctx, K kern, size_t smem, int32_t n_rows, int* grid) {
  int sms = 148, per_sm = 1;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx->device);
  LAMB_CUDA(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kSymThreads, smem));
  *grid = std::max(1, std::min(n_rows, sms * std::max(per_sm, 1)));
  return LAMB_GPU_OK;
}

// Shared memory of k_sym_fill for the given sizes.
static size_t sym_fill_smem(int32_t n_words, int64_t na_max, int64_t nc_max) {
  return (size_t)(32 * na_max + 8 * (int64_t)n_words + 4 * (nc_max + 1));
}

int32_t symbolic_phase(Ctx* ctx, DevMatrix* A, DevMatrix* B, DevMatrix* C, double eps, bool filt, bool want_ids,
                       const int64_t* a_offk, Symbolic* out, const int64_t* b_meta) {
  out->c_nnz = out->n_ent = out->n_pairs = 0;
  out->flops = 0;
  LAMB_TRY(check_compatible(ctx, A, B));
  LAMB_TRY(ensure_norms(ctx, A));
  LAMB_TRY(ensure_norms(ctx, B));
  trace_mark(ctx, "operand norms");
  if (A->nnz >= (1ll << 31) || B->nnz >= (1ll << 31))
    return fail(ctx, LAMB_LEVEL_FAILURE, LAMB_TYPE_UNIMPLEMENTED, "more than 2^31 blocks in an operand");
  const bool pattern_now = out->pattern_only || out->chunked_fill;
  if (!want_ids && !a_offk && !pattern_now)
    return fail(ctx, LAMB_LEVEL_FAILURE, LAMB_TYPE_INTERNAL_ERROR, "symbolic: no A meta");
  // C takes A's row subsets and B's column subsets.  Its data buffer is kept
  // for the new pattern when large enough (freed on every early return).
  struct KeptData {
    Ctx* ctx;
    double* p;
    int64_t cap;
    ~KeptData() { dfree(ctx, p); }
  } kept{ctx, C->data, C->data_cap};
  C->data = nullptr;
  free_matrix_buffers(ctx, C);
  copy_structure(C, A, true, B, true);
  LAMB_TRY(inherit_row_locality(ctx, C, A));
  LAMB_TRY(upload_block_sizes(ctx, C));
  trace_mark(ctx, "C structure");
  const int32_t n_rows = C->n_rows;
  const int32_t n_words = (C->n_cols + 31) / 32;
  LAMB_TRY(dalloc(ctx, &C->row_p, n_rows + 1));
  int64_t *c_cnt = nullptr, *s_cnt = nullptr, *p_cnt = nullptr;
  double* rfl = nullptr;
  LAMB_TRY(dalloc(ctx, &c_cnt, std::max(n_rows, 1)));
  LAMB_TRY(dalloc(ctx, &s_cnt, std::max(n_rows, 1)));
  LAMB_TRY(dalloc(ctx, &p_cnt, std::max(n_rows, 1)));
  LAMB_TRY(dalloc(ctx, &rfl, std::max(n_rows, 1)));
  unsigned* d_max_na = nullptr;
  LAMB_TRY(dalloc(ctx, &d_max_na, 1));
  LAMB_CUDA(ctx, cudaMemsetAsync(d_max_na, 0, sizeof(unsigned), ctx->stream));
  // No product falls below eps when the smallest norms of A and B multiply to
  // at least eps (fl(x*y) is monotone in x and y): the count kernel then
  // skips the norm loads.  Any NaN norm keeps the test.
  bool count_filt = filt;
  if (filt && A->nnz && B->nnz) {
    double min_a = 0.0, min_b = 0.0;
    LAMB_TRY(min_f64(ctx, A->norms, A->nnz, &min_a));
    LAMB_TRY(min_f64(ctx, B->norms, B->nnz, &min_b));
    if (min_a * min_b >= eps) count_filt = false;
  }
  const double fill_eps = filt ? eps : 0.0;
  const size_t smem_count = sizeof(uint32_t) * (size_t)std::max(n_words, 1);
  if (smem_count > 200 * 1024)
    return fail(ctx, LAMB_LEVEL_FAILURE, LAMB_TYPE_UNIMPLEMENTED, "too many block columns for the symbolic bitmap");
  if (n_rows > 0) {
    auto count_kern = count_filt ? k_sym_count<true> : k_sym_count<false>;
    if (smem_count > 48 * 1024)
      LAMB_CUDA(ctx, cudaFuncSetAttribute(count_kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_count));
    int grid = 1;
    LAMB_TRY(resident_grid(ctx, count_kern, smem_count, n_rows, &grid));
    count_kern<<<grid, kSymThreads, smem_count, ctx->stream>>>(
        n_rows, A->row_p, A->col, A->norms, B->row_p, B->col, B->norms, C->row_bs, B->row_bs, C->col_bs, eps,
        n_words, c_cnt, s_cnt, p_cnt, rfl, d_max_na);
    LAMB_LAUNCHED(ctx);
  }
  unsigned max_na = 0;
  std::vector<int64_t> h_s(n_rows), h_p(n_rows);
  std::vector<double> h_f(n_rows);
  out->h_row_len.assign(n_rows, 0);
  if (n_rows) {
    LAMB_CUDA(ctx, cudaMemcpyAsync(out->h_row_len.data(), c_cnt, sizeof(int64_t) * n_rows, cudaMemcpyDeviceToHost, ctx->stream));
    LAMB_CUDA(ctx, cudaMemcpyAsync(h_s.data(), s_cnt, sizeof(int64_t) * n_rows, cudaMemcpyDeviceToHost, ctx->stream));
    LAMB_CUDA(ctx, cudaMemcpyAsync(h_p.data(), p_cnt, sizeof(int64_t) * n_rows, cudaMemcpyDeviceToHost, ctx->stream));
    LAMB_CUDA(ctx, cudaMemcpyAsync(h_f.data(), rfl, sizeof(double) * n_rows, cudaMemcpyDeviceToHost, ctx->stream));
    LAMB_CUDA(ctx, cudaMemcpyAsync(&max_na, d_max_na, sizeof(unsigned), cudaMemcpyDeviceToHost, ctx->stream));
    LAMB_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  }
  trace_mark(ctx, "symbolic count");
  std::vector<int64_t> h_crp(n_rows + 1, 0), h_srb(n_rows + 1, 0);
  int64_t max_c = 0, max_s = 0;
  for (int r = 0; r < n_rows; ++r) {
    h_crp[r + 1] = h_crp[r] + out->h_row_len[r];
    h_srb[r + 1] = h_srb[r] + h_s[r];
    out->n_pairs += h_p[r];
    out->flops += h_f[r];
    max_c = std::max(max_c, out->h_row_len[r]);
    max_s = std::max(max_s, h_s[r]);
  }
  out->c_nnz = h_crp[n_rows];
  out->n_ent = h_srb[n_rows];
  if (out->n_ent >= (1ll << 40) || max_s >= (1ll << 24))
    return fail(ctx, LAMB_LEVEL_FAILURE, LAMB_TYPE_UNIMPLEMENTED, "stack too large");
  C->nnz = out->c_nnz;
  int64_t* s_row_base = nullptr;
  LAMB_TRY(dalloc(ctx, &s_row_base, n_rows + 1));
  LAMB_CUDA(ctx, cudaMemcpyAsync(C->row_p, h_crp.data(), sizeof(int64_t) * (n_rows + 1), cudaMemcpyHostToDevice, ctx->stream));
  LAMB_CUDA(ctx, cudaMemcpyAsync(s_row_base, h_srb.data(), sizeof(int64_t) * (n_rows + 1), cudaMemcpyHostToDevice, ctx->stream));
  LAMB_TRY(dalloc(ctx, &C->col, std::max<int64_t>(C->nnz, 1)));
  LAMB_TRY(dalloc(ctx, &out->stack_p, C->nnz + 1));
  if (want_ids)
    LAMB_TRY(dalloc(ctx, &out->ids, std::max<int64_t>(out->n_ent, 1)));
  else if (pattern_now)
    out->ent = nullptr;
  else if (out->use_scratch)
    LAMB_TRY(scratch(ctx, kScrEnt, out->n_ent, &out->ent));
  else
    LAMB_TRY(dalloc(ctx, &out->ent, std::max<int64_t>(out->n_ent, 1)));
  LAMB_CUDA(ctx, cudaMemcpyAsync(out->stack_p + C->nnz, &h_srb[n_rows], sizeof(int64_t), cudaMemcpyHostToDevice, ctx->stream));
  trace_mark(ctx, "symbolic allocations");
  const size_t smem_fill = sym_fill_smem(std::max(n_words, 1), std::max<int64_t>(max_na, 1), max_c);
  if (out->chunked_fill) {
    out->h_row_ent = h_s;
    out->fill_n_words = std::max(n_words, 1);
    out->fill_na_max = (int32_t)std::max<int64_t>(max_na, 1);
    out->fill_nc_max = (int32_t)max_c;
    out->fill_eps = fill_eps;
    out->fill_smem = smem_fill;
    if (smem_fill > 220 * 1024)
      return fail(ctx, LAMB_LEVEL_FAILURE, LAMB_TYPE_UNIMPLEMENTED, "C block row too long for the symbolic fill");
  }
  if (pattern_now && n_rows > 0 && C->nnz > 0) {
    const size_t smem_pat = sizeof(uint32_t) * 2 * (size_t)std::max(n_words, 1);
    if (smem_pat > 48 * 1024)
      LAMB_CUDA(ctx, cudaFuncSetAttribute(k_sym_pattern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_pat));
    int pgrid = 1;
    LAMB_TRY(resident_grid(ctx, k_sym_pattern, smem_pat, n_rows, &pgrid));
    k_sym_pattern<<<pgrid, kSymThreads, smem_pat, ctx->stream>>>(n_rows, A->row_p, A->col, A->norms, B->row_p, B->col,
                                                                B->norms, fill_eps, n_words, C->row_p, C->col);
    LAMB_LAUNCHED(ctx);
  } else if (smem_fill > 220 * 1024) {
    return fail(ctx, LAMB_LEVEL_FAILURE, LAMB_TYPE_UNIMPLEMENTED, "C block row too long for the symbolic fill");
  }
  if (!pattern_now && n_rows > 0 && C->nnz > 0) {
    auto kern = want_ids ? k_sym_fill<true> : k_sym_fill<false>;
    if (smem_fill > 48 * 1024)
      LAMB_CUDA(ctx, cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_fill));
    // As many CTAs as fit at once (6 per SM at 40 registers): CTAs of a larger
    // grid start only when a resident one has finished all its rows (a grid
    // of 8 per SM took 1.8 ms longer at 6,144 waters).
    int fgrid = 1;
    LAMB_TRY(resident_grid(ctx, kern, smem_fill, n_rows, &fgrid));
    kern<<<fgrid, kSymThreads, smem_fill, ctx->stream>>>(
        n_rows, A->row_p, A->col, A->norms, B->row_p, B->col, B->norms, fill_eps, n_words, (int32_t)max_na,
        (int32_t)max_c, C->row_p, s_row_base, C->col, out->stack_p, a_offk, b_meta ? b_meta : B->off, out->ent,
        out->ids, nullptr, 1);
    LAMB_LAUNCHED(ctx);
  }
  trace_mark(ctx, "symbolic fill");
  LAMB_TRY(dalloc(ctx, &out->c_row, std::max<int64_t>(C->nnz, 1)));
  LAMB_TRY(layout_sector_major(ctx, C, out->c_row, true, &out->h_base));
  trace_mark(ctx, "sector layout");
  if (C->data_len >= kMask40) return fail(ctx, LAMB_LEVEL_FAILURE, LAMB_TYPE_UNIMPLEMENTED, "C data too large");
  const int64_t need = std::max<int64_t>(C->data_len, 1);
  if (kept.p && kept.cap >= need) {
    C->data = kept.p;
    C->data_cap = kept.cap;
    kept.p = nullptr;
  } else {
    dfree(ctx, kept.p);
    LAMB_TRY(dalloc(ctx, &C->data, need));
    C->data_cap = need;
  }
  dfree(ctx, c_cnt); dfree(ctx, s_cnt); dfree(ctx, p_cnt); dfree(ctx, rfl); dfree(ctx, s_row_base);
  dfree(ctx, d_max_na);
  trace_mark(ctx, "C data allocation");
  return LAMB_GPU_OK;
}

// ---- operand meta: data offset and inner block size in one word ------------------------
__global__ void k_pack_offk(int32_t n_rows, const int64_t* __restrict__ row_p, const int32_t* __restrict__ col,
                            const int64_t* __restrict__ off, const int8_t* __restrict__ row_bs,
                            const int8_t* __restrict__ col_bs, int k_is_col, int64_t* __restrict__ out) {
  for (int64_t r = global_warp(); r < n_rows; r += grid_warps())
    for (int64_t b = row_p[r] + (threadIdx.x & 31); b < row_p[r + 1]; b += 32)
      out[b] = off[b] | ((int64_t)(k_is_col ? col_bs[col[b]] : row_bs[r]) << 56);
}

int32_t pack_offk(Ctx* ctx, const DevMatrix* m, bool k_is_col, int64_t** offk) {
  LAMB_TRY(dalloc(ctx, offk, std::max<int64_t>(m->nnz, 1)));
  if (m->data_len > kOffMask) return fail(ctx, LAMB_LEVEL_FAILURE, LAMB_TYPE_UNIMPLEMENTED, "operand data too large");
  if (m->nnz) {
    k_pack_offk<<<grid_for(32ll * m->n_rows, 256), 256, 0, ctx->stream>>>(m->n_rows, m->row_p, m->col, m->off, m->row_bs,
                                                                     m->col_bs, k_is_col ? 1 : 0, *offk);
    LAMB_LAUNCHED(ctx);
  }
  return LAMB_GPU_OK;
}

// ---- work list in the row processing order --------------------------------------------
// row_end (optional, by position): end of every row's stack; given when the
// stacks of consecutive rows in CSR order need not be adjacent (row chunks).
__global__ void k_build_work(int32_t n_rows, const int32_t* __restrict__ order, const int64_t* __restrict__ cum,
                             const int64_t* __restrict__ row_p, const int32_t* __restrict__ col,
                             const int64_t* __restrict__ off, const int8_t* __restrict__ row_bs,
                             const int8_t* __restrict__ col_bs, const int64_t* __restrict__ stack_p,
                             Work* __restrict__ work, int32_t* __restrict__ work_c,
                             const int64_t* __restrict__ row_end) {
  const int lane = threadIdx.x & 31;
  for (int64_t w = global_warp(); w < n_rows; w += grid_warps()) {
    const int r = order[w];
    const long long bi = row_bs[r];
    const int64_t c0 = row_p[r], c1 = row_p[r + 1], v0 = cum[w] - c0;
    for (int64_t c = c0 + lane; c < c1; c += 32) {
      const long long bj = col_bs[col[c]];
      const long long n = ((row_end && c + 1 == c1) ? row_end[w] : stack_p[c + 1]) - stack_p[c];
      work[v0 + c] = Work{(long long)off[c] | (bi << 40) | (bj << 48), (long long)stack_p[c] | (n << 40)};
      work_c[v0 + c] = (int32_t)c;
    }
  }
}

__global__ void k_order_lens(int32_t n_rows, const int32_t* __restrict__ order, const int64_t* __restrict__ row_p,
                             int64_t* __restrict__ lens) {
  for (int64_t w = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; w < n_rows; w += (int64_t)gridDim.x * blockDim.x) {
    const int r = order[w];
    lens[w] = row_p[r + 1] - row_p[r];
  }
}

int32_t build_work(Ctx* ctx, const DevMatrix* C, const Symbolic& sym, const DevMatrix* order_src, Work** work,
                   int32_t** work_c, bool use_scratch) {
  const int n = C->n_rows;
  if (use_scratch) {
    LAMB_TRY(scratch(ctx, kScrWork, sym.c_nnz, work));
    LAMB_TRY(scratch(ctx, kScrWorkC, sym.c_nnz, work_c));
  } else {
    LAMB_TRY(dalloc(ctx, work, std::max<int64_t>(sym.c_nnz, 1)));
    LAMB_TRY(dalloc(ctx, work_c, std::max<int64_t>(sym.c_nnz, 1)));
  }
  if (sym.c_nnz == 0 || n == 0) return LAMB_GPU_OK;
  if ((int)order_src->h_order.size() != n || !order_src->order)
    return fail(ctx, LAMB_LEVEL_FAILURE, LAMB_TYPE_INTERNAL_ERROR, "work list: row order missing");
  // first work item of every row position: exclusive scan of the C row
  // lengths taken in the processing order (on the device, no host round trip)
  int64_t *d_len = nullptr, *d_cum = nullptr;
  LAMB_TRY(dalloc(ctx, &d_len, n));
  LAMB_TRY(dalloc(ctx, &d_cum, n));
  k_order_lens<<<grid_for(n, 128), 128, 0, ctx->stream>>>(n, order_src->order, C->row_p, d_len);
  LAMB_LAUNCHED(ctx);
  LAMB_TRY(exclusive_scan_i64(ctx, d_len, d_cum, n));
  k_build_work<<<grid_for(32ll * n, 256), 256, 0, ctx->stream>>>(n, order_src->order, d_cum, C->row_p, C->col, C->off,
                                                            C->row_bs, C->col_bs, sym.stack_p, *work, *work_c,
                                                            nullptr);
  LAMB_LAUNCHED(ctx);
  dfree(ctx, d_len);
  dfree(ctx, d_cum);
  return LAMB_GPU_OK;
}

// ---- result filter ----------------------------------------------------------------------
// Keeps C block c iff !(c_nrm[c] < eps).  Entirely on the device: kept counts
// per (row, column subset), new row pointers by a scan, the compacted index,
// and per-sector counts that reach the host asynchronously (settle() applies
// them).  The data stay where they are (extents may leave holes in a
// sector's data, as LAMB's data stores allow).
__global__ void k_keep_counts(int32_t n_rows, int32_t S, const int32_t* __restrict__ csub_base,
                              const int32_t* __restrict__ rsub_base, int32_t n_rsub,
                              const int64_t* __restrict__ row_p, const int32_t* __restrict__ col,
                              const double* __restrict__ c_nrm, double eps, int64_t* __restrict__ row_kept,
                              unsigned long long* __restrict__ sec_kept) {
  const int lane = threadIdx.x & 31;
  for (int64_t r = global_warp(); r < n_rows; r += grid_warps()) {
    const int m = row_subset(rsub_base, n_rsub, r);
    const int64_t b1 = row_p[r + 1];
    int64_t lo = row_p[r], tot = 0;
    for (int n = 0; n < S; ++n) {
      const int64_t hi = lower_col(col, lo, b1, csub_base[n + 1]);
      int64_t k = 0;
      for (int64_t b0 = lo; b0 < hi; b0 += 32) {
        const int64_t b = b0 + lane;
        k += __popc(__ballot_sync(0xffffffffu, b < hi && !(c_nrm[b] < eps)));
      }
      if (k && lane == 0) atomicAdd(&sec_kept[(int64_t)m * S + n], (unsigned long long)k);
      tot += k;
      lo = hi;
    }
    if (lane == 0) row_kept[r + 1] = tot;
  }
}

__global__ void k_compact(int32_t n_rows, const int64_t* __restrict__ row_p, const int32_t* __restrict__ col,
                          const int64_t* __restrict__ off, const double* __restrict__ c_nrm, double eps,
                          const int64_t* __restrict__ new_row_p, int32_t* __restrict__ ncol,
                          int64_t* __restrict__ noff) {
  const int lane = threadIdx.x & 31;
  const unsigned below = (1u << lane) - 1u;
  for (int64_t r = global_warp(); r < n_rows; r += grid_warps()) {
    int64_t q = new_row_p[r];
    const int64_t b1 = row_p[r + 1];
    for (int64_t b0 = row_p[r]; b0 < b1; b0 += 32) {
      const int64_t b = b0 + lane;
      const bool keep = b < b1 && !(c_nrm[b] < eps);
      const unsigned kb = __ballot_sync(0xffffffffu, keep);
      if (keep) {
        const int64_t p = q + __popc(kb & below);
        ncol[p] = col[b];
        noff[p] = off[b];
      }
      q += __popc(kb);
    }
  }
}

int32_t result_filter(Ctx* ctx, DevMatrix* C, const double* c_nrm, double eps) {
  const int S = C->n_csub;
  const size_t n_sec = (size_t)C->n_rsub * S;
  if (C->nnz == 0 || C->n_rows == 0 || n_sec == 0) return LAMB_GPU_OK;
  LAMB_TRY(settle(ctx));
  if (ctx->pend_cap < n_sec) {
    if (ctx->pend_h) cudaFreeHost(ctx->pend_h);
    ctx->pend_h = nullptr;
    ctx->pend_cap = 0;
    LAMB_CUDA(ctx, cudaMallocHost(&ctx->pend_h, sizeof(int64_t) * n_sec));
    ctx->pend_cap = n_sec;
  }
  if (!ctx->pend_ev) LAMB_CUDA(ctx, cudaEventCreateWithFlags(&ctx->pend_ev, cudaEventDisableTiming));
  int64_t *row_kept = nullptr, *nrp = nullptr, *noff = nullptr;
  unsigned long long* sec_kept = nullptr;
  int32_t *d_cb = nullptr, *d_rb = nullptr, *ncol = nullptr;
  LAMB_TRY(dalloc(ctx, &row_kept, (int64_t)C->n_rows + 1));
  LAMB_TRY(dalloc(ctx, &nrp, (int64_t)C->n_rows + 1));
  LAMB_TRY(dalloc(ctx, &sec_kept, (int64_t)n_sec));
  LAMB_TRY(dalloc(ctx, &d_cb, S + 1));
  LAMB_TRY(dalloc(ctx, &d_rb, C->n_rsub + 1));
  LAMB_TRY(dalloc(ctx, &ncol, C->nnz));
  LAMB_TRY(dalloc(ctx, &noff, C->nnz));
  // csub_base / rsub_base are members of C: they outlive the copies.
  LAMB_CUDA(ctx, cudaMemcpyAsync(d_cb, C->csub_base.data(), sizeof(int32_t) * (S + 1), cudaMemcpyHostToDevice, ctx->stream));
  LAMB_CUDA(ctx, cudaMemcpyAsync(d_rb, C->rsub_base.data(), sizeof(int32_t) * (C->n_rsub + 1), cudaMemcpyHostToDevice, ctx->stream));
  LAMB_CUDA(ctx, cudaMemsetAsync(row_kept, 0, sizeof(int64_t), ctx->stream));
  LAMB_CUDA(ctx, cudaMemsetAsync(sec_kept, 0, sizeof(unsigned long long) * n_sec, ctx->stream));
  k_keep_counts<<<grid_for(32ll * C->n_rows, 256), 256, 0, ctx->stream>>>(C->n_rows, S, d_cb, d_rb, C->n_rsub, C->row_p,
                                                                    C->col, c_nrm, eps, row_kept, sec_kept);
  LAMB_LAUNCHED(ctx);
  LAMB_TRY(inclusive_scan_i64(ctx, row_kept, nrp, (int64_t)C->n_rows + 1));
  k_compact<<<grid_for(32ll * C->n_rows, 256), 256, 0, ctx->stream>>>(C->n_rows, C->row_p, C->col, C->off, c_nrm, eps, nrp,
                                                                ncol, noff);
  LAMB_LAUNCHED(ctx);
  LAMB_CUDA(ctx, cudaMemcpyAsync(ctx->pend_h, sec_kept, sizeof(int64_t) * n_sec, cudaMemcpyDeviceToHost, ctx->stream));
  LAMB_CUDA(ctx, cudaEventRecord(ctx->pend_ev, ctx->stream));
  dfree(ctx, C->row_p); dfree(ctx, C->col); dfree(ctx, C->off);
  C->row_p = nrp; C->col = ncol; C->off = noff;
  touch(C);
  C->norms_valid = false;
  dfree(ctx, row_kept); dfree(ctx, sec_kept); dfree(ctx, d_cb); dfree(ctx, d_rb);
  ctx->pend_m = C;
  return LAMB_GPU_OK;
}

// ---- FP64 numeric phase in row chunks --------------------------------------------------
// Stack entries of one row chunk at most: 2^27 (2 GiB of 16-byte entries), or
// the largest single C row's entries when that is more (a row is not split).
constexpr int64_t kStackCapEntries = 1ll << 27;

// The rows, in processing order, are cut into chunks: first into kMinChunks
// of about equal C-block count (downloads copy a chunk as soon as it is
// done), then wherever a chunk would hold more than the stack cap.  Per chunk
// the stacks are filled into one reused buffer, the chunk's work items
// built, and k_stacked launched; an event after each marks its rows' C data
// complete.  Inside a sector, C's data follow the processing order
// (layout_sector_major by_order), so chunk p's data in sector s is one
// contiguous range.
static int32_t numeric_chunks(Ctx* ctx, DevMatrix* A, DevMatrix* B, DevMatrix* C, const Symbolic& sym,
                              const int64_t* a_offk, double* c_nrm) {
  const int mi = max_block(A->h_col_bs);
  const int n = C->n_rows, S = C->n_csub, R = C->n_rsub;
  const size_t n_sec = (size_t)R * S;
  C->n_chunks = 0;
  C->chunk_rng.clear();
  if (n == 0 || sym.c_nnz == 0) return LAMB_GPU_OK;
  const std::vector<int32_t>& ord = A->h_order;
  if ((int)ord.size() != n || !A->order || (int)sym.h_row_ent.size() != n)
    return fail(ctx, LAMB_LEVEL_FAILURE, LAMB_TYPE_INTERNAL_ERROR, "numeric: row order or row stacks missing");
  const bool layout_ok = (int64_t)C->h_order.size() == n && (int64_t)sym.h_base.size() == (int64_t)n * S;
  // The fill runs one CTA per C row: a chunk gets at least as many rows as
  // the fill keeps resident, so that it fills the GPU (few heavy rows, as in
  // the products of dense density matrices, would otherwise leave most SMs idle).
  auto fill = k_sym_fill<false>;
  if (sym.fill_smem > 48 * 1024)
    LAMB_CUDA(ctx, cudaFuncSetAttribute(fill, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sym.fill_smem));
  int fgrid_all = 1;
  LAMB_TRY(resident_grid(ctx, fill, sym.fill_smem, n, &fgrid_all));
  const int min_rows = std::max(1, fgrid_all);
  // ---- chunk boundaries (processing positions) ----
  const int P0 = (layout_ok && sym.c_nnz >= 4 * kMinChunks) ? std::max(1, std::min(kMinChunks, n / min_rows)) : 1;
  std::vector<int> q0(P0 + 1, n);
  q0[0] = 0;
  {
    int64_t acc = 0;
    int p = 1;
    for (int w = 0; w < n && p < P0; ++w) {
      acc += sym.h_row_len[ord[w]];
      while (p < P0 && acc * P0 >= (int64_t)p * sym.c_nnz) q0[p++] = w + 1;
    }
  }
  int64_t cap = kStackCapEntries;
  for (int w = 0; w < n; ++w) cap = std::max(cap, sym.h_row_ent[ord[w]]);
  std::vector<int> q;
  for (;;) {
    q.assign(1, 0);
    for (int p = 0; p < P0; ++p) {
      int64_t ent = 0;
      for (int w = q0[p]; w < q0[p + 1]; ++w) {
        const int64_t re = sym.h_row_ent[ord[w]];
        if (ent + re > cap && w - q.back() >= min_rows) {
          q.push_back(w);
          ent = 0;
        }
        ent += re;
      }
      if (q0[p + 1] > q.back()) q.push_back(q0[p + 1]);
    }
    if ((int)q.size() - 1 <= kMaxChunks) break;
    cap *= 2;  // more chunks than events: larger chunks
  }
  const int P = (int)q.size() - 1;
  // entries before every position inside its chunk, and every chunk's total
  std::vector<int64_t> rel(n), ends(n), ent_of(P, 0);
  for (int p = 0; p < P; ++p) {
    int64_t e = 0;
    for (int w = q[p]; w < q[p + 1]; ++w) {
      rel[w] = e;
      e += sym.h_row_ent[ord[w]];
      ends[w] = e;
    }
    ent_of[p] = e;
  }
  const int64_t max_ent = *std::max_element(ent_of.begin(), ent_of.end());
  // C blocks before every boundary (work items are in processing order)
  std::vector<int64_t> item(P + 1, 0);
  for (int p = 0; p < P; ++p) {
    int64_t acc = 0;
    for (int w = q[p]; w < q[p + 1]; ++w) acc += sym.h_row_len[ord[w]];
    item[p + 1] = item[p] + acc;
  }
  // ---- download ranges of every chunk in every sector ----
  if (layout_ok) {
    std::vector<int32_t> sub_of(n);
    for (int a = 0; a < R; ++a)
      for (int r = C->rsub_base[a]; r < C->rsub_base[a + 1]; ++r) sub_of[r] = a;
    std::vector<int64_t> before((size_t)(P + 1) * R, 0);  // rows of subset a at positions < q[p]
    {
      std::vector<int64_t> cnt(R, 0);
      int p = 0;
      for (int w = 0; w <= n; ++w) {
        while (p <= P && q[p] == w) {
          for (int a = 0; a < R; ++a) before[(size_t)p * R + a] = cnt[a];
          ++p;
        }
        if (w < n) ++cnt[sub_of[ord[w]]];
      }
    }
    C->chunk_rng.assign(2 * (size_t)P * n_sec, 0);
    for (int p = 0; p < P; ++p)
      for (int a = 0; a < R; ++a)
        for (int b = 0; b < S; ++b) {
          const size_t s2 = (size_t)a * S + b;
          const int64_t cnt_a = C->rsub_cnt[a];
          auto at = [&](int64_t rank) -> int64_t {  // data offset in the sector before local rank `rank`
            if (rank >= cnt_a) return C->sec_dlen[s2];
            return sym.h_base[(size_t)C->rsub_base[a] * S + (size_t)b * cnt_a + rank] - C->sec_base[s2];
          };
          C->chunk_rng[2 * ((size_t)p * n_sec + s2)] = at(before[(size_t)p * R + a]);
          C->chunk_rng[2 * ((size_t)p * n_sec + s2) + 1] = at(before[(size_t)(p + 1) * R + a]);
        }
  }
  // ---- buffers ----
  Ent* ent = nullptr;
  Work* work = nullptr;
  int32_t* work_c = nullptr;
  LAMB_TRY(scratch(ctx, kScrEnt, max_ent, &ent));
  LAMB_TRY(scratch(ctx, kScrWork, sym.c_nnz, &work));
  LAMB_TRY(scratch(ctx, kScrWorkC, sym.c_nnz, &work_c));
  int64_t *d_rel = nullptr, *d_end = nullptr, *d_len = nullptr, *d_cum = nullptr;
  struct Free {
    Ctx* ctx;
    int64_t** p[4];
    ~Free() { for (auto q : p) dfree(ctx, *q); }
  } fr{ctx, {&d_rel, &d_end, &d_len, &d_cum}};
  LAMB_TRY(dalloc(ctx, &d_rel, n));
  LAMB_TRY(dalloc(ctx, &d_end, n));
  LAMB_TRY(dalloc(ctx, &d_len, n));
  LAMB_TRY(dalloc(ctx, &d_cum, n));
  LAMB_CUDA(ctx, cudaMemcpyAsync(d_rel, rel.data(), sizeof(int64_t) * n, cudaMemcpyHostToDevice, ctx->stream));
  LAMB_CUDA(ctx, cudaMemcpyAsync(d_end, ends.data(), sizeof(int64_t) * n, cudaMemcpyHostToDevice, ctx->stream));
  // the chunk's work items: row lengths in processing order, their scan, the items
  k_order_lens<<<grid_for(n, 128), 128, 0, ctx->stream>>>(n, A->order, C->row_p, d_len);
  LAMB_LAUNCHED(ctx);
  ctx->kern_chunks = P;
  for (int p = 0; p < P; ++p) {
    const int nr = q[p + 1] - q[p];
    if (nr == 0) {
      LAMB_CUDA(ctx, cudaEventRecord(ctx->kern_ev[0][p], ctx->stream));
      LAMB_CUDA(ctx, cudaEventRecord(ctx->kern_ev[1][p], ctx->stream));
      continue;
    }
    fill<<<std::min(fgrid_all, nr), kSymThreads, sym.fill_smem, ctx->stream>>>(
        nr, A->row_p, A->col, A->norms, B->row_p, B->col, B->norms, sym.fill_eps, sym.fill_n_words, sym.fill_na_max,
        sym.fill_nc_max, C->row_p, d_rel + q[p], C->col, sym.stack_p, a_offk, B->off, ent, nullptr, A->order + q[p],
        0);
    LAMB_LAUNCHED(ctx);
    LAMB_TRY(exclusive_scan_i64(ctx, d_len + q[p], d_cum + q[p], nr));
    k_build_work<<<grid_for(32ll * nr, 256), 256, 0, ctx->stream>>>(nr, A->order + q[p], d_cum + q[p], C->row_p, C->col,
                                                                 C->off, C->row_bs, C->col_bs, sym.stack_p,
                                                                 work + item[p], work_c + item[p], d_end + q[p]);
    LAMB_LAUNCHED(ctx);
    LAMB_CUDA(ctx, cudaEventRecord(ctx->kern_ev[0][p], ctx->stream));
    LAMB_TRY(run_stacked(ctx, item[p + 1] - item[p], work + item[p], work_c + item[p], ent, A->data, B->data,
                         C->data, c_nrm, false, false, mi));
    LAMB_CUDA(ctx, cudaEventRecord(ctx->kern_ev[1][p], ctx->stream));
    LAMB_CUDA(ctx, cudaEventRecord(ctx->chunk_ev[p], ctx->stream));
  }
  if (layout_ok) {
    C->n_chunks = P;
    C->chunk_data = C->data;
    ctx->chunk_m = C;
  }
  return LAMB_GPU_OK;
}

// ---- driver -------------------------------------------------------------------------------
int32_t multiply_impl(Ctx* ctx, DevMatrix* A, DevMatrix* B, DevMatrix* C, double eps, uint32_t flags,
                      lamb_gpu_mult_stats* stats) {
  if (A == C || B == C)
    return fail(ctx, LAMB_LEVEL_FAILURE, LAMB_TYPE_WRONG_ARGS, "C must be distinct from A and B");
  if (flags & LAMB_GPU_ACCUMULATE)
    return fail(ctx, LAMB_LEVEL_FAILURE, LAMB_TYPE_UNIMPLEMENTED, "LAMB_GPU_ACCUMULATE: use lamb_gpu_matrix_axpby");
  const bool filt_p = eps > 0 && !(flags & LAMB_GPU_NO_PRODUCT_FILTER);
  const bool filt_r = eps > 0 && !(flags & LAMB_GPU_NO_RESULT_FILTER);
  const bool timed = !(flags & LAMB_GPU_ASYNC);
  lamb_gpu_mult_stats st{};
  const int64_t launches0 = ctx->launches;
  if (timed) LAMB_CUDA(ctx, cudaEventRecord(ctx->ev[0], ctx->stream));
  ctx->kern_chunks = 0;
  Symbolic sym;
  int64_t* a_offk = nullptr;
  double* c_nrm = nullptr;
  Work* work = nullptr;
  int32_t* work_c = nullptr;
  int slices = 0;
  double tensor_ops = 0.0;
  int64_t dropped = 0;
  MixedPlanes mp;
  const bool mixed = (flags & LAMB_GPU_MIXED) != 0;
  // LAMB_GPU_MIXED_MMA_SYNC=1 selects the mma.sync digit kernel for every shape.
  const char* force_sync = std::getenv("LAMB_GPU_MIXED_MMA_SYNC");
  bool tc_path = mixed && mixed_tc_eligible(A, B) && !(force_sync && force_sync[0] == '1');
  sym.use_scratch = true;
  LAMB_TRY(settle(ctx));
  auto body = [&]() -> int32_t {
    trace_mark(ctx, "multiply: start");
    LAMB_TRY(check_compatible(ctx, A, B));
    LAMB_TRY(ensure_row_order(ctx, A));
    trace_mark(ctx, "row order");
    if (mixed && tc_path) {
      // tensor-core path: exponents, C's pattern (no stacks), then panels,
      // tiles and the tile kernel inside numeric_mixed_tc
      slices = kMixedTcSlices;
      LAMB_TRY(build_slices(ctx, A, B, slices, &mp, true));
      sym.pattern_only = true;
      LAMB_TRY(symbolic_phase(ctx, A, B, C, eps, filt_p, false, nullptr, &sym));
      LAMB_TRY(dalloc(ctx, &c_nrm, std::max<int64_t>(sym.c_nnz, 1)));
      if (timed) LAMB_CUDA(ctx, cudaEventRecord(ctx->ev[4], ctx->stream));
      trace_mark(ctx, "symbolic (pattern)");
      bool ran = false;
      LAMB_TRY(numeric_mixed_tc(ctx, A, B, C, mp, c_nrm, &ran, timed ? ctx->ev[1] : nullptr, &tensor_ops));
      trace_mark(ctx, "numeric (tensor cores)");
      if (ran) {
        if (timed) LAMB_CUDA(ctx, cudaEventRecord(ctx->ev[2], ctx->stream));
        if (filt_r) LAMB_TRY(result_filter(ctx, C, c_nrm, eps));
        trace_mark(ctx, "result filter");
        if (timed) LAMB_CUDA(ctx, cudaEventRecord(ctx->ev[3], ctx->stream));
        return LAMB_GPU_OK;
      }
      // a tile beyond the kernel's limits: the mma.sync path below
      tc_path = false;
      free_slices(ctx, &mp);
      mp = MixedPlanes{};
      dfree(ctx, c_nrm);
      free_symbolic(ctx, sym);
      sym = Symbolic{};
      sym.use_scratch = true;
      if (timed) LAMB_CUDA(ctx, cudaEventRecord(ctx->ev[0], ctx->stream));
    }
    if (mixed) {
      slices = mixed_slices_from_env();
      LAMB_TRY(build_slices(ctx, A, B, slices, &mp));
      if (timed) LAMB_CUDA(ctx, cudaEventRecord(ctx->ev[4], ctx->stream));
      trace_mark(ctx, "digit slices");
      LAMB_TRY(pack_plane_meta(ctx, A, mp, &a_offk));
      LAMB_TRY(symbolic_phase(ctx, A, B, C, eps, filt_p, false, a_offk, &sym, mp.b_soff));
    } else {
      LAMB_TRY(pack_offk(ctx, A, true, &a_offk));
      sym.chunked_fill = true;
      LAMB_TRY(symbolic_phase(ctx, A, B, C, eps, filt_p, false, a_offk, &sym));
    }
    trace_mark(ctx, "symbolic");
    if (mixed) LAMB_TRY(build_work(ctx, C, sym, A, &work, &work_c, true));
    LAMB_TRY(dalloc(ctx, &c_nrm, std::max<int64_t>(sym.c_nnz, 1)));
    trace_mark(ctx, "work items");
    if (timed) LAMB_CUDA(ctx, cudaEventRecord(ctx->ev[1], ctx->stream));
    if (mixed)
      LAMB_TRY(numeric_mixed(ctx, A, B, C, sym, work, work_c, c_nrm, mp));
    else
      LAMB_TRY(numeric_chunks(ctx, A, B, C, sym, a_offk, c_nrm));
    trace_mark(ctx, "numeric");
    if (timed) LAMB_CUDA(ctx, cudaEventRecord(ctx->ev[2], ctx->stream));
    if (filt_r) LAMB_TRY(result_filter(ctx, C, c_nrm, eps));
    trace_mark(ctx, "result filter");
    if (timed) LAMB_CUDA(ctx, cudaEventRecord(ctx->ev[3], ctx->stream));
    return LAMB_GPU_OK;
  };
  int32_t rc = body();
  free_slices(ctx, &mp);
  dfree(ctx, a_offk);
  dfree(ctx, c_nrm);
  free_symbolic(ctx, sym);
  if (rc != LAMB_GPU_OK) return rc;
  C->norms_valid = false;
  // Without LAMB_GPU_ASYNC the filter's counts are applied now; with it the
  // next call that touches a matrix applies them.
  const int64_t c_before = sym.c_nnz;
  if (timed) {
    LAMB_TRY(settle(ctx));
    dropped = c_before - C->nnz;
  }
  st.n_products = sym.n_ent;
  st.n_products_skipped = sym.n_pairs - sym.n_ent;
  st.n_c_blocks = C->nnz;
  st.n_c_blocks_dropped = dropped;
  st.flops = sym.flops;
  st.mixed_slices = slices;
  st.tensor_ops = tc_path ? tensor_ops : 0.0;
  st.kernel_launches = (int32_t)(ctx->launches - launches0);
  if (timed) {
    LAMB_CUDA(ctx, cudaEventSynchronize(ctx->ev[3]));
    float t01 = 0, t12 = 0, t03 = 0, t23 = 0, t04 = 0;
    cudaEventElapsedTime(&t01, ctx->ev[0], ctx->ev[1]);
    cudaEventElapsedTime(&t12, ctx->ev[1], ctx->ev[2]);
    cudaEventElapsedTime(&t03, ctx->ev[0], ctx->ev[3]);
    cudaEventElapsedTime(&t23, ctx->ev[2], ctx->ev[3]);
    if (mixed && tc_path)
      cudaEventElapsedTime(&t04, ctx->ev[4], ctx->ev[1]);  // panels, tiles and inner lists
    else if (mixed)
      cudaEventElapsedTime(&t04, ctx->ev[0], ctx->ev[4]);  // digit planes
    st.ms_symbolic = t01;
    st.ms_numeric = t12;
    st.ms_total = t03;
    st.ms_filter = t23;
    st.ms_prepare = t04;
    st.ms_kernel = t12;  // the numeric phase is the product kernel, except in the FP64 row chunks:
    if (!mixed && ctx->kern_chunks > 0) {
      double s = 0.0;
      for (int p = 0; p < ctx->kern_chunks; ++p) {
        float e = 0.f;
        cudaEventElapsedTime(&e, ctx->kern_ev[0][p], ctx->kern_ev[1][p]);
        s += e;
      }
      st.ms_kernel = s;
    }
  }
  ctx->last_stats = st;
  if (stats) *stats = st;
  return LAMB_GPU_OK;
}

// ---- stacks in the caller's numbering ----------------------------------------------------
// Sector and sector-local block id of every block of a device matrix, from its CSR.
static void host_block_ids(const DevMatrix* m, const std::vector<int64_t>& row_p, const std::vector<int32_t>& col,
                           std::vector<int32_t>& sec, std::vector<int64_t>& lid) {
  const int S = m->n_csub;
  sec.assign(col.size(), 0);
  lid.assign(col.size(), 0);
  std::vector<int64_t> cnt((size_t)m->n_rsub * S, 0);
  for (int a = 0; a < m->n_rsub; ++a)
    for (int l = 0; l < m->rsub_cnt[a]; ++l) {
      const int r = m->rsub_base[a] + l;
      int n = 0;
      for (int64_t b = row_p[r]; b < row_p[r + 1]; ++b) {
        while (col[b] >= m->csub_base[n + 1]) ++n;
        const size_t s = (size_t)a * S + n;
        sec[b] = (int32_t)s;
        lid[b] = cnt[s]++;
      }
    }
}

static int32_t stacks_export(Ctx* ctx, DevMatrix* A, DevMatrix* B, DevMatrix* C, const Symbolic& sym,
                             int64_t* entries, int64_t* n_entries) {
  auto d2h_csr = [&](const DevMatrix* m, std::vector<int64_t>& rp, std::vector<int32_t>& cl) -> int32_t {
    rp.resize(m->n_rows + 1);
    cl.resize(m->nnz);
    LAMB_CUDA(ctx, cudaMemcpyAsync(rp.data(), m->row_p, sizeof(int64_t) * (m->n_rows + 1), cudaMemcpyDeviceToHost, ctx->stream));
    if (m->nnz)
      LAMB_CUDA(ctx, cudaMemcpyAsync(cl.data(), m->col, sizeof(int32_t) * m->nnz, cudaMemcpyDeviceToHost, ctx->stream));
    return LAMB_GPU_OK;
  };
  std::vector<int64_t> arp, brp, crp, sp(sym.c_nnz + 1);
  std::vector<int32_t> acl, bcl, ccl;
  std::vector<int2> st(sym.n_ent);
  LAMB_TRY(d2h_csr(A, arp, acl));
  LAMB_TRY(d2h_csr(B, brp, bcl));
  LAMB_TRY(d2h_csr(C, crp, ccl));
  LAMB_CUDA(ctx, cudaMemcpyAsync(sp.data(), sym.stack_p, sizeof(int64_t) * (sym.c_nnz + 1), cudaMemcpyDeviceToHost, ctx->stream));
  if (sym.n_ent)
    LAMB_CUDA(ctx, cudaMemcpyAsync(st.data(), sym.ids, sizeof(int2) * sym.n_ent, cudaMemcpyDeviceToHost, ctx->stream));
  LAMB_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  if (!entries) { *n_entries = sym.n_ent; return LAMB_GPU_OK; }
  if (*n_entries < sym.n_ent) return fail(ctx, LAMB_LEVEL_FAILURE, LAMB_TYPE_WRONG_ARGS, "stacks: capacity too small");
  std::vector<int32_t> asec, bsec, csec;
  std::vector<int64_t> alid, blid, clid;
  host_block_ids(A, arp, acl, asec, alid);
  host_block_ids(B, brp, bcl, bsec, blid);
  host_block_ids(C, crp, ccl, csec, clid);
  // C blocks of every sector in sector CSR order.
  const int S = C->n_csub;
  std::vector<std::vector<int64_t>> by_sec((size_t)C->n_rsub * S);
  for (int r = 0; r < C->n_rows; ++r)
    for (int64_t b = crp[r]; b < crp[r + 1]; ++b) by_sec[csec[b]].push_back(b);
  int64_t out = 0;
  struct E { int bi, bj, bk; int64_t seq; int64_t v[5]; };
  std::vector<E> v;
  for (size_t s = 0; s < by_sec.size(); ++s) {
    v.clear();
    int64_t seq = 0;
    for (int64_t cb : by_sec[s]) {
      int r = (int)(std::upper_bound(crp.begin(), crp.end(), cb) - crp.begin() - 1);
      const int bi = C->h_row_bs[r], bj = C->h_col_bs[ccl[cb]];
      for (int64_t e = sp[cb]; e < sp[cb + 1]; ++e) {
        const int ab = st[e].x, bb = st[e].y;
        const int bk = A->h_col_bs[acl[ab]];
        v.push_back(E{bi, bj, bk, seq++, {asec[ab], alid[ab], bsec[bb], blid[bb], clid[cb]}});
      }
    }
    std::stable_sort(v.begin(), v.end(), [](const E& x, const E& y) {
      if (x.bi != y.bi) return x.bi < y.bi;
      if (x.bj != y.bj) return x.bj < y.bj;
      return x.bk < y.bk;
    });
    for (const E& e : v) {
      for (int f = 0; f < 5; ++f) entries[5 * out + f] = e.v[f];
      ++out;
    }
  }
  *n_entries = out;
  return LAMB_GPU_OK;
}

}  // namespace lamb

using namespace lamb;

extern "C" {

int32_t lamb_gpu_multiply(lamb_gpu_ctx* c, lamb_gpu_matrix a, lamb_gpu_matrix b, lamb_gpu_matrix cm, double eps,
                          uint32_t flags, lamb_gpu_mult_stats* stats) {
  auto* ctx = reinterpret_cast<Ctx*>(c);
  if (!ctx) return make_status(LAMB_LEVEL_FAILURE, LAMB_TYPE_WRONG_ARGS);
  DevMatrix *A = get_matrix(ctx, a), *B = get_matrix(ctx, b), *C = get_matrix(ctx, cm);
  if (!A || !B || !C) return fail(ctx, LAMB_LEVEL_FAILURE, LAMB_TYPE_WRONG_ARGS, "multiply: invalid handle");
  if (eps != eps) return fail(ctx, LAMB_LEVEL_FAILURE, LAMB_TYPE_WRONG_ARGS, "multiply: eps is NaN");
  cudaSetDevice(ctx->device);
  return multiply_impl(ctx, A, B, C, eps, flags, stats);
}

int32_t lamb_gpu_multiply_stacks(lamb_gpu_ctx* c, lamb_gpu_matrix a, lamb_gpu_matrix b, lamb_gpu_matrix cm,
                                 double eps, uint32_t flags, int64_t* entries, int64_t* n_entries) {
  auto* ctx = reinterpret_cast<Ctx*>(c);
  if (!ctx || !n_entries) return make_status(LAMB_LEVEL_FAILURE, LAMB_TYPE_WRONG_ARGS);
  DevMatrix *A = get_matrix(ctx, a), *B = get_matrix(ctx, b), *C = get_matrix(ctx, cm);
  if (!A || !B || !C || A == C || B == C)
    return fail(ctx, LAMB_LEVEL_FAILURE, LAMB_TYPE_WRONG_ARGS, "stacks: invalid handle");
  cudaSetDevice(ctx->device);
  const bool filt_p = eps > 0 && !(flags & LAMB_GPU_NO_PRODUCT_FILTER);
  Symbolic sym;
  int32_t rc = symbolic_phase(ctx, A, B, C, eps, filt_p, true, nullptr, &sym);
  if (rc == LAMB_GPU_OK) rc = stacks_export(ctx, A, B, C, sym, entries, n_entries);
  free_symbolic(ctx, sym);
  return rc;
}

}  // extern "C"
