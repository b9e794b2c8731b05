// Adjoint of the pattern-fixed product C = A.B (no reference counterpart):
//   dA = (dC . B^T) restricted to A's pattern,
//   dB = (A^T . dC) restricted to B's pattern.
// Each output block is a stacked small GEMM whose stack is the intersection
// of two sorted block rows: for dA_ik, the j with dC_ij and B_kj present;
// for dB_kj, the i with A_ik and dC_ij present (rows of the transposed
// patterns of A and dC).  The stacks feed the same DMMA kernel as the
// forward product, with B_kj (dA) or A_ik (dB) read transposed.
#include <cub/cub.cuh>

#include <algorithm>

#include "algebra.cuh"
#include "multiply.cuh"

namespace lamb {

// Transposed block index of m: for every column c, the blocks (row r, id b)
// of that column with r ascending.
struct TIndex {
  int32_t n = 0;            // columns of m = rows of the transpose
  int64_t* row_p = nullptr;  // [n+1]
  int32_t* col = nullptr;    // original rows
  int32_t* blk = nullptr;    // original block ids
};

static void free_tindex(Ctx* ctx, TIndex& t) {
  dfree(ctx, t.row_p);
  dfree(ctx, t.col);
  dfree(ctx, t.blk);
}

__global__ void k_iota32(int64_t n, int32_t* __restrict__ v) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    v[i] = (int32_t)i;
}
__global__ void k_col_hist(int64_t n, const int32_t* __restrict__ col, int64_t* __restrict__ cnt) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    atomicAdd((unsigned long long*)&cnt[col[i]], 1ull);
}
__global__ void k_gather_rows(int64_t n, const int32_t* __restrict__ blk, const int32_t* __restrict__ row_of,
                              int32_t* __restrict__ out) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    out[i] = row_of[blk[i]];
}

static int32_t transpose_index(Ctx* ctx, const DevMatrix* m, TIndex* t) {
  t->n = m->n_cols;
  const int64_t nnz = m->nnz;
  LAMB_TRY(dalloc(ctx, &t->row_p, t->n + 1));
  LAMB_TRY(dalloc(ctx, &t->col, std::max<int64_t>(nnz, 1)));
  LAMB_TRY(dalloc(ctx, &t->blk, std::max<int64_t>(nnz, 1)));
  int64_t* cnt = nullptr;
  LAMB_TRY(dalloc(ctx, &cnt, t->n + 1));
  LAMB_CUDA(ctx, cudaMemsetAsync(cnt, 0, sizeof(int64_t) * (t->n + 1), ctx->stream));
  if (nnz) {
    int32_t *ids = nullptr, *keys_out = nullptr, *row_of = nullptr;
    LAMB_TRY(dalloc(ctx, &ids, nnz));
    LAMB_TRY(dalloc(ctx, &keys_out, nnz));
    LAMB_TRY(expand_rows(ctx, m, &row_of));
    k_iota32<<<grid_for(nnz), kThreads, 0, ctx->stream>>>(nnz, ids);
    LAMB_LAUNCHED(ctx);
    k_col_hist<<<grid_for(nnz), kThreads, 0, ctx->stream>>>(nnz, m->col, cnt);
    LAMB_LAUNCHED(ctx);
    // stable sort of block ids by column keeps rows ascending within a column
    size_t bytes = 0;
    LAMB_CUDA(ctx, cub::DeviceRadixSort::SortPairs(nullptr, bytes, m->col, keys_out, ids, t->blk, nnz, 0, 32,
                                                   ctx->stream));
    void* tmp = nullptr;
    LAMB_TRY(dalloc(ctx, (char**)&tmp, (int64_t)bytes + 16));
    cudaError_t e = cub::DeviceRadixSort::SortPairs(tmp, bytes, m->col, keys_out, ids, t->blk, nnz, 0, 32, ctx->stream);
    cudaFreeAsync(tmp, ctx->stream);
    LAMB_CUDA(ctx, e);
    k_gather_rows<<<grid_for(nnz), kThreads, 0, ctx->stream>>>(nnz, t->blk, row_of, t->col);
    LAMB_LAUNCHED(ctx);
    dfree(ctx, ids);
    dfree(ctx, keys_out);
    dfree(ctx, row_of);
  }
  LAMB_TRY(exclusive_scan_i64(ctx, cnt, t->row_p, t->n + 1));
  dfree(ctx, cnt);
  return LAMB_GPU_OK;
}

// For output block z = (r, c) of pattern Z: entries over the sorted
// intersection of L's row r and R's row c (column lists lcol/rcol; block ids
// lblk/rblk, or identity when null).  Entry = (L offset | inner << 56, R offset)
// with inner = ksz[column].  One warp per output block: lanes take 32 entries
// of L's row at a time and binary-search their columns in R's row; a ballot
// keeps the matches in ascending column order.
template <bool FILL>
__global__ void k_masked_sym(int32_t n_rows, int64_t n_z, const int64_t* __restrict__ zrp,
                             const int32_t* __restrict__ zcol, const int64_t* __restrict__ lrp,
                             const int32_t* __restrict__ lcol, const int32_t* __restrict__ lblk,
                             const int64_t* __restrict__ loff, const int64_t* __restrict__ rrp,
                             const int32_t* __restrict__ rcol, const int32_t* __restrict__ rblk,
                             const int64_t* __restrict__ roff, const int8_t* __restrict__ ksz,
                             int64_t* __restrict__ cnt, const int64_t* __restrict__ sp, Ent* __restrict__ ent) {
  const int lane = threadIdx.x & 31;
  const unsigned below = (1u << lane) - 1u;
  for (int64_t z = global_warp(); z < n_z; z += grid_warps()) {
    int64_t lo = 0, hi = n_rows;  // the row r with zrp[r] <= z < zrp[r + 1]
    while (hi - lo > 1) {
      const int64_t mid = (lo + hi) >> 1;
      if (zrp[mid] <= z) lo = mid; else hi = mid;
    }
    const int64_t r = lo;
    const int c = zcol[z];
    const int64_t ae = lrp[r + 1], b0 = rrp[c], be = rrp[c + 1];
    int64_t w = FILL ? sp[z] : 0, n = 0;
    for (int64_t a = lrp[r]; a < ae; a += 32) {
      const int64_t ai = a + lane;
      int ja = 0;
      int64_t bp = be;
      if (ai < ae) {
        ja = lcol[ai];
        bp = lower_col(rcol, b0, be, ja);
      }
      const bool hit = bp < be && rcol[bp] == ja;
      const unsigned m = __ballot_sync(0xffffffffu, hit);
      if (FILL && hit) {
        const int64_t la = lblk ? lblk[ai] : ai, rb = rblk ? rblk[bp] : bp;
        ent[w + __popc(m & below)] = Ent{(long long)loff[la] | ((long long)ksz[ja] << 56), (long long)roff[rb]};
      }
      w += __popc(m);
      n += __popc(m);
    }
    if (!FILL && lane == 0) cnt[z] = n;
  }
}

__global__ void k_masked_work(int32_t n_rows, const int64_t* __restrict__ zrp, const int32_t* __restrict__ zcol,
                              const int64_t* __restrict__ zoff, const int8_t* __restrict__ rbs,
                              const int8_t* __restrict__ cbs, const int64_t* __restrict__ sp,
                              Work* __restrict__ work, int32_t* __restrict__ work_c) {
  for (int64_t r = global_warp(); r < n_rows; r += grid_warps())
    for (int64_t z = zrp[r] + (threadIdx.x & 31); z < zrp[r + 1]; z += 32) {
      const long long M = rbs[r], N = cbs[zcol[z]], n = sp[z + 1] - sp[z];
      work[z] = Work{(long long)zoff[z] | (M << 40) | (N << 48), (long long)sp[z] | (n << 40)};
      work_c[z] = (int32_t)z;
    }
}

// out (pattern of Z, fresh data) := sum over intersections of op1 . op2.
static int32_t masked_product(Ctx* ctx, const DevMatrix* Z, DevMatrix* out, const int64_t* lrp, const int32_t* lcol,
                              const int32_t* lblk, const int64_t* loff, const double* ldata, const int64_t* rrp,
                              const int32_t* rcol, const int32_t* rblk, const int64_t* roff, const double* rdata,
                              const int8_t* ksz, int max_inner, bool t1, bool t2) {
  // out takes Z's structure and pattern with a fresh sector-major layout
  free_matrix_buffers(ctx, out);
  copy_structure(out, Z, true, Z, true);
  out->h_pos = Z->h_pos;
  memcpy(out->box, Z->box, sizeof(out->box));
  out->nnz = Z->nnz;
  LAMB_TRY(upload_block_sizes(ctx, out));
  LAMB_TRY(dalloc(ctx, &out->row_p, out->n_rows + 1));
  LAMB_TRY(dalloc(ctx, &out->col, std::max<int64_t>(out->nnz, 1)));
  LAMB_CUDA(ctx, cudaMemcpyAsync(out->row_p, Z->row_p, sizeof(int64_t) * (out->n_rows + 1), cudaMemcpyDeviceToDevice, ctx->stream));
  if (out->nnz)
    LAMB_CUDA(ctx, cudaMemcpyAsync(out->col, Z->col, sizeof(int32_t) * out->nnz, cudaMemcpyDeviceToDevice, ctx->stream));
  LAMB_TRY(layout_sector_major(ctx, out, nullptr));
  LAMB_TRY(dalloc(ctx, &out->data, std::max<int64_t>(out->data_len, 1)));
  if (out->nnz == 0) return LAMB_GPU_OK;
  int64_t *cnt = nullptr, *sp = nullptr;
  Ent* ent = nullptr;
  Work* work = nullptr;
  int32_t* work_c = nullptr;
  const int n = out->n_rows;
  LAMB_TRY(dalloc(ctx, &cnt, out->nnz + 1));
  LAMB_TRY(dalloc(ctx, &sp, out->nnz + 1));
  LAMB_CUDA(ctx, cudaMemsetAsync(cnt + out->nnz, 0, sizeof(int64_t), ctx->stream));
  k_masked_sym<false><<<grid_for(32ll * out->nnz, 256), 256, 0, ctx->stream>>>(
      n, out->nnz, out->row_p, out->col, lrp, lcol, lblk, loff, rrp, rcol, rblk, roff, ksz, cnt, nullptr, nullptr);
  LAMB_LAUNCHED(ctx);
  LAMB_TRY(exclusive_scan_i64(ctx, cnt, sp, out->nnz + 1));
  int64_t n_ent = 0, max_cnt = 0;
  LAMB_CUDA(ctx, cudaMemcpyAsync(&n_ent, sp + out->nnz, sizeof(int64_t), cudaMemcpyDeviceToHost, ctx->stream));
  LAMB_TRY(max_i64(ctx, cnt, out->nnz, &max_cnt));  // waits for the stream
  // The work items pack the C data offset and the first entry in 40 bits and
  // an entry count in 24 bits (as the forward multiply does).
  auto release = [&]() { dfree(ctx, cnt); dfree(ctx, sp); };
  if (n_ent >= (1ll << 40) || max_cnt >= (1ll << 24)) {
    release();
    return fail(ctx, LAMB_LEVEL_FAILURE, LAMB_TYPE_UNIMPLEMENTED, "adjoint: stack too large");
  }
  if (out->data_len >= kMask40) {
    release();
    return fail(ctx, LAMB_LEVEL_FAILURE, LAMB_TYPE_UNIMPLEMENTED, "adjoint: output data too large");
  }
  LAMB_TRY(dalloc(ctx, &ent, std::max<int64_t>(n_ent, 1)));
  LAMB_TRY(dalloc(ctx, &work, out->nnz));
  LAMB_TRY(dalloc(ctx, &work_c, out->nnz));
  k_masked_sym<true><<<grid_for(32ll * out->nnz, 256), 256, 0, ctx->stream>>>(
      n, out->nnz, out->row_p, out->col, lrp, lcol, lblk, loff, rrp, rcol, rblk, roff, ksz, nullptr, sp, ent);
  LAMB_LAUNCHED(ctx);
  k_masked_work<<<grid_for(32ll * n, 256), 256, 0, ctx->stream>>>(n, out->row_p, out->col, out->off, out->row_bs,
                                                             out->col_bs, sp, work, work_c);
  LAMB_LAUNCHED(ctx);
  int32_t rc = run_stacked(ctx, out->nnz, work, work_c, ent, ldata, rdata, out->data, nullptr, t1, t2, max_inner);
  dfree(ctx, cnt); dfree(ctx, sp); dfree(ctx, ent); dfree(ctx, work); dfree(ctx, work_c);
  return rc;
}

int32_t adjoint_impl(Ctx* ctx, DevMatrix* A, DevMatrix* B, DevMatrix* dC, DevMatrix* dA, DevMatrix* dB) {
  LAMB_TRY(check_compatible(ctx, A, B));
  if (dC->n_rsub != A->n_rsub || dC->rsub_cnt != A->rsub_cnt || dC->h_row_bs != A->h_row_bs ||
      dC->n_csub != B->n_csub || dC->csub_cnt != B->csub_cnt || dC->h_col_bs != B->h_col_bs)
    return fail(ctx, LAMB_LEVEL_FAILURE, LAMB_TYPE_WRONG_ARGS, "adjoint: dC structure does not match A.B");
  if (dA == A || dA == B || dA == dC || dB == A || dB == B || dB == dC || (dA && dA == dB))
    return fail(ctx, LAMB_LEVEL_FAILURE, LAMB_TYPE_WRONG_ARGS, "adjoint: outputs must be distinct matrices");
  if (dA) {
    // dA_ik = sum_j dC_ij . B_kj^T: rows of dC and rows of B, op2 transposed.
    LAMB_TRY(masked_product(ctx, A, dA, dC->row_p, dC->col, nullptr, dC->off, dC->data, B->row_p, B->col, nullptr,
                            B->off, B->data, dC->col_bs, max_block(dC->h_col_bs), false, true));
  }
  if (dB) {
    // dB_kj = sum_i A_ik^T . dC_ij: columns of A and of dC, op1 transposed.
    TIndex at, ct;
    int32_t rc = transpose_index(ctx, A, &at);
    if (rc == LAMB_GPU_OK) rc = transpose_index(ctx, dC, &ct);
    if (rc == LAMB_GPU_OK)
      rc = masked_product(ctx, B, dB, at.row_p, at.col, at.blk, A->off, A->data, ct.row_p, ct.col, ct.blk, dC->off,
                          dC->data, A->row_bs, max_block(A->h_row_bs), true, false);
    free_tindex(ctx, at);
    free_tindex(ctx, ct);
    LAMB_TRY(rc);
  }
  LAMB_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return LAMB_GPU_OK;
}

}  // namespace lamb

using namespace lamb;

extern "C" int32_t lamb_gpu_multiply_adjoint(lamb_gpu_ctx* c, lamb_gpu_matrix a, lamb_gpu_matrix b,
                                             lamb_gpu_matrix dc, lamb_gpu_matrix da, lamb_gpu_matrix db) {
  auto* ctx = reinterpret_cast<Ctx*>(c);
  if (!ctx) return make_status(LAMB_LEVEL_FAILURE, LAMB_TYPE_WRONG_ARGS);
  cudaSetDevice(ctx->device);
  DevMatrix *A = get_matrix(ctx, a), *B = get_matrix(ctx, b), *dC = get_matrix(ctx, dc);
  DevMatrix* dA = da ? get_matrix(ctx, da) : nullptr;
  DevMatrix* dB = db ? get_matrix(ctx, db) : nullptr;
  if (!A || !B || !dC || (da && !dA) || (db && !dB))
    return fail(ctx, LAMB_LEVEL_FAILURE, LAMB_TYPE_WRONG_ARGS, "adjoint: invalid handle");
  return adjoint_impl(ctx, A, B, dC, dA, dB);
}
