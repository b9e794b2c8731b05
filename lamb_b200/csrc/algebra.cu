// Block-sparse matrix algebra on device matrices: union-pattern axpby, copy,
// scale and shift, traces and Frobenius norms.  These are the building
// blocks of McWeeny purification; the reference has no counterpart (its
// lamb_matrix_operations, src/lamb_matrix_operations.F90, only loads and
// distributes matrices).
#include <cub/cub.cuh>

#include <algorithm>

#include "algebra.cuh"

namespace lamb {

bool same_structure(const DevMatrix* x, const DevMatrix* y) {
  return x->n_rsub == y->n_rsub && x->n_csub == y->n_csub && x->rsub_cnt == y->rsub_cnt &&
         x->csub_cnt == y->csub_cnt && x->h_row_bs == y->h_row_bs && x->h_col_bs == y->h_col_bs;
}

bool is_square(const DevMatrix* x) {
  return x->n_rsub == x->n_csub && x->rsub_cnt == x->csub_cnt && x->h_row_bs == x->h_col_bs;
}

__global__ void k_expand_rows(int32_t n_rows, const int64_t* __restrict__ row_p, int32_t* __restrict__ row_of) {
  for (int64_t r = global_warp(); r < n_rows; r += grid_warps())
    for (int64_t b = row_p[r] + (threadIdx.x & 31); b < row_p[r + 1]; b += 32) row_of[b] = (int32_t)r;
}

int32_t expand_rows(Ctx* ctx, const DevMatrix* m, int32_t** row_of) {
  LAMB_TRY(dalloc(ctx, row_of, std::max<int64_t>(m->nnz, 1)));
  if (m->nnz) {
    k_expand_rows<<<grid_for(32ll * m->n_rows, 256), 256, 0, ctx->stream>>>(m->n_rows, m->row_p, *row_of);
    LAMB_LAUNCHED(ctx);
  }
  return LAMB_GPU_OK;
}

int32_t sum_f64(Ctx* ctx, const double* in, int64_t n, double* host_out) {
  *host_out = 0.0;
  if (n <= 0) return LAMB_GPU_OK;
  double* d_out = nullptr;
  LAMB_TRY(dalloc(ctx, &d_out, 1));
  size_t bytes = 0;
  LAMB_CUDA(ctx, cub::DeviceReduce::Sum(nullptr, bytes, in, d_out, n, ctx->stream));
  void* tmp = nullptr;
  LAMB_TRY(dalloc(ctx, (char**)&tmp, (int64_t)bytes + 16));
  cudaError_t e = cub::DeviceReduce::Sum(tmp, bytes, in, d_out, n, ctx->stream);
  cudaFreeAsync(tmp, ctx->stream);
  LAMB_CUDA(ctx, e);
  LAMB_CUDA(ctx, cudaMemcpyAsync(host_out, d_out, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  LAMB_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  dfree(ctx, d_out);
  return LAMB_GPU_OK;
}

// ---- union pattern ----------------------------------------------------------------------
// Union of the sorted block rows of X and Y, one warp per row.  The union
// has |X| + |Y| - |X and Y| blocks.  The block at rank a of X's row sits at
// union position a + (blocks of Y's row with a smaller column) - (columns in
// both rows smaller than its own), the second term by binary search in Y's
// row, the third by a running count of X's blocks found in Y; Y's blocks
// likewise.  A column in both rows is written by the X side.
__global__ void k_union_count(int32_t n_rows, const int64_t* __restrict__ xrp, const int32_t* __restrict__ xc,
                              const int64_t* __restrict__ yrp, const int32_t* __restrict__ yc,
                              int64_t* __restrict__ cnt) {
  const int lane = threadIdx.x & 31;
  for (int64_t r = global_warp(); r < n_rows; r += grid_warps()) {
    const int64_t a0 = xrp[r], ae = xrp[r + 1], b0 = yrp[r], be = yrp[r + 1];
    int64_t both = 0;
    for (int64_t a = a0; a < ae; a += 32) {
      bool hit = false;
      if (a + lane < ae) {
        const int c = xc[a + lane];
        const int64_t bp = lower_col(yc, b0, be, c);
        hit = bp < be && yc[bp] == c;
      }
      both += __popc(__ballot_sync(0xffffffffu, hit));
    }
    if (lane == 0) cnt[r] = (ae - a0) + (be - b0) - both;
  }
}

__global__ void k_union_fill(int32_t n_rows, const int64_t* __restrict__ xrp, const int32_t* __restrict__ xc,
                             const int64_t* __restrict__ yrp, const int32_t* __restrict__ yc,
                             const int64_t* __restrict__ urp, int32_t* __restrict__ uc, int64_t* __restrict__ xi,
                             int64_t* __restrict__ yi) {
  const int lane = threadIdx.x & 31;
  for (int64_t r = global_warp(); r < n_rows; r += grid_warps()) {
    const int64_t a0 = xrp[r], ae = xrp[r + 1], b0 = yrp[r], be = yrp[r + 1], u0 = urp[r];
    const unsigned below = (1u << lane) - 1u;
    int64_t both = 0;  // columns in both rows before the current chunk of X
    for (int64_t a1 = a0; a1 < ae; a1 += 32) {
      const int64_t a = a1 + lane;
      int c = 0;
      int64_t bp = be;
      if (a < ae) {
        c = xc[a];
        bp = lower_col(yc, b0, be, c);
      }
      const bool hit = bp < be && yc[bp] == c;
      const unsigned m = __ballot_sync(0xffffffffu, hit);
      if (a < ae) {
        const int64_t u = u0 + (a - a0) + (bp - b0) - (both + __popc(m & below));
        uc[u] = c;
        xi[u] = a;
        yi[u] = hit ? bp : -1;
      }
      both += __popc(m);
    }
    both = 0;  // now: columns in both rows before the current chunk of Y
    for (int64_t b1 = b0; b1 < be; b1 += 32) {
      const int64_t b = b1 + lane;
      int c = 0;
      int64_t ap = ae;
      if (b < be) {
        c = yc[b];
        ap = lower_col(xc, a0, ae, c);
      }
      const bool hit = ap < ae && xc[ap] == c;
      const unsigned m = __ballot_sync(0xffffffffu, hit);
      if (b < be && !hit) {
        const int64_t u = u0 + (b - b0) + (ap - a0) - (both + __popc(m & below));
        uc[u] = c;
        xi[u] = -1;
        yi[u] = b;
      }
      both += __popc(m);
    }
  }
}

int32_t union_pattern(Ctx* ctx, const DevMatrix* X, const DevMatrix* Y, DevMatrix* U, int64_t** xi, int64_t** yi,
                      int32_t** row_of) {
  if (!same_structure(X, Y))
    return fail(ctx, LAMB_LEVEL_FAILURE, LAMB_TYPE_WRONG_ARGS, "matrices have different subset structures");
  copy_structure(U, X, true, X, true);
  LAMB_TRY(upload_block_sizes(ctx, U));
  const int n = U->n_rows;
  int64_t* cnt = nullptr;
  LAMB_TRY(dalloc(ctx, &cnt, std::max(n, 1)));
  LAMB_TRY(dalloc(ctx, &U->row_p, n + 1));
  if (n) {
    k_union_count<<<grid_for(32ll * n, 256), 256, 0, ctx->stream>>>(n, X->row_p, X->col, Y->row_p, Y->col, cnt);
    LAMB_LAUNCHED(ctx);
  }
  std::vector<int64_t> h(n), rp(n + 1, 0);
  if (n) {
    LAMB_CUDA(ctx, cudaMemcpyAsync(h.data(), cnt, sizeof(int64_t) * n, cudaMemcpyDeviceToHost, ctx->stream));
    LAMB_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  }
  for (int r = 0; r < n; ++r) rp[r + 1] = rp[r] + h[r];
  U->nnz = rp[n];
  LAMB_CUDA(ctx, cudaMemcpyAsync(U->row_p, rp.data(), sizeof(int64_t) * (n + 1), cudaMemcpyHostToDevice, ctx->stream));
  LAMB_TRY(dalloc(ctx, &U->col, std::max<int64_t>(U->nnz, 1)));
  LAMB_TRY(dalloc(ctx, xi, std::max<int64_t>(U->nnz, 1)));
  LAMB_TRY(dalloc(ctx, yi, std::max<int64_t>(U->nnz, 1)));
  if (U->nnz) {
    k_union_fill<<<grid_for(32ll * n, 256), 256, 0, ctx->stream>>>(n, X->row_p, X->col, Y->row_p, Y->col, U->row_p, U->col,
                                                              *xi, *yi);
    LAMB_LAUNCHED(ctx);
  }
  LAMB_TRY(dalloc(ctx, row_of, std::max<int64_t>(U->nnz, 1)));
  LAMB_TRY(layout_sector_major(ctx, U, *row_of));
  LAMB_TRY(dalloc(ctx, &U->data, std::max<int64_t>(U->data_len, 1)));
  LAMB_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  dfree(ctx, cnt);
  return LAMB_GPU_OK;
}

// out_u = alpha*x + beta*y blockwise; mode 1 writes (x-y)^2 block sums instead.
__global__ void k_combine(int64_t nnz, const int32_t* __restrict__ row_of, const int32_t* __restrict__ ucol,
                          const int8_t* __restrict__ row_bs, const int8_t* __restrict__ col_bs,
                          const int64_t* __restrict__ uoff, const int64_t* __restrict__ xi,
                          const int64_t* __restrict__ yi, const int64_t* __restrict__ xoff,
                          const int64_t* __restrict__ yoff, const double* __restrict__ xd,
                          const double* __restrict__ yd, double alpha, double beta, double* __restrict__ ud,
                          double* __restrict__ blk_sq) {
  const int lane = threadIdx.x & 31;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t u = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; u < nnz; u += nw) {
    const int n = row_bs[row_of[u]] * col_bs[ucol[u]];
    const int64_t a = xi[u], b = yi[u];
    const double* xp = a >= 0 ? xd + xoff[a] : nullptr;
    const double* yp = b >= 0 ? yd + yoff[b] : nullptr;
    double sq = 0.0;
    for (int e = lane; e < n; e += 32) {
      const double xv = xp ? xp[e] : 0.0, yv = yp ? yp[e] : 0.0;
      if (blk_sq) {
        const double d = xv - yv;
        sq = __fma_rn(d, d, sq);
      } else {
        ud[uoff[u] + e] = alpha * xv + beta * yv;
      }
    }
    if (blk_sq) {
      sq = warp_sum(sq);
      if (lane == 0) blk_sq[u] = sq;
    }
  }
}

// Moves the buffers of src into dst (dst's old buffers are freed).
void move_matrix(Ctx* ctx, DevMatrix* dst, DevMatrix* src) {
  std::vector<float> pos = dst->h_pos;
  float box[3] = {dst->box[0], dst->box[1], dst->box[2]};
  std::vector<int32_t> ord = dst->h_order;
  free_matrix_buffers(ctx, dst);
  *dst = std::move(*src);
  *src = DevMatrix{};
  touch(dst);
  if (!pos.empty() && dst->h_pos.empty() && (int64_t)pos.size() == 3ll * dst->n_rows) {
    dst->h_pos = pos;
    memcpy(dst->box, box, sizeof(box));
  }
  if (dst->h_order.empty() && (int)ord.size() == dst->n_rows) dst->h_order = ord;
}

int32_t axpby_impl(Ctx* ctx, double alpha, DevMatrix* X, double beta, DevMatrix* Y) {
  DevMatrix U;
  int64_t *xi = nullptr, *yi = nullptr;
  int32_t* row_of = nullptr;
  int32_t rc = union_pattern(ctx, X, Y, &U, &xi, &yi, &row_of);
  if (rc == LAMB_GPU_OK && U.nnz) {
    k_combine<<<grid_for(U.nnz * 32), kThreads, 0, ctx->stream>>>(U.nnz, row_of, U.col, U.row_bs, U.col_bs, U.off,
                                                                   xi, yi, X->off, Y->off, X->data, Y->data, alpha,
                                                                   beta, U.data, nullptr);
    ++ctx->launches;
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) rc = fail(ctx, LAMB_LEVEL_FAILURE, LAMB_TYPE_EXTERNAL_ERROR, cudaGetErrorString(e));
  }
  dfree(ctx, xi);
  dfree(ctx, yi);
  dfree(ctx, row_of);
  if (rc != LAMB_GPU_OK) {
    free_matrix_buffers(ctx, &U);
    return rc;
  }
  move_matrix(ctx, Y, &U);
  return LAMB_GPU_OK;
}

int32_t copy_impl(Ctx* ctx, const DevMatrix* X, DevMatrix* Y) {
  if (X == Y) return LAMB_GPU_OK;
  free_matrix_buffers(ctx, Y);
  DevMatrix tmp;
  copy_structure(&tmp, X, true, X, true);
  tmp.nnz = X->nnz;
  tmp.data_len = X->data_len;
  tmp.sec_base = X->sec_base;
  tmp.sec_dlen = X->sec_dlen;
  tmp.sec_nblk = X->sec_nblk;
  tmp.h_pos = X->h_pos;
  memcpy(tmp.box, X->box, sizeof(tmp.box));
  tmp.h_order = X->h_order;
  LAMB_TRY(upload_block_sizes(ctx, &tmp));
  LAMB_TRY(dalloc(ctx, &tmp.row_p, tmp.n_rows + 1));
  LAMB_TRY(dalloc(ctx, &tmp.col, std::max<int64_t>(tmp.nnz, 1)));
  LAMB_TRY(dalloc(ctx, &tmp.off, std::max<int64_t>(tmp.nnz, 1)));
  LAMB_TRY(dalloc(ctx, &tmp.data, std::max<int64_t>(tmp.data_len, 1)));
  LAMB_CUDA(ctx, cudaMemcpyAsync(tmp.row_p, X->row_p, sizeof(int64_t) * (tmp.n_rows + 1), cudaMemcpyDeviceToDevice, ctx->stream));
  if (tmp.nnz) {
    LAMB_CUDA(ctx, cudaMemcpyAsync(tmp.col, X->col, sizeof(int32_t) * tmp.nnz, cudaMemcpyDeviceToDevice, ctx->stream));
    LAMB_CUDA(ctx, cudaMemcpyAsync(tmp.off, X->off, sizeof(int64_t) * tmp.nnz, cudaMemcpyDeviceToDevice, ctx->stream));
  }
  if (tmp.data_len)
    LAMB_CUDA(ctx, cudaMemcpyAsync(tmp.data, X->data, sizeof(double) * tmp.data_len, cudaMemcpyDeviceToDevice, ctx->stream));
  *Y = std::move(tmp);
  return LAMB_GPU_OK;
}

__global__ void k_scale(int64_t n, double* __restrict__ d, double alpha) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    d[i] *= alpha;
}

__global__ void k_identity(int32_t n_rows, const int64_t* __restrict__ row_p, const int64_t* __restrict__ off,
                           const int8_t* __restrict__ bs, double* __restrict__ d) {
  for (int64_t r = global_warp(); r < n_rows; r += grid_warps()) {
    if (row_p[r + 1] == row_p[r]) continue;
    const int b = bs[r];
    double* p = d + off[row_p[r]];
    for (int e = threadIdx.x & 31; e < b * b; e += 32) p[e] = (e % b == e / b) ? 1.0 : 0.0;
  }
}

int32_t identity_like(Ctx* ctx, const DevMatrix* X, DevMatrix* I) {
  if (!is_square(X)) return fail(ctx, LAMB_LEVEL_FAILURE, LAMB_TYPE_WRONG_ARGS, "identity needs a square structure");
  copy_structure(I, X, true, X, true);
  LAMB_TRY(upload_block_sizes(ctx, I));
  const int n = I->n_rows;
  std::vector<int64_t> rp(n + 1, 0);
  std::vector<int32_t> cl;
  for (int r = 0; r < n; ++r) {
    if (I->h_row_bs[r] > 0) cl.push_back(r);
    rp[r + 1] = (int64_t)cl.size();
  }
  I->nnz = (int64_t)cl.size();
  LAMB_TRY(dalloc(ctx, &I->row_p, n + 1));
  LAMB_TRY(dalloc(ctx, &I->col, std::max<int64_t>(I->nnz, 1)));
  LAMB_CUDA(ctx, cudaMemcpyAsync(I->row_p, rp.data(), sizeof(int64_t) * (n + 1), cudaMemcpyHostToDevice, ctx->stream));
  if (I->nnz)
    LAMB_CUDA(ctx, cudaMemcpyAsync(I->col, cl.data(), sizeof(int32_t) * I->nnz, cudaMemcpyHostToDevice, ctx->stream));
  LAMB_TRY(layout_sector_major(ctx, I, nullptr));
  LAMB_TRY(dalloc(ctx, &I->data, std::max<int64_t>(I->data_len, 1)));
  if (n) {
    k_identity<<<grid_for(32ll * n, 256), 256, 0, ctx->stream>>>(n, I->row_p, I->off, I->row_bs, I->data);
    LAMB_LAUNCHED(ctx);
  }
  LAMB_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return LAMB_GPU_OK;
}

int32_t scale_shift_impl(Ctx* ctx, DevMatrix* X, double alpha, double shift) {
  if (shift == 0.0) {
    if (X->data_len) {
      k_scale<<<grid_for(X->data_len), kThreads, 0, ctx->stream>>>(X->data_len, X->data, alpha);
      LAMB_LAUNCHED(ctx);
    }
    X->norms_valid = false;
    return LAMB_GPU_OK;
  }
  DevMatrix I;
  int32_t rc = identity_like(ctx, X, &I);
  if (rc == LAMB_GPU_OK) rc = axpby_impl(ctx, shift, &I, alpha, X);
  free_matrix_buffers(ctx, &I);
  X->norms_valid = false;
  return rc;
}

// ---- traces and norms --------------------------------------------------------------------
__global__ void k_trace_rows(int32_t n_rows, const int64_t* __restrict__ row_p, const int32_t* __restrict__ col,
                             const int64_t* __restrict__ off, const int8_t* __restrict__ bs,
                             const double* __restrict__ d, double* __restrict__ part) {
  for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < n_rows; r += (int64_t)gridDim.x * blockDim.x) {
    int64_t lo = row_p[r], hi = row_p[r + 1] - 1;
    double s = 0.0;
    while (lo <= hi) {
      const int64_t mid = (lo + hi) >> 1;
      const int c = col[mid];
      if (c == r) {
        const int b = bs[r];
        for (int e = 0; e < b; ++e) s += d[off[mid] + (int64_t)e * b + e];
        break;
      }
      if (c < r) lo = mid + 1; else hi = mid - 1;
    }
    part[r] = s;
  }
}

int32_t trace_impl(Ctx* ctx, const DevMatrix* X, double* tr) {
  if (!is_square(X)) return fail(ctx, LAMB_LEVEL_FAILURE, LAMB_TYPE_WRONG_ARGS, "trace needs a square structure");
  double* part = nullptr;
  LAMB_TRY(dalloc(ctx, &part, std::max(X->n_rows, 1)));
  if (X->n_rows) {
    k_trace_rows<<<grid_for(X->n_rows, 128), 128, 0, ctx->stream>>>(X->n_rows, X->row_p, X->col, X->off, X->row_bs,
                                                                       X->data, part);
    LAMB_LAUNCHED(ctx);
  }
  int32_t rc = sum_f64(ctx, part, X->n_rows, tr);
  dfree(ctx, part);
  return rc;
}

// Tr(X.Y) = sum over blocks X_ij of <X_ij, Y_ji^T>.
__global__ void k_trace_prod(int64_t nnz, const int32_t* __restrict__ xrow, const int32_t* __restrict__ xcol,
                             const int64_t* __restrict__ xoff, const double* __restrict__ xd,
                             const int8_t* __restrict__ row_bs, const int8_t* __restrict__ col_bs,
                             const int64_t* __restrict__ yrp, const int32_t* __restrict__ ycol,
                             const int64_t* __restrict__ yoff, const double* __restrict__ yd,
                             double* __restrict__ part) {
  const int lane = threadIdx.x & 31;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t u = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; u < nnz; u += nw) {
    const int i = xrow[u], j = xcol[u];
    const int bi = row_bs[i], bj = col_bs[j];
    int64_t lo = yrp[j], hi = yrp[j + 1] - 1, yb = -1;
    while (lo <= hi) {
      const int64_t mid = (lo + hi) >> 1;
      const int c = ycol[mid];
      if (c == i) { yb = mid; break; }
      if (c < i) lo = mid + 1; else hi = mid - 1;
    }
    double s = 0.0;
    if (yb >= 0) {
      const double* xp = xd + xoff[u];
      const double* yp = yd + yoff[yb];
      for (int e = lane; e < bi * bj; e += 32) {
        const int p = e % bi, q = e / bi;      // X_ij(p,q); Y_ji(q,p) at q + p*bj
        s = __fma_rn(xp[e], yp[q + (int64_t)p * bj], s);
      }
    }
    s = warp_sum(s);
    if (lane == 0) part[u] = s;
  }
}

int32_t trace_product_impl(Ctx* ctx, const DevMatrix* X, const DevMatrix* Y, double* tr) {
  if (X->n_rsub != Y->n_csub || X->n_csub != Y->n_rsub || X->rsub_cnt != Y->csub_cnt || X->csub_cnt != Y->rsub_cnt)
    return fail(ctx, LAMB_LEVEL_FAILURE, LAMB_TYPE_WRONG_ARGS, "trace_product: X and Y^T structures differ");
  int32_t* xrow = nullptr;
  double* part = nullptr;
  LAMB_TRY(expand_rows(ctx, X, &xrow));
  LAMB_TRY(dalloc(ctx, &part, std::max<int64_t>(X->nnz, 1)));
  if (X->nnz) {
    k_trace_prod<<<grid_for(X->nnz * 32), kThreads, 0, ctx->stream>>>(X->nnz, xrow, X->col, X->off, X->data,
                                                                       X->row_bs, X->col_bs, Y->row_p, Y->col,
                                                                       Y->off, Y->data, part);
    LAMB_LAUNCHED(ctx);
  }
  int32_t rc = sum_f64(ctx, part, X->nnz, tr);
  dfree(ctx, xrow);
  dfree(ctx, part);
  return rc;
}

int32_t diff_frobenius_impl(Ctx* ctx, const DevMatrix* X, const DevMatrix* Y, double* out) {
  DevMatrix U;
  int64_t *xi = nullptr, *yi = nullptr;
  int32_t* row_of = nullptr;
  double* part = nullptr;
  int32_t rc = union_pattern(ctx, X, Y, &U, &xi, &yi, &row_of);
  if (rc == LAMB_GPU_OK) rc = dalloc(ctx, &part, std::max<int64_t>(U.nnz, 1));
  if (rc == LAMB_GPU_OK && U.nnz) {
    k_combine<<<grid_for(U.nnz * 32), kThreads, 0, ctx->stream>>>(U.nnz, row_of, U.col, U.row_bs, U.col_bs, U.off,
                                                                   xi, yi, X->off, Y ? Y->off : nullptr, X->data,
                                                                   Y->data, 1.0, -1.0, nullptr, part);
    ++ctx->launches;
  }
  double s = 0.0;
  if (rc == LAMB_GPU_OK) rc = sum_f64(ctx, part, U.nnz, &s);
  *out = std::sqrt(s);
  dfree(ctx, xi); dfree(ctx, yi); dfree(ctx, row_of); dfree(ctx, part);
  free_matrix_buffers(ctx, &U);
  return rc;
}

int32_t frobenius_impl(Ctx* ctx, const DevMatrix* X, double* out) {
  // |X|_F = |X - Z|_F with Z the empty matrix of the same structure
  DevMatrix Z;
  copy_structure(&Z, X, true, X, true);
  LAMB_TRY(upload_block_sizes(ctx, &Z));
  LAMB_TRY(dalloc(ctx, &Z.row_p, Z.n_rows + 1));
  LAMB_CUDA(ctx, cudaMemsetAsync(Z.row_p, 0, sizeof(int64_t) * (Z.n_rows + 1), ctx->stream));
  int32_t rc = diff_frobenius_impl(ctx, X, &Z, out);
  free_matrix_buffers(ctx, &Z);
  return rc;
}

}  // namespace lamb

using namespace lamb;

#define CTX_OR_FAIL(c)                                                    \
  auto* ctx = reinterpret_cast<Ctx*>(c);                                  \
  if (!ctx) return make_status(LAMB_LEVEL_FAILURE, LAMB_TYPE_WRONG_ARGS); \
  cudaSetDevice(ctx->device)

extern "C" {

int32_t lamb_gpu_matrix_axpby(lamb_gpu_ctx* c, double alpha, lamb_gpu_matrix x, double beta, lamb_gpu_matrix y) {
  CTX_OR_FAIL(c);
  DevMatrix *X = get_matrix(ctx, x), *Y = get_matrix(ctx, y);
  if (!X || !Y) return fail(ctx, LAMB_LEVEL_FAILURE, LAMB_TYPE_WRONG_ARGS, "axpby: invalid handle");
  if (X == Y) return scale_shift_impl(ctx, Y, alpha + beta, 0.0);
  int32_t rc = axpby_impl(ctx, alpha, X, beta, Y);
  if (rc == LAMB_GPU_OK) LAMB_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return rc;
}

int32_t lamb_gpu_matrix_copy(lamb_gpu_ctx* c, lamb_gpu_matrix x, lamb_gpu_matrix y) {
  CTX_OR_FAIL(c);
  DevMatrix *X = get_matrix(ctx, x), *Y = get_matrix(ctx, y);
  if (!X || !Y) return fail(ctx, LAMB_LEVEL_FAILURE, LAMB_TYPE_WRONG_ARGS, "copy: invalid handle");
  LAMB_TRY(copy_impl(ctx, X, Y));
  LAMB_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return LAMB_GPU_OK;
}

int32_t lamb_gpu_matrix_trace(lamb_gpu_ctx* c, lamb_gpu_matrix x, double* tr) {
  CTX_OR_FAIL(c);
  DevMatrix* X = get_matrix(ctx, x);
  if (!X || !tr) return fail(ctx, LAMB_LEVEL_FAILURE, LAMB_TYPE_WRONG_ARGS, "trace: invalid argument");
  return trace_impl(ctx, X, tr);
}

int32_t lamb_gpu_matrix_trace_product(lamb_gpu_ctx* c, lamb_gpu_matrix x, lamb_gpu_matrix y, double* tr) {
  CTX_OR_FAIL(c);
  DevMatrix *X = get_matrix(ctx, x), *Y = get_matrix(ctx, y);
  if (!X || !Y || !tr) return fail(ctx, LAMB_LEVEL_FAILURE, LAMB_TYPE_WRONG_ARGS, "trace_product: invalid argument");
  return trace_product_impl(ctx, X, Y, tr);
}

int32_t lamb_gpu_matrix_frobenius(lamb_gpu_ctx* c, lamb_gpu_matrix x, double* norm) {
  CTX_OR_FAIL(c);
  DevMatrix* X = get_matrix(ctx, x);
  if (!X || !norm) return fail(ctx, LAMB_LEVEL_FAILURE, LAMB_TYPE_WRONG_ARGS, "frobenius: invalid argument");
  return frobenius_impl(ctx, X, norm);
}

int32_t lamb_gpu_matrix_diff_frobenius(lamb_gpu_ctx* c, lamb_gpu_matrix x, lamb_gpu_matrix y, double* norm) {
  CTX_OR_FAIL(c);
  DevMatrix *X = get_matrix(ctx, x), *Y = get_matrix(ctx, y);
  if (!X || !Y || !norm) return fail(ctx, LAMB_LEVEL_FAILURE, LAMB_TYPE_WRONG_ARGS, "diff_frobenius: invalid argument");
  return diff_frobenius_impl(ctx, X, Y, norm);
}

int32_t lamb_gpu_matrix_scale_shift(lamb_gpu_ctx* c, lamb_gpu_matrix x, double alpha, double shift) {
  CTX_OR_FAIL(c);
  DevMatrix* X = get_matrix(ctx, x);
  if (!X) return fail(ctx, LAMB_LEVEL_FAILURE, LAMB_TYPE_WRONG_ARGS, "scale_shift: invalid handle");
  LAMB_TRY(scale_shift_impl(ctx, X, alpha, shift));
  LAMB_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return LAMB_GPU_OK;
}

}  // extern "C"
