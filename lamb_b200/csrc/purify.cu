// McWeeny purification P <- 3P^2 - 2P^3 on device matrices (no reference
// counterpart; the reference stops at the multiply).  The early steps may
// run their products in the mixed (int8 split-slice) mode; the last
// `fp64_tail` steps, the trace and the idempotency check run in FP64.
#include <cub/cub.cuh>

#include <algorithm>
#include <cmath>

#include "algebra.cuh"
#include "multiply.cuh"

namespace lamb {

// Gershgorin discs of every element row: lo = H_pp - sum_{q != p} |H_pq|,
// hi = H_pp + sum_{q != p} |H_pq|.  One warp per block row, one lane per
// element row.
__global__ void k_gershgorin(int32_t n_rows, const int64_t* __restrict__ row_p, const int32_t* __restrict__ col,
                             const int64_t* __restrict__ off, const int8_t* __restrict__ bs,
                             const double* __restrict__ d, double* __restrict__ lo, double* __restrict__ hi) {
  const int lane = threadIdx.x & 31;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t r = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; r < n_rows; r += nw) {
    const int bi = bs[r];
    for (int p = lane; p < bi; p += 32) {
      double center = 0.0, rad = 0.0;
      for (int64_t b = row_p[r]; b < row_p[r + 1]; ++b) {
        const int j = col[b], bj = bs[j];
        const double* x = d + off[b];
        for (int q = 0; q < bj; ++q) {
          const double v = x[(int64_t)q * bi + p];
          if (j == r && q == p) center = v;
          else rad += fabs(v);
        }
      }
      lo[r * 32 + p] = center - rad;
      hi[r * 32 + p] = center + rad;
    }
  }
}

int32_t spectral_bounds(Ctx* ctx, const DevMatrix* H, double* emin, double* emax) {
  const int n = H->n_rows;
  for (int8_t b : H->h_row_bs)
    if (b > 32) return fail(ctx, LAMB_LEVEL_FAILURE, LAMB_TYPE_UNIMPLEMENTED, "spectral bounds: block above 32");
  double *lo = nullptr, *hi = nullptr;
  LAMB_TRY(dalloc(ctx, &lo, (int64_t)n * 32 + 1));
  LAMB_TRY(dalloc(ctx, &hi, (int64_t)n * 32 + 1));
  if (n) {
    k_gershgorin<<<grid_for((int64_t)n * 32), kThreads, 0, ctx->stream>>>(n, H->row_p, H->col, H->off, H->row_bs,
                                                                           H->data, lo, hi);
    LAMB_LAUNCHED(ctx);
  }
  std::vector<double> hl((size_t)n * 32), hh((size_t)n * 32);
  if (n) {
    LAMB_CUDA(ctx, cudaMemcpyAsync(hl.data(), lo, sizeof(double) * n * 32, cudaMemcpyDeviceToHost, ctx->stream));
    LAMB_CUDA(ctx, cudaMemcpyAsync(hh.data(), hi, sizeof(double) * n * 32, cudaMemcpyDeviceToHost, ctx->stream));
    LAMB_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  }
  double a = INFINITY, b = -INFINITY;
  for (int r = 0; r < n; ++r)
    for (int p = 0; p < H->h_row_bs[r]; ++p) {
      a = std::min(a, hl[(size_t)r * 32 + p]);
      b = std::max(b, hh[(size_t)r * 32 + p]);
    }
  *emin = a;
  *emax = b;
  dfree(ctx, lo);
  dfree(ctx, hi);
  return LAMB_GPU_OK;
}

int32_t purify_impl(Ctx* ctx, DevMatrix* H, double mu, int steps, int tail, double eps, DevMatrix* P,
                    lamb_gpu_purify_report* rep) {
  if (!is_square(H)) return fail(ctx, LAMB_LEVEL_FAILURE, LAMB_TYPE_WRONG_ARGS, "purify: H must be square");
  if (steps < 0 || tail < 0) return fail(ctx, LAMB_LEVEL_FAILURE, LAMB_TYPE_WRONG_ARGS, "purify: negative steps");
  LAMB_CUDA(ctx, cudaEventRecord(ctx->ev[5], ctx->stream));
  double emin = 0, emax = 0;
  LAMB_TRY(spectral_bounds(ctx, H, &emin, &emax));
  if (!(emax > mu && emin < mu))
    return fail(ctx, LAMB_LEVEL_FAILURE, LAMB_TYPE_PRECONDITION_FAILED, "purify: mu outside the spectral bounds");
  const double lambda = std::min(1.0 / (emax - mu), 1.0 / (mu - emin));
  // P0 = lambda/2 (mu I - H) + I/2
  LAMB_TRY(copy_impl(ctx, H, P));
  LAMB_TRY(scale_shift_impl(ctx, P, -0.5 * lambda, 0.5 * lambda * mu + 0.5));
  DevMatrix P2, P3;
  copy_structure(&P2, P, true, P, true);
  copy_structure(&P3, P, true, P, true);
  int mixed_steps = 0;
  int32_t rc = LAMB_GPU_OK;
  for (int s = 0; s < steps && rc == LAMB_GPU_OK; ++s) {
    const bool mixed = s < steps - tail;
    const uint32_t fl = mixed ? LAMB_GPU_MIXED : LAMB_GPU_FP64;
    mixed_steps += mixed;
    rc = multiply_impl(ctx, P, P, &P2, eps, fl, nullptr);
    if (rc == LAMB_GPU_OK) rc = multiply_impl(ctx, &P2, P, &P3, eps, fl, nullptr);
    if (rc == LAMB_GPU_OK) rc = axpby_impl(ctx, -2.0, &P3, 3.0, &P2);  // P2 := 3 P2 - 2 P3
    if (rc == LAMB_GPU_OK) {
      move_matrix(ctx, P, &P2);
      copy_structure(&P2, P, true, P, true);
    }
  }
  double tr = 0, idem = 0, np = 0;
  if (rc == LAMB_GPU_OK) rc = trace_impl(ctx, P, &tr);
  if (rc == LAMB_GPU_OK) rc = multiply_impl(ctx, P, P, &P2, eps, LAMB_GPU_FP64, nullptr);
  if (rc == LAMB_GPU_OK) rc = diff_frobenius_impl(ctx, &P2, P, &idem);
  if (rc == LAMB_GPU_OK) rc = frobenius_impl(ctx, P, &np);
  free_matrix_buffers(ctx, &P2);
  free_matrix_buffers(ctx, &P3);
  LAMB_TRY(rc);
  LAMB_CUDA(ctx, cudaEventRecord(ctx->ev[6], ctx->stream));
  LAMB_CUDA(ctx, cudaEventSynchronize(ctx->ev[6]));
  float ms = 0;
  cudaEventElapsedTime(&ms, ctx->ev[5], ctx->ev[6]);
  if (rep) {
    rep->steps_done = steps;
    rep->steps_mixed = mixed_steps;
    rep->trace = tr;
    rep->idempotency = np > 0 ? idem / np : idem;
    rep->ms_total = ms;
  }
  return LAMB_GPU_OK;
}

}  // namespace lamb

using namespace lamb;

extern "C" int32_t lamb_gpu_purify_mcweeny(lamb_gpu_ctx* c, lamb_gpu_matrix h, double mu, int32_t steps,
                                           int32_t fp64_tail, double eps, lamb_gpu_matrix p,
                                           lamb_gpu_purify_report* rep) {
  auto* ctx = reinterpret_cast<Ctx*>(c);
  if (!ctx) return make_status(LAMB_LEVEL_FAILURE, LAMB_TYPE_WRONG_ARGS);
  cudaSetDevice(ctx->device);
  DevMatrix *H = get_matrix(ctx, h), *P = get_matrix(ctx, p);
  if (!H || !P || H == P) return fail(ctx, LAMB_LEVEL_FAILURE, LAMB_TYPE_WRONG_ARGS, "purify: invalid handle");
  return purify_impl(ctx, H, mu, steps, fp64_tail, eps, P, rep);
}
