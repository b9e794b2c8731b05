// Internal interfaces of the block-sparse algebra (algebra.cu).
#pragma once
#include <cmath>

#include "common.cuh"

namespace lamb {

bool same_structure(const DevMatrix* x, const DevMatrix* y);
bool is_square(const DevMatrix* x);
int32_t expand_rows(Ctx* ctx, const DevMatrix* m, int32_t** row_of);
int32_t sum_f64(Ctx* ctx, const double* in, int64_t n, double* host_out);
// U := union pattern of X and Y (same structure); xi/yi map every U block to
// its X / Y block or -1; row_of gets each U block's row.
int32_t union_pattern(Ctx* ctx, const DevMatrix* X, const DevMatrix* Y, DevMatrix* U, int64_t** xi, int64_t** yi,
                      int32_t** row_of);
void move_matrix(Ctx* ctx, DevMatrix* dst, DevMatrix* src);
int32_t axpby_impl(Ctx* ctx, double alpha, DevMatrix* X, double beta, DevMatrix* Y);
int32_t copy_impl(Ctx* ctx, const DevMatrix* X, DevMatrix* Y);
int32_t identity_like(Ctx* ctx, const DevMatrix* X, DevMatrix* I);
int32_t scale_shift_impl(Ctx* ctx, DevMatrix* X, double alpha, double shift);
int32_t trace_impl(Ctx* ctx, const DevMatrix* X, double* tr);
int32_t trace_product_impl(Ctx* ctx, const DevMatrix* X, const DevMatrix* Y, double* tr);
int32_t frobenius_impl(Ctx* ctx, const DevMatrix* X, double* out);
int32_t diff_frobenius_impl(Ctx* ctx, const DevMatrix* X, const DevMatrix* Y, double* out);

}  // namespace lamb
