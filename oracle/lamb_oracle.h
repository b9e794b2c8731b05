/*
 * lamb_oracle.h -- CPU restatement of LAMB's sector-based block-sparse
 * multiply.  TEST INFRASTRUCTURE ONLY: tests, the smoke check and the
 * benchmark's CPU-baseline leg use it as the checker; the product never
 * links or calls it.
 *
 * PARITY UNPINNED: the reference's sector_multiply is an empty stub
 * (src/lamb_multiplication.F90:206-225), it ships no golden vectors or
 * fixtures for this path (small.dbcsr / small.coor / test.f1 are absent), and
 * it cannot be compiled here (Fortran 2003 + MPI + Python 2).  This oracle
 * therefore restates the mathematical definition on the reference's own
 * storage conventions and loop structure, and is cross-checked in the tests
 * against an independent dense product (numpy) on the same inputs.
 *
 * What it follows (paths within uborstnik/LAMB):
 *   - sector pairing: for every A sector (m,k) and B sector (k',n) with
 *     k == k', the C sector (m,n) receives A(m,k).B(k,n)
 *     (src/lamb_multiplication.F90:180-201); k sectors are visited in
 *     ascending subset order because sectors are listed in (1,1),(1,2),...
 *     order (src/lamb_plexus_operations.F90:454-488);
 *   - block CSR: row_p exclusive offsets, col_i 1-based and sorted in a row,
 *     extents 1-based inclusive, column-major block data
 *     (src/lamb_index_types.F90:86-105, src/lamb_index_methods.F90:81-107,248-274,
 *     src/lamb_io_operations.F90:666-682);
 *   - cumulative data append (the intent of lamb_data_X_add_data,
 *     src/lamb_data_X_methods.F90:176-204; its data_len line :197 is a bug).
 * Build-defined rules (no reference counterpart):
 *   - block norm |X|_F = sqrt(s), s accumulated with fma(x,x,s) over the block
 *     in storage (column-major) order;
 *   - product filter: A_ik.B_kj is skipped when |A_ik|*|B_kj| < eps;
 *   - C pattern: (i,j) is present iff at least one product survives;
 *   - result filter: C_ij is dropped when |C_ij|_F < eps;
 *   - C sector layout: blocks in CSR order, data contiguous in that order;
 *   - summation order for C_ij: k ascending over (k subset, local k), each
 *     block product accumulated with fma over the inner index.
 */
#ifndef LAMB_ORACLE_H
#define LAMB_ORACLE_H
#include <stdint.h>
#include "../include/lamb_gpu.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct lamb_oracle_result lamb_oracle_result;

/* flags: LAMB_GPU_NO_PRODUCT_FILTER / LAMB_GPU_NO_RESULT_FILTER from lamb_gpu.h;
 * ORACLE_LONG_DOUBLE accumulates in long double (error reference). */
#define ORACLE_LONG_DOUBLE 0x100u
/* ORACLE_NO_STACKS: keep no stack entries (full-size runs; saves 48 bytes per product). */
#define ORACLE_NO_STACKS 0x200u
/* n_threads <= 0: use all OpenMP threads. row_stride > 1 computes only every
 * row_stride-th row of each C sector (a bounded sample for timing). */
int32_t lamb_oracle_multiply(const lamb_c_sector* a, int32_t na, const lamb_c_sector* b, int32_t nb,
                             double eps, uint32_t flags, int32_t n_threads, int32_t row_stride,
                             lamb_oracle_result** out);
int32_t lamb_oracle_n_sectors(const lamb_oracle_result* r);
int32_t lamb_oracle_sector(const lamb_oracle_result* r, int32_t s, lamb_c_sector* out);
/* products executed, products skipped, flops (2*b_i*b_k*b_j summed), C blocks dropped */
int32_t lamb_oracle_stats(const lamb_oracle_result* r, int64_t* n_products, int64_t* n_skipped, double* flops,
                          int64_t* n_dropped);
/* Stack entries in the canonical order of lamb_gpu_multiply_stacks (count
 * query with entries == NULL).  Only valid when the result was computed
 * without row sampling. */
int32_t lamb_oracle_stacks(const lamb_oracle_result* r, int64_t* entries, int64_t* n_entries);
int32_t lamb_oracle_free(lamb_oracle_result* r);
/* Whole-result check of a device C against a result computed with
 * LAMB_GPU_NO_RESULT_FILTER: pattern mismatches under the filter rule at eps,
 * sum of squared differences and of squared reference values over the kept
 * blocks, and the closest relative distance of any block norm to eps. */
int32_t lamb_oracle_compare(const lamb_oracle_result* r, const lamb_c_sector* got, int32_t n_got, double eps,
                            int32_t n_threads, int64_t* n_mismatch, double* num, double* den, double* min_gap);
/* Block norm exactly as the GPU computes it. */
double lamb_oracle_block_norm(const double* x, int64_t n);

#ifdef __cplusplus
}
#endif
#endif
