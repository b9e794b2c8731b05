/*
 * lamb_gpu.h -- C ABI of the B200 sector-based block-sparse multiply.
 *
 * This header is the drop-in boundary between a single-rank LAMB run and the
 * GPU implementation of C = A . B over LAMB sector storage.  A Fortran caller
 * binds it with ISO_C_BINDING (the interface module is
 * lamb_b200/fortran/lamb_gpu_binding.F90); Python binds it with ctypes
 * (lamb_b200/abi.py).
 *
 * Reference interfaces replaced (paths within uborstnik/LAMB):
 *   - lamb_multiply(matrix_a, matrix_b, matrix_c, error)
 *       src/lamb_multiplication.F90:116-204.  Its sector-pair loop (:180-201,
 *       pair A(m,k) with B(k,n), C sector from lamb_plexus_get_sector_i) and
 *       the sector_multiply stub (:206-225) are replaced by ONE call,
 *       lamb_gpu_multiply(), over all sector triples.
 *   - service_schedule / lamb_market_* / lamb_mp_window_* exchange
 *       src/lamb_multiplication.F90:227-320, src/lamb_market_X_methods.F90:94-415:
 *       at one rank every sector is local, so the exchange is a host no-op and
 *       has no entry point here.
 *   - Sector storage: lamb_sector_X_type (src/lamb_sector_X_types.F90:79-87),
 *       lamb_index_type / lamb_blk_info_type (src/lamb_index_types.F90:86-105),
 *       lamb_data_X_type (src/lamb_data_X_types.F90:77-83).  A sector crosses
 *       the ABI as lamb_c_sector below; lamb_blk_info_type is not BIND(C), so
 *       the caller repacks extents into one contiguous int64 array.
 *
 * Conventions (identical to the reference's sector storage):
 *   row_p[n_rows+1]  int64, exclusive offsets, row_p[0] == 0, blocks of local
 *                    row r are row_p[r] .. row_p[r+1]-1 (0-based block ids);
 *                    src/lamb_index_methods.F90:248-274.
 *   col_i[n_blks]    int16, 1-based local column, strictly increasing within
 *                    a row (lamb_index_get_blk_n binary search,
 *                    src/lamb_index_methods.F90:81-107, requires it).
 *   extents[2*n_blks] int64 pairs (first,last), 1-based inclusive positions in
 *                    data; last-first+1 == row_blk_size*col_blk_size.
 *   data[data_len]   float64, each block column-major (Fortran order).
 *   Block sizes are int8 (blksz_k, src/lamb_kinds.F90:175); zero is allowed.
 *
 * Status codes: every function returns int32.  0 is success.  A failure is
 *   encoded as level*100000 + (type + 50000) where level is a LAMB error level
 *   (src/lamb_error.F90:120-134: note 1 .. fatal 5) and type a LAMB error type
 *   (src/lamb_error.F90:141-159, e.g. lamb_wrong_args = 100,
 *   lamb_internal_error = -1, lamb_unimplemented = -1000,
 *   lamb_external_error = -2000).  lamb_gpu_status_level/type decode it and
 *   lamb_gpu_last_error() returns the message.  No exception, abort or exit
 *   crosses this boundary.
 *
 * Threading: one context owns one CUDA stream and must be driven by one host
 * thread at a time.  Calls are synchronous on return unless LAMB_GPU_ASYNC is
 * given.
 */
#ifndef LAMB_GPU_H
#define LAMB_GPU_H

#include <stdint.h>

#if defined(__GNUC__)
#define LAMB_API __attribute__((visibility("default")))
#else
#define LAMB_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status encoding -------------------------------------------------- */
#define LAMB_GPU_OK 0
#define LAMB_LEVEL_NOTE 1
#define LAMB_LEVEL_WARNING 2
#define LAMB_LEVEL_FAILURE 3
#define LAMB_LEVEL_MEMORY 4
#define LAMB_LEVEL_FATAL 5
#define LAMB_TYPE_CALLER_ERROR 1
#define LAMB_TYPE_WRONG_ARGS 100
#define LAMB_TYPE_PRECONDITION_FAILED 200
#define LAMB_TYPE_INTERNAL_ERROR (-1)
#define LAMB_TYPE_OVERFLOW_ERROR (-2)
#define LAMB_TYPE_UNIMPLEMENTED (-1000)
#define LAMB_TYPE_EXTERNAL_ERROR (-2000)

/* ---- multiply flags ------------------------------------------------------ */
#define LAMB_GPU_FP64 0u              /* plain FP64 block products            */
#define LAMB_GPU_MIXED 1u             /* int8 split-slice products, FP64 recombination */
#define LAMB_GPU_NO_PRODUCT_FILTER 2u /* keep products with |A_ik||B_kj| < eps */
#define LAMB_GPU_NO_RESULT_FILTER 4u  /* keep C blocks with |C_ij| < eps      */
#define LAMB_GPU_ASYNC 8u             /* return once the work is queued (see lamb_gpu_multiply) */
#define LAMB_GPU_ACCUMULATE 16u       /* reserved: C := C + A.B; lamb_gpu_multiply refuses it with
                                         lamb_unimplemented (accumulate with lamb_gpu_matrix_axpby) */

/* One sector of a LAMB matrix in the reference's storage (see above). */
typedef struct lamb_c_sector {
  int32_t subset_row;           /* subset position of the rows (1-based) */
  int32_t subset_col;           /* subset position of the columns        */
  int32_t n_rows;               /* atoms in the row subset               */
  int32_t n_cols;               /* atoms in the column subset            */
  const int8_t* row_blk_sizes;  /* [n_rows]                              */
  const int8_t* col_blk_sizes;  /* [n_cols]                              */
  const int64_t* row_p;         /* [n_rows+1]                            */
  const int16_t* col_i;         /* [n_blks]                              */
  const int64_t* extents;       /* [2*n_blks]                            */
  const double* data;           /* [data_len]                            */
  int64_t n_blks;
  int64_t data_len;
} lamb_c_sector;

/* Writable sector for downloads; the caller allocates every array with the
 * sizes returned by lamb_gpu_matrix_query (two-phase size->fill protocol,
 * because the Fortran side owns its allocations:
 * lamb_data_X_ensure_length / lamb_index_ensure_size). */
typedef struct lamb_c_sector_out {
  int32_t subset_row, subset_col, n_rows, n_cols;
  int8_t* row_blk_sizes;
  int8_t* col_blk_sizes;
  int64_t* row_p;
  int16_t* col_i;
  int64_t* extents;
  double* data;
  int64_t n_blks;   /* in: capacity of col_i/extents; out: blocks written */
  int64_t data_len; /* in: capacity of data; out: doubles written          */
} lamb_c_sector_out;

/* Sizes of one sector of a device matrix. */
typedef struct lamb_c_sector_sizes {
  int32_t subset_row, subset_col, n_rows, n_cols;
  int64_t n_blks, data_len;
} lamb_c_sector_sizes;

/* Statistics of the last multiply on a context. */
typedef struct lamb_gpu_mult_stats {
  int64_t n_products;        /* block products executed (after the filter)   */
  int64_t n_products_skipped;/* block products removed by the product filter */
  int64_t n_c_blocks;        /* C blocks kept                                 */
  int64_t n_c_blocks_dropped;/* C blocks removed by the result filter         */
  double flops;              /* sum over executed products of 2*b_i*b_k*b_j   */
  double ms_symbolic;        /* device time of the symbolic phase             */
  double ms_numeric;         /* device time of the numeric phase              */
  double ms_total;           /* device time of the whole multiply             */
  int32_t mixed_slices;      /* int8 slices per operand (0 for FP64)          */
  int32_t kernel_launches;   /* this library's kernels launched by the call   */
  double ms_prepare;         /* part of ms_symbolic spent preparing operands
                                (mixed: digit planes / panels; FP64: 0)       */
  double ms_filter;          /* device time of the result filter              */
  double tensor_ops;         /* mixed, tensor-core path: int8 multiply-add ops
                                the tile kernel executed (2 per MAC, padding
                                of the cluster tiles included); else 0       */
  double ms_kernel;          /* device time of the product kernel's launches
                                alone: FP64, the k_stacked launches of all row
                                chunks (without the chunks' stack fills);
                                mixed, the numeric phase                      */
} lamb_gpu_mult_stats;

typedef struct lamb_gpu_ctx lamb_gpu_ctx;
typedef int64_t lamb_gpu_matrix; /* handle, > 0 when valid */

/* ---- context ------------------------------------------------------------- */
/* Replaces nothing in the reference directly: it owns the CUDA stream and the
 * device buffers that back lamb_data_X/lamb_index storage on the GPU
 * (ownership mirrors lamb_data_X_type%mine, src/lamb_data_X_types.F90:80). */
LAMB_API int32_t lamb_gpu_ctx_create(int32_t device, lamb_gpu_ctx** ctx);
LAMB_API int32_t lamb_gpu_ctx_destroy(lamb_gpu_ctx* ctx);
/* Copies the last error message (NUL-terminated, truncated to len). */
LAMB_API int32_t lamb_gpu_last_error(const lamb_gpu_ctx* ctx, char* msg, int32_t len);
LAMB_API int32_t lamb_gpu_status_level(int32_t status);
LAMB_API int32_t lamb_gpu_status_type(int32_t status);
/* Runs on the context's stream (cudaStream_t passed as void*). */
LAMB_API int32_t lamb_gpu_ctx_get_stream(const lamb_gpu_ctx* ctx, void** stream);
LAMB_API int32_t lamb_gpu_ctx_synchronize(lamb_gpu_ctx* ctx);

/* ---- matrices -------------------------------------------------------------- */
/* Uploads the local sectors of a matrix (lamb_matrix_X_type%sectors(:),
 * src/lamb_matrix_X_types.F90:78-86) to device block-CSR storage.  Sectors
 * may come in any order; each (subset_row, subset_col) at most once; a
 * missing sector is empty.  Host arrays are not retained after return. */
LAMB_API int32_t lamb_gpu_matrix_upload(lamb_gpu_ctx* ctx, const lamb_c_sector* sectors, int32_t n_sectors,
                               lamb_gpu_matrix* handle);
/* Creates an empty matrix with the row/column subsets of `like` (what
 * lamb_matrix_copy + clearing gives the reference's C argument). */
LAMB_API int32_t lamb_gpu_matrix_create_like(lamb_gpu_ctx* ctx, lamb_gpu_matrix like, lamb_gpu_matrix* handle);
LAMB_API int32_t lamb_gpu_matrix_destroy(lamb_gpu_ctx* ctx, lamb_gpu_matrix handle);
/* Optional locality hint: coordinates of the row atoms in sector order
 * (xyz[3*n_rows], subset 1's atoms in local order first) and the orthorhombic
 * cell lengths (box[3]).  LAMB's distributions carry these coordinates
 * (lamb_set coordinates, real_4, src/lamb_set_partition_methods.F90:69-144);
 * the multiply uses them only to order its work along a Morton curve so that
 * concurrently processed C rows share B rows in L2.  Without the hint a
 * Cuthill-McKee order of the block pattern is used.  Results do not depend
 * on the order. */
LAMB_API int32_t lamb_gpu_matrix_set_positions(lamb_gpu_ctx* ctx, lamb_gpu_matrix handle, const float* xyz,
                                               int32_t n_rows, const float* box);
/* Builds a device matrix from a coordinate block list (host arrays): block b
 * sits at global atoms (blk_row[b], blk_col[b]) (1-based) and its
 * column-major elements at data[extents[2b]-1 .. extents[2b+1]-1] (1-based,
 * inclusive; the extent length must equal the block size).  Every atom names
 * its subset (1-based); local atoms follow global order inside a subset.
 * Replaces, on the GPU, lamb_dist_localize_index + internal_distribute at one
 * rank + fill_local_sectors + lamb_index_convert_to_csr
 * (src/lamb_matrix_operations.F90:88-371, src/lamb_index_methods.F90:224-246);
 * blocks may come in any order (they are sorted on the device), duplicates
 * are an error. */
LAMB_API int32_t lamb_gpu_matrix_from_coo(lamb_gpu_ctx* ctx, int32_t n_atom_rows, int32_t n_atom_cols,
                                          const int8_t* row_blk_sizes, const int8_t* col_blk_sizes,
                                          const int32_t* row_subset, const int32_t* col_subset, int64_t n_blks,
                                          const int32_t* blk_row, const int32_t* blk_col, const int64_t* extents,
                                          const double* data, int64_t data_len, lamb_gpu_matrix* handle);

/* DBCSR dump files (the format lamb_load_dbcsr reads,
 * src/lamb_io_operations.F90:267-756).  Host-only; no device needed. */
typedef struct lamb_dbcsr_info {
  char name[81];         /* matrix name (sub-header 1), trailing blanks removed */
  char matrix_type;      /* 'N' (no symmetry), 'S', 'A', 'H', 'K'             */
  int32_t n_chunks;      /* numnodes: chunks (one per writing process)         */
  int32_t data_type;     /* DBCSR data type code as stored                     */
  int32_t n_block_rows;  /* nblkrows_total                                     */
  int32_t n_block_cols;  /* nblkcols_total                                     */
  int64_t n_blks;        /* blocks over all chunks                             */
  int64_t data_len;      /* doubles read: per chunk up to its largest extent   */
} lamb_dbcsr_info;
/* Sizes of a dump (size phase of the size->fill protocol); on failure
 * msg[msg_len] gets the reason. */
LAMB_API int32_t lamb_dbcsr_scan(const char* path, lamb_dbcsr_info* info, char* msg, int32_t msg_len);
/* The dump's blocks in coordinate form (load_dbcsr_chunks,
 * src/lamb_io_operations.F90:525-700): block sizes [n_block_rows] and
 * [n_block_cols], rows/cols [n_blks] (1-based global atoms, chunk after
 * chunk, CSR order inside a chunk), extents [2*n_blks] (1-based, inclusive)
 * into data, the chunks' data areas concatenated (data_cap >= data_len). */
LAMB_API int32_t lamb_dbcsr_read(const char* path, int32_t* row_blk_size, int32_t* col_blk_size, int32_t* rows,
                                 int32_t* cols, int64_t* extents, double* data, int64_t data_cap, char* msg,
                                 int32_t msg_len);
/* lamb_load_dbcsr at one rank: reads a dump ('N' matrices) and builds the
 * device matrix through lamb_gpu_matrix_from_coo.  Atoms are split into
 * n_x_cubes subsets along x by the single-rank partition rule
 * 1 + mod(int(x * (n_x_cubes / h11)), n_x_cubes) in single precision, with
 * h11 the largest x of the coordinates (xyz[3*n_block_rows], the contents of
 * the reference's coordinate file; columns take the row atoms'
 * coordinates); n_x_cubes = 1 puts every atom in subset 1 and needs no
 * coordinates. */
LAMB_API int32_t lamb_gpu_matrix_load_dbcsr(lamb_gpu_ctx* ctx, const char* path, const float* xyz,
                                            int32_t n_x_cubes, lamb_gpu_matrix* handle);
/* Number of sectors, then per-sector sizes (sizes[n_sectors]). */
LAMB_API int32_t lamb_gpu_matrix_n_sectors(lamb_gpu_ctx* ctx, lamb_gpu_matrix handle, int32_t* n_sectors);
/* After a LAMB_GPU_ASYNC multiply into `handle` the block counts are those
 * before the result filter (capacities; data lengths are exact), so the query
 * does not wait for the multiply. */
LAMB_API int32_t lamb_gpu_matrix_query(lamb_gpu_ctx* ctx, lamb_gpu_matrix handle, lamb_c_sector_sizes* sizes,
                              int32_t n_sectors);
/* Fills caller-allocated sectors (out[n_sectors], order as from query);
 * out[s].n_blks and data_len return what was written.  A multiply's result is
 * copied in row chunks, each as soon as the numeric phase has finished it, so
 * after a LAMB_GPU_ASYNC multiply the transfer overlaps the computation. */
LAMB_API int32_t lamb_gpu_matrix_download(lamb_gpu_ctx* ctx, lamb_gpu_matrix handle, lamb_c_sector_out* out,
                                 int32_t n_sectors);

/* ---- goods messages (one sector on the wire) --------------------------------- */
/* The message lamb_goods_X_create packs for the sector exchange
 * (src/lamb_goods_X_types.F90:79-268) and lamb_goods_X_unpack reads
 * (src/lamb_goods_X_methods.F90:166-218): an int64 index (12 1-based
 * (offset, size) slots for index, data, row_p, col_i, extents, flags; then
 * row_p, col_i as int16 four to a word, extents, zero flags; each section at
 * least one word) and the sector's float64 data store.  row_p carries all
 * n_rows + 1 offsets.  Buffers may be host or device memory, so a message can
 * go from one GPU's memory to another's (NCCL or peer copies) or through the
 * host.  `sector` counts in lamb_gpu_matrix_query order. */
LAMB_API int32_t lamb_gpu_goods_size(lamb_gpu_ctx* ctx, lamb_gpu_matrix handle, int32_t sector, int64_t* index_words,
                                     int64_t* data_len);
LAMB_API int32_t lamb_gpu_goods_pack(lamb_gpu_ctx* ctx, lamb_gpu_matrix handle, int32_t sector, int64_t* index,
                                     double* data);
/* A received message as a device matrix of one sector (subset positions 1,1);
 * the receiver supplies what the message does not carry: its column count
 * and the row and column block sizes. */
LAMB_API int32_t lamb_gpu_goods_unpack(lamb_gpu_ctx* ctx, const int64_t* index, int64_t index_words,
                                       const double* data, int32_t n_cols, const int8_t* row_blk_sizes,
                                       const int8_t* col_blk_sizes, lamb_gpu_matrix* handle);

/* ---- multiplication -------------------------------------------------------- */
/* C := A . B (or C += A . B with LAMB_GPU_ACCUMULATE) over all sector triples
 * (A(m,k), B(k,n)) -> C(m,n); replaces lamb_multiply
 * (src/lamb_multiplication.F90:116-204).  A product A_ik.B_kj is skipped when
 * |A_ik|_F*|B_kj|_F < eps and a C block is dropped when |C_ij|_F < eps
 * (both switchable by flags; eps <= 0 disables both).  `c` must be a handle
 * from lamb_gpu_matrix_create_like or a previous multiply; its contents are
 * replaced.  stats may be NULL.  With LAMB_GPU_ASYNC the call returns after
 * the symbolic phase, once the numeric phase and the result filter are
 * queued on the context's stream; the statistics then carry no timings,
 * n_c_blocks counts blocks before the filter and the next call that uses any
 * matrix of the context (or lamb_gpu_matrix_download on C) completes it. */
LAMB_API int32_t lamb_gpu_multiply(lamb_gpu_ctx* ctx, lamb_gpu_matrix a, lamb_gpu_matrix b, lamb_gpu_matrix c,
                          double eps, uint32_t flags, lamb_gpu_mult_stats* stats);

/* Symbolic phase only: builds C's pattern and the block-product stacks and
 * exports the stacks in canonical order for checking.  Per C sector (order
 * of lamb_gpu_matrix_query on the C handle after this call) the stack entries
 * are int64 triples (a_sector, a_blk, b_sector, b_blk, c_blk) with 0-based
 * sector indices into the A/B query order and 0-based block ids within the
 * sector, grouped by block shape (m,n,k) = (row size of C, column size of C,
 * inner size) in ascending order, and ordered by (C row, C column, k) within a
 * group.  n_entries is the capacity on input and the count on output; with
 * entries == NULL only the count is returned. */
LAMB_API int32_t lamb_gpu_multiply_stacks(lamb_gpu_ctx* ctx, lamb_gpu_matrix a, lamb_gpu_matrix b, lamb_gpu_matrix c,
                                 double eps, uint32_t flags, int64_t* entries, int64_t* n_entries);

/* ---- block-sparse matrix algebra used by purification ------------------- */
/* Y := alpha*X + beta*Y over the union pattern (result pattern of Y grows). */
LAMB_API int32_t lamb_gpu_matrix_axpby(lamb_gpu_ctx* ctx, double alpha, lamb_gpu_matrix x, double beta, lamb_gpu_matrix y);
/* Y := copy of X (pattern and values). */
LAMB_API int32_t lamb_gpu_matrix_copy(lamb_gpu_ctx* ctx, lamb_gpu_matrix x, lamb_gpu_matrix y);
/* trace(X) (diagonal blocks of diagonal sectors) and Tr(X.Y) = sum X_ij*Y_ji. */
LAMB_API int32_t lamb_gpu_matrix_trace(lamb_gpu_ctx* ctx, lamb_gpu_matrix x, double* trace);
LAMB_API int32_t lamb_gpu_matrix_trace_product(lamb_gpu_ctx* ctx, lamb_gpu_matrix x, lamb_gpu_matrix y, double* trace);
/* |X|_F and |X - Y|_F over the union pattern. */
LAMB_API int32_t lamb_gpu_matrix_frobenius(lamb_gpu_ctx* ctx, lamb_gpu_matrix x, double* norm);
LAMB_API int32_t lamb_gpu_matrix_diff_frobenius(lamb_gpu_ctx* ctx, lamb_gpu_matrix x, lamb_gpu_matrix y, double* norm);
/* X := alpha*X + shift*I (identity on the diagonal blocks). */
LAMB_API int32_t lamb_gpu_matrix_scale_shift(lamb_gpu_ctx* ctx, lamb_gpu_matrix x, double alpha, double shift);

/* ---- McWeeny purification ------------------------------------------------ */
typedef struct lamb_gpu_purify_report {
  int32_t steps_done;
  int32_t steps_mixed;        /* steps whose products ran in the mixed mode  */
  double trace;               /* Tr(P) after the last step                   */
  double idempotency;         /* |P.P - P|_F / |P|_F after the last step     */
  double ms_total;
} lamb_gpu_purify_report;
/* P_0 := (mu*I - H)*lambda/2 + I/2 with lambda from Gershgorin bounds of H,
 * then `steps` iterations P := 3P^2 - 2P^3; the first steps-fp64_tail run with
 * LAMB_GPU_MIXED products, the last fp64_tail in FP64.  p must come from
 * lamb_gpu_matrix_create_like(h). */
LAMB_API int32_t lamb_gpu_purify_mcweeny(lamb_gpu_ctx* ctx, lamb_gpu_matrix h, double mu, int32_t steps,
                                int32_t fp64_tail, double eps, lamb_gpu_matrix p, lamb_gpu_purify_report* rep);

/* ---- adjoint of C = A.B on a fixed pattern ------------------------------ */
/* dA := (dC . B^T) restricted to A's pattern, dB := (A^T . dC) restricted to
 * B's pattern.  dC must have C's pattern (any pattern is accepted: absent
 * blocks count as zero).  dA/dB must come from create_like(a)/(b) and are
 * overwritten with A's/B's pattern. */
LAMB_API int32_t lamb_gpu_multiply_adjoint(lamb_gpu_ctx* ctx, lamb_gpu_matrix a, lamb_gpu_matrix b, lamb_gpu_matrix dc,
                                  lamb_gpu_matrix da, lamb_gpu_matrix db);

/* ---- batched multiplication ----------------------------------------------- */
/* Many independent C_b = A_b . B_b (FP64) in one persistent launch over a
 * global work queue, replayed from a captured CUDA graph.  All handles must
 * be distinct matrices on this context; c[i] from create_like(a[i]). */
typedef struct lamb_gpu_batch lamb_gpu_batch;
LAMB_API int32_t lamb_gpu_batch_create(lamb_gpu_ctx* ctx, const lamb_gpu_matrix* a, const lamb_gpu_matrix* b,
                              const lamb_gpu_matrix* c, int32_t n, double eps, lamb_gpu_batch** batch);
/* Runs the batch's numeric phase once (first call captures the graph; later
 * calls replay).  Product-filter decisions and C patterns are those of the
 * last full run (or of creation); the block products are recomputed from the
 * current A/B values.  Same as lamb_gpu_batch_run(batch, 0, stats). */
LAMB_API int32_t lamb_gpu_batch_execute(lamb_gpu_batch* batch, lamb_gpu_mult_stats* stats);
/* With LAMB_GPU_BATCH_FULL: the whole multiply of every instance -- symbolic
 * phase from the current values (C patterns, stacks, work queue), the
 * graph-replayed persistent numeric launch (captured again only when the
 * queue's length changed), and the result filter at the batch's eps; the
 * statistics give ms_symbolic, ms_numeric, ms_filter and ms_total for the
 * three parts.  Without it, as lamb_gpu_batch_execute. */
#define LAMB_GPU_BATCH_FULL 1u
LAMB_API int32_t lamb_gpu_batch_run(lamb_gpu_batch* batch, uint32_t flags, lamb_gpu_mult_stats* stats);
/* Queue order the autotuner picked: 0 instance-major (largest instance
 * first), 1 grouped by C block shape. */
LAMB_API int32_t lamb_gpu_batch_queue_order(const lamb_gpu_batch* batch, int32_t* by_shape);
/* Launch shape the autotuner picked at creation: warps per CTA, stack entries
 * per column-table chunk, work items per queue fetch.  The choice is cached
 * per problem signature in the process and, when LAMB_GPU_AUTOTUNE_CACHE
 * names a file, across processes. */
LAMB_API int32_t lamb_gpu_batch_config(const lamb_gpu_batch* batch, int32_t* warps, int32_t* cap, int32_t* grab);
LAMB_API int32_t lamb_gpu_batch_destroy(lamb_gpu_batch* batch);

/* ---- allocation-free entry point ------------------------------------------ */
/* A block-CSR matrix already resident on the device, in the global sector
 * order described above (all pointers are device addresses): row r's blocks
 * are row_p[r] .. row_p[r+1]-1 with global columns col[] ascending, block b
 * is row_bs[r] x col_bs[col[b]] column-major at data + off[b]. */
typedef struct lamb_gpu_dcsr {
  int32_t n_rows, n_cols;
  int64_t nnz;
  const int8_t* row_bs;
  const int8_t* col_bs;
  const int64_t* row_p;
  const int32_t* col;
  const int64_t* off;
  const double* data;
} lamb_gpu_dcsr;

#define LAMB_GPU_NOALLOC_MAX_BLOCKS (1 << 20)

/* Tr(X.Y) for callers that must not allocate device memory (no counterpart in
 * the reference).  Some hosts cannot let a library call cudaMalloc: a code
 * that has handed the whole GPU to its own memory pool at start-up (as
 * Fortran electronic-structure codes often do, so a late cudaMalloc fails or
 * fragments that pool), or one that runs this call between its own
 * pre-allocated stages where an allocation would synchronise the device and
 * break its timing.  This variant takes X and Y as caller-owned device
 * arrays, returns the trace in *result (host memory) and keeps its working
 * storage in a fixed array inside the library: 8 MiB of device memory per
 * GPU, held from the library's first use on that GPU until the process
 * exits.  X may hold at most LAMB_GPU_NOALLOC_MAX_BLOCKS blocks; larger X is
 * rejected with a lamb_wrong_args status, and so is a Y whose block Y_ji is
 * not shaped like X_ij transposed (the two blockings differ).  An empty Y
 * (nnz == 0) may pass null arrays; the trace is then 0.  A CUDA error that
 * was already pending when the call starts is reported as
 * lamb_external_error without launching anything.  The first call on a device looks
 * up that array's device address (cudaGetSymbolAddress) with the device
 * current; make that first call before any stream capture.  Every call uses
 * the same array, so calls whose work overlaps on the GPU (other streams or
 * threads) race with each other; serialise them.  Runs on `stream` (a
 * cudaStream_t, NULL for the legacy default stream) and synchronises it. */
LAMB_API int32_t lamb_gpu_trace_product_noalloc(const lamb_gpu_dcsr* x, const lamb_gpu_dcsr* y, void* stream,
                                                double* result);

#ifdef __cplusplus
}
#endif
#endif /* LAMB_GPU_H */
