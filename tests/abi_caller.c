/*
 * abi_caller.c -- a plain C99 program that drives lamb_gpu.h the way a
 * compiled LAMB caller would: the body of lamb_multiply
 * (src/lamb_multiplication.F90:116-204) reduced to upload A and B, create C
 * like A, multiply, query the sizes of C, allocate, download, destroy.  No
 * Python, torch or C++ is involved on this path.
 *
 *   abi_caller IN OUT EPS FLAGS
 *
 * IN holds A then B, OUT receives C, each as
 *   int64 n_sectors, then per sector
 *   int64 subset_row, subset_col, n_rows, n_cols, n_blks, data_len,
 *   int8 row_blk_sizes[n_rows], int8 col_blk_sizes[n_cols],
 *   int64 row_p[n_rows+1], int16 col_i[n_blks], int64 extents[2*n_blks],
 *   float64 data[data_len]
 * (little-endian, no padding).  The program also checks that a bad handle is
 * refused with a decodable status and a message.
 *
 * Exit codes: 0 success, 1 usage or I/O error, 2 a library call failed,
 * 3 no device could be opened (lamb_gpu_ctx_create failed; the status and
 * message are printed).
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "lamb_gpu.h"

typedef struct {
  int32_t n;
  lamb_c_sector* s;
} host_matrix;

static int read_all(FILE* f, void* p, size_t size, size_t count) {
  if (count == 0) return 0;
  return fread(p, size, count, f) == count ? 0 : -1;
}

static void* xalloc(size_t bytes) {
  void* p = malloc(bytes > 0 ? bytes : 1);
  if (!p) {
    fprintf(stderr, "out of host memory\n");
    exit(1);
  }
  return p;
}

static int read_matrix(FILE* f, host_matrix* m) {
  int64_t n = 0;
  int32_t i;
  if (read_all(f, &n, sizeof n, 1) || n < 0 || n > 1 << 20) return -1;
  m->n = (int32_t)n;
  m->s = (lamb_c_sector*)xalloc(sizeof(lamb_c_sector) * (size_t)n);
  for (i = 0; i < m->n; ++i) {
    int64_t h[6];
    int8_t *rb, *cb;
    int64_t *row_p, *ext;
    int16_t* col_i;
    double* data;
    if (read_all(f, h, sizeof(int64_t), 6)) return -1;
    if (h[2] < 0 || h[3] < 0 || h[4] < 0 || h[5] < 0) return -1;
    rb = (int8_t*)xalloc((size_t)h[2]);
    cb = (int8_t*)xalloc((size_t)h[3]);
    row_p = (int64_t*)xalloc(sizeof(int64_t) * (size_t)(h[2] + 1));
    col_i = (int16_t*)xalloc(sizeof(int16_t) * (size_t)h[4]);
    ext = (int64_t*)xalloc(sizeof(int64_t) * 2 * (size_t)h[4]);
    data = (double*)xalloc(sizeof(double) * (size_t)h[5]);
    if (read_all(f, rb, 1, (size_t)h[2]) || read_all(f, cb, 1, (size_t)h[3]) ||
        read_all(f, row_p, sizeof(int64_t), (size_t)h[2] + 1) || read_all(f, col_i, sizeof(int16_t), (size_t)h[4]) ||
        read_all(f, ext, sizeof(int64_t), 2 * (size_t)h[4]) || read_all(f, data, sizeof(double), (size_t)h[5]))
      return -1;
    m->s[i].subset_row = (int32_t)h[0];
    m->s[i].subset_col = (int32_t)h[1];
    m->s[i].n_rows = (int32_t)h[2];
    m->s[i].n_cols = (int32_t)h[3];
    m->s[i].row_blk_sizes = rb;
    m->s[i].col_blk_sizes = cb;
    m->s[i].row_p = row_p;
    m->s[i].col_i = col_i;
    m->s[i].extents = ext;
    m->s[i].data = data;
    m->s[i].n_blks = h[4];
    m->s[i].data_len = h[5];
  }
  return 0;
}

static void free_matrix(host_matrix* m) {
  int32_t i;
  for (i = 0; i < m->n; ++i) {
    free((void*)m->s[i].row_blk_sizes);
    free((void*)m->s[i].col_blk_sizes);
    free((void*)m->s[i].row_p);
    free((void*)m->s[i].col_i);
    free((void*)m->s[i].extents);
    free((void*)m->s[i].data);
  }
  free(m->s);
}

static int report(lamb_gpu_ctx* ctx, const char* what, int32_t st) {
  char msg[512];
  msg[0] = '\0';
  if (ctx) lamb_gpu_last_error(ctx, msg, (int32_t)sizeof msg);
  fprintf(stderr, "%s: status %d level %d type %d: %s\n", what, (int)st, (int)lamb_gpu_status_level(st),
          (int)lamb_gpu_status_type(st), msg);
  return 2;
}

#define CALL(what, expr)                          \
  do {                                            \
    const int32_t st_ = (expr);                   \
    if (st_ != LAMB_GPU_OK) return report(ctx, what, st_); \
  } while (0)

static int write_sector(FILE* f, const lamb_c_sector_out* s) {
  const int64_t h[6] = {s->subset_row, s->subset_col, s->n_rows, s->n_cols, s->n_blks, s->data_len};
  size_t ok = fwrite(h, sizeof(int64_t), 6, f) == 6;
  ok = ok && fwrite(s->row_blk_sizes, 1, (size_t)s->n_rows, f) == (size_t)s->n_rows;
  ok = ok && fwrite(s->col_blk_sizes, 1, (size_t)s->n_cols, f) == (size_t)s->n_cols;
  ok = ok && fwrite(s->row_p, sizeof(int64_t), (size_t)s->n_rows + 1, f) == (size_t)s->n_rows + 1;
  ok = ok && fwrite(s->col_i, sizeof(int16_t), (size_t)s->n_blks, f) == (size_t)s->n_blks;
  ok = ok && fwrite(s->extents, sizeof(int64_t), 2 * (size_t)s->n_blks, f) == 2 * (size_t)s->n_blks;
  ok = ok && fwrite(s->data, sizeof(double), (size_t)s->data_len, f) == (size_t)s->data_len;
  return ok ? 0 : -1;
}

static int run(lamb_gpu_ctx* ctx, const host_matrix* a, const host_matrix* b, double eps, uint32_t flags,
               const char* out_path) {
  lamb_gpu_matrix ha = 0, hb = 0, hc = 0;
  lamb_gpu_mult_stats stats;
  lamb_c_sector_sizes* sizes;
  lamb_c_sector_out* out;
  int32_t n = 0, i, st;
  FILE* f;

  CALL("upload A", lamb_gpu_matrix_upload(ctx, a->s, a->n, &ha));
  CALL("upload B", lamb_gpu_matrix_upload(ctx, b->s, b->n, &hb));
  CALL("create C", lamb_gpu_matrix_create_like(ctx, ha, &hc));

  /* A handle that was never issued must be refused, not crash. */
  st = lamb_gpu_multiply(ctx, ha, hb, hc + 1000, eps, flags, &stats);
  if (st == LAMB_GPU_OK || lamb_gpu_status_level(st) < LAMB_LEVEL_FAILURE) {
    fprintf(stderr, "a bad handle was accepted (status %d)\n", (int)st);
    return 2;
  }
  report(ctx, "bad handle (expected)", st);

  CALL("multiply", lamb_gpu_multiply(ctx, ha, hb, hc, eps, flags, &stats));
  CALL("n_sectors", lamb_gpu_matrix_n_sectors(ctx, hc, &n));
  sizes = (lamb_c_sector_sizes*)xalloc(sizeof(lamb_c_sector_sizes) * (size_t)n);
  out = (lamb_c_sector_out*)xalloc(sizeof(lamb_c_sector_out) * (size_t)n);
  CALL("query", lamb_gpu_matrix_query(ctx, hc, sizes, n));
  for (i = 0; i < n; ++i) {
    out[i].subset_row = sizes[i].subset_row;
    out[i].subset_col = sizes[i].subset_col;
    out[i].n_rows = sizes[i].n_rows;
    out[i].n_cols = sizes[i].n_cols;
    out[i].row_blk_sizes = (int8_t*)xalloc((size_t)sizes[i].n_rows);
    out[i].col_blk_sizes = (int8_t*)xalloc((size_t)sizes[i].n_cols);
    out[i].row_p = (int64_t*)xalloc(sizeof(int64_t) * ((size_t)sizes[i].n_rows + 1));
    out[i].col_i = (int16_t*)xalloc(sizeof(int16_t) * (size_t)sizes[i].n_blks);
    out[i].extents = (int64_t*)xalloc(sizeof(int64_t) * 2 * (size_t)sizes[i].n_blks);
    out[i].data = (double*)xalloc(sizeof(double) * (size_t)sizes[i].data_len);
    out[i].n_blks = sizes[i].n_blks;
    out[i].data_len = sizes[i].data_len;
  }
  CALL("download", lamb_gpu_matrix_download(ctx, hc, out, n));

  f = fopen(out_path, "wb");
  if (!f) {
    fprintf(stderr, "cannot write %s\n", out_path);
    return 1;
  }
  {
    const int64_t n64 = n;
    int bad = fwrite(&n64, sizeof n64, 1, f) != 1;
    for (i = 0; i < n && !bad; ++i) bad = write_sector(f, &out[i]) != 0;
    if (fclose(f) != 0 || bad) {
      fprintf(stderr, "short write to %s\n", out_path);
      return 1;
    }
  }
  printf("products %lld skipped %lld c_blocks %lld dropped %lld flops %.0f launches %d\n",
         (long long)stats.n_products, (long long)stats.n_products_skipped, (long long)stats.n_c_blocks,
         (long long)stats.n_c_blocks_dropped, stats.flops, (int)stats.kernel_launches);
  for (i = 0; i < n; ++i) {
    free(out[i].row_blk_sizes);
    free(out[i].col_blk_sizes);
    free(out[i].row_p);
    free(out[i].col_i);
    free(out[i].extents);
    free(out[i].data);
  }
  free(out);
  free(sizes);
  CALL("destroy C", lamb_gpu_matrix_destroy(ctx, hc));
  CALL("destroy B", lamb_gpu_matrix_destroy(ctx, hb));
  CALL("destroy A", lamb_gpu_matrix_destroy(ctx, ha));
  return 0;
}

int main(int argc, char** argv) {
  host_matrix a, b;
  lamb_gpu_ctx* ctx = NULL;
  FILE* f;
  int32_t st;
  int rc;
  if (argc != 5) {
    fprintf(stderr, "usage: %s IN OUT EPS FLAGS\n", argv[0]);
    return 1;
  }
  f = fopen(argv[1], "rb");
  if (!f) {
    fprintf(stderr, "cannot open %s\n", argv[1]);
    return 1;
  }
  if (read_matrix(f, &a) || read_matrix(f, &b)) {
    fprintf(stderr, "malformed input %s\n", argv[1]);
    fclose(f);
    return 1;
  }
  fclose(f);
  st = lamb_gpu_ctx_create(0, &ctx);
  if (st != LAMB_GPU_OK) {
    fprintf(stderr, "ctx_create: status %d level %d type %d\n", (int)st, (int)lamb_gpu_status_level(st),
            (int)lamb_gpu_status_type(st));
    free_matrix(&a);
    free_matrix(&b);
    return 3;
  }
  rc = run(ctx, &a, &b, strtod(argv[3], NULL), (uint32_t)strtoul(argv[4], NULL, 0), argv[2]);
  st = lamb_gpu_ctx_destroy(ctx);
  if (rc == 0 && st != LAMB_GPU_OK) rc = report(NULL, "ctx_destroy", st);
  free_matrix(&a);
  free_matrix(&b);
  return rc;
}
