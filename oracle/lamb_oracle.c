/*
 * CPU restatement of LAMB's sector multiply -- TEST INFRASTRUCTURE ONLY.
 * Rules, reference anchors and the "parity unpinned" status are stated in
 * lamb_oracle.h.  Compiled with -ffp-contract=off so that the only fused
 * operations are the explicit fma() calls.
 */
#include "lamb_oracle.h"

#include <math.h>
#include <omp.h>
#include <stdlib.h>
#include <string.h>

#define ORACLE_KEEP_STACKS_LIMIT 50000000LL

typedef struct {
  int64_t n_blks, n_data;
  int64_t* cols;      /* 0-based local column of each kept block */
  double* data;       /* kept blocks, contiguous, column-major */
  int64_t n_ent;      /* stack entries of the row (pre result filter) */
  int64_t* ent;       /* 6 per entry: a_sector, a_blk, b_sector, b_blk, c_pos_in_row(pre filter), b_k */
  int64_t n_pre;      /* C blocks of the row before the result filter */
  int64_t* pre_cols;  /* their columns (sorted) */
} row_out;

typedef struct {
  int32_t sr, sc, nr, nc;
  int8_t* rbs;
  int8_t* cbs;
  int64_t* row_p;
  int16_t* col_i;
  int64_t* extents;
  double* data;
  int64_t n_blks, data_len;
  /* pre-filter pattern, for the stacks */
  int64_t* pre_row_p;
  int64_t* pre_cols;
  int64_t n_ent;
  int64_t* ent; /* 6 per entry, c = pre-filter block id within the sector, then b_k */
} csec;

struct lamb_oracle_result {
  int32_t n;
  csec* s;
  int64_t n_products, n_skipped, n_dropped;
  double flops;
  int has_stacks;
};

double lamb_oracle_block_norm(const double* x, int64_t n) {
  double s = 0.0;
  for (int64_t e = 0; e < n; ++e) s = fma(x[e], x[e], s);
  return sqrt(s);
}

static int find_sector(const lamb_c_sector* v, int32_t n, int32_t sr, int32_t sc) {
  for (int32_t i = 0; i < n; ++i)
    if (v[i].subset_row == sr && v[i].subset_col == sc) return i;
  return -1;
}

static double* sector_norms(const lamb_c_sector* s) {
  double* nr = (double*)malloc(sizeof(double) * (size_t)(s->n_blks > 0 ? s->n_blks : 1));
  for (int32_t r = 0; r < s->n_rows; ++r)
    for (int64_t b = s->row_p[r]; b < s->row_p[r + 1]; ++b) {
      int64_t len = s->extents[2 * b + 1] - s->extents[2 * b] + 1;
      nr[b] = len > 0 ? lamb_oracle_block_norm(s->data + s->extents[2 * b] - 1, len) : 0.0;
    }
  return nr;
}

typedef struct { int64_t pos, sa, ab, sb, bb, bk; } entry;

static int cmp_i64(const void* x, const void* y) {
  int64_t a = *(const int64_t*)x, b = *(const int64_t*)y;
  return (a > b) - (a < b);
}

int32_t lamb_oracle_multiply(const lamb_c_sector* a, int32_t na, const lamb_c_sector* b, int32_t nb, double eps,
                             uint32_t flags, int32_t n_threads, int32_t row_stride, lamb_oracle_result** out) {
  if (!out || (!a && na) || (!b && nb)) return 1;
  if (row_stride < 1) row_stride = 1;
  const int filt_p = eps > 0 && !(flags & LAMB_GPU_NO_PRODUCT_FILTER);
  const int filt_r = eps > 0 && !(flags & LAMB_GPU_NO_RESULT_FILTER);
  const int use_ld = (flags & ORACLE_LONG_DOUBLE) != 0;
  int32_t Sm = 0, Sk = 0, Sn = 0;
  for (int i = 0; i < na; ++i) {
    if (a[i].subset_row > Sm) Sm = a[i].subset_row;
    if (a[i].subset_col > Sk) Sk = a[i].subset_col;
  }
  for (int i = 0; i < nb; ++i) {
    if (b[i].subset_row > Sk) Sk = b[i].subset_row;
    if (b[i].subset_col > Sn) Sn = b[i].subset_col;
  }
  double** norm_a = (double**)calloc((size_t)na + 1, sizeof(double*));
  double** norm_b = (double**)calloc((size_t)nb + 1, sizeof(double*));
  for (int i = 0; i < na; ++i) norm_a[i] = sector_norms(&a[i]);
  for (int i = 0; i < nb; ++i) norm_b[i] = sector_norms(&b[i]);

  lamb_oracle_result* R = (lamb_oracle_result*)calloc(1, sizeof(*R));
  R->n = Sm * Sn;
  R->s = (csec*)calloc((size_t)R->n > 0 ? R->n : 1, sizeof(csec));
  R->has_stacks = (row_stride == 1) && !(flags & ORACLE_NO_STACKS);
  int nt = n_threads > 0 ? n_threads : omp_get_max_threads();

  for (int32_t m = 1; m <= Sm; ++m)
    for (int32_t n = 1; n <= Sn; ++n) {
      csec* C = &R->s[(m - 1) * Sn + (n - 1)];
      C->sr = m;
      C->sc = n;
      /* Row/column subsets of C come from A's rows and B's columns. */
      int ra = -1, cb = -1;
      for (int i = 0; i < na && ra < 0; ++i) if (a[i].subset_row == m) ra = i;
      for (int i = 0; i < nb && cb < 0; ++i) if (b[i].subset_col == n) cb = i;
      C->nr = ra >= 0 ? a[ra].n_rows : 0;
      C->nc = cb >= 0 ? b[cb].n_cols : 0;
      C->rbs = (int8_t*)malloc((size_t)C->nr + 1);
      C->cbs = (int8_t*)malloc((size_t)C->nc + 1);
      if (C->nr) memcpy(C->rbs, a[ra].row_blk_sizes, (size_t)C->nr);
      if (C->nc) memcpy(C->cbs, b[cb].col_blk_sizes, (size_t)C->nc);
      row_out* rows = (row_out*)calloc((size_t)C->nr + 1, sizeof(row_out));
      int64_t np = 0, nsk = 0, ndr = 0;
      double fl = 0.0;
#pragma omp parallel num_threads(nt) reduction(+ : np, nsk, ndr, fl)
      {
        int64_t* marker = (int64_t*)malloc(sizeof(int64_t) * ((size_t)C->nc + 1));
        for (int32_t j = 0; j < C->nc; ++j) marker[j] = -1;
        int64_t cap_e = 1024, cap_c = 256;
        entry* ents = (entry*)malloc(sizeof(entry) * (size_t)cap_e);
        int64_t* cols = (int64_t*)malloc(sizeof(int64_t) * (size_t)cap_c);
        double* acc = NULL;
        long double* accl = NULL;
        int64_t cap_acc = 0;
#pragma omp for schedule(dynamic, 4)
        for (int32_t l = 0; l < C->nr; ++l) {
          if (l % row_stride) continue;
          const int bi = C->rbs[l];
          int64_t ne = 0, nc = 0;
          for (int32_t ks = 1; ks <= Sk; ++ks) {
            int sa = find_sector(a, na, m, ks), sb = find_sector(b, nb, ks, n);
            if (sa < 0 || sb < 0) continue;
            const lamb_c_sector* A = &a[sa];
            const lamb_c_sector* B = &b[sb];
            for (int64_t ab = A->row_p[l]; ab < A->row_p[l + 1]; ++ab) {
              const int32_t k = A->col_i[ab] - 1;
              const double nA = norm_a[sa][ab];
              const int bk = A->col_blk_sizes[k];
              for (int64_t bb = B->row_p[k]; bb < B->row_p[k + 1]; ++bb) {
                const int32_t j = B->col_i[bb] - 1;
                if (filt_p && nA * norm_b[sb][bb] < eps) { ++nsk; continue; }
                if (marker[j] < 0) {
                  if (nc == cap_c) { cap_c *= 2; cols = (int64_t*)realloc(cols, sizeof(int64_t) * (size_t)cap_c); }
                  marker[j] = nc;
                  cols[nc++] = j;
                }
                if (ne == cap_e) { cap_e *= 2; ents = (entry*)realloc(ents, sizeof(entry) * (size_t)cap_e); }
                ents[ne].pos = j;
                ents[ne].sa = sa; ents[ne].ab = ab; ents[ne].sb = sb; ents[ne].bb = bb; ents[ne].bk = bk;
                ++ne;
                ++np;
                fl += 2.0 * bi * bk * C->cbs[j];
              }
            }
          }
          for (int64_t t = 0; t < nc; ++t) marker[cols[t]] = -1;
          qsort(cols, (size_t)nc, sizeof(int64_t), cmp_i64);
          for (int64_t t = 0; t < nc; ++t) marker[cols[t]] = t;
          /* stable counting sort of the entries by C position */
          int64_t* cstart = (int64_t*)calloc((size_t)nc + 1, sizeof(int64_t));
          for (int64_t e = 0; e < ne; ++e) cstart[marker[ents[e].pos] + 1]++;
          for (int64_t t = 0; t < nc; ++t) cstart[t + 1] += cstart[t];
          entry* sorted = (entry*)malloc(sizeof(entry) * (size_t)(ne > 0 ? ne : 1));
          int64_t* cur = (int64_t*)malloc(sizeof(int64_t) * ((size_t)nc + 1));
          memcpy(cur, cstart, sizeof(int64_t) * (size_t)nc);
          for (int64_t e = 0; e < ne; ++e) {
            int64_t p = marker[ents[e].pos];
            sorted[cur[p]] = ents[e];
            sorted[cur[p]].pos = p;
            cur[p]++;
          }
          free(cur);
          row_out* ro = &rows[l];
          ro->n_pre = nc;
          ro->pre_cols = (int64_t*)malloc(sizeof(int64_t) * (size_t)(nc > 0 ? nc : 1));
          memcpy(ro->pre_cols, cols, sizeof(int64_t) * (size_t)nc);
          if (R->has_stacks && ne <= ORACLE_KEEP_STACKS_LIMIT) {
            ro->n_ent = ne;
            ro->ent = (int64_t*)malloc(sizeof(int64_t) * 6 * (size_t)(ne > 0 ? ne : 1));
            for (int64_t e = 0; e < ne; ++e) {
              ro->ent[6 * e + 0] = sorted[e].sa;
              ro->ent[6 * e + 1] = sorted[e].ab;
              ro->ent[6 * e + 2] = sorted[e].sb;
              ro->ent[6 * e + 3] = sorted[e].bb;
              ro->ent[6 * e + 4] = sorted[e].pos;
              ro->ent[6 * e + 5] = sorted[e].bk;
            }
          }
          /* numeric phase */
          int64_t tot = 0;
          for (int64_t t = 0; t < nc; ++t) tot += (int64_t)bi * C->cbs[cols[t]];
          ro->cols = (int64_t*)malloc(sizeof(int64_t) * (size_t)(nc > 0 ? nc : 1));
          ro->data = (double*)malloc(sizeof(double) * (size_t)(tot > 0 ? tot : 1));
          int64_t kept = 0, dpos = 0;
          for (int64_t t = 0; t < nc; ++t) {
            const int bj = C->cbs[cols[t]];
            const int64_t sz = (int64_t)bi * bj;
            if (sz > cap_acc) {
              cap_acc = sz;
              acc = (double*)realloc(acc, sizeof(double) * (size_t)sz);
              accl = (long double*)realloc(accl, sizeof(long double) * (size_t)sz);
            }
            for (int64_t e = 0; e < sz; ++e) { acc[e] = 0.0; accl[e] = 0.0L; }
            for (int64_t e = cstart[t]; e < cstart[t + 1]; ++e) {
              const lamb_c_sector* A = &a[sorted[e].sa];
              const lamb_c_sector* B = &b[sorted[e].sb];
              const int32_t k = A->col_i[sorted[e].ab] - 1;
              const int bk = A->col_blk_sizes[k];
              const double* pa = A->data + A->extents[2 * sorted[e].ab] - 1;
              const double* pb = B->data + B->extents[2 * sorted[e].bb] - 1;
              if (use_ld) {
                for (int q = 0; q < bj; ++q)
                  for (int kk = 0; kk < bk; ++kk) {
                    const long double bv = pb[q * bk + kk];
                    for (int p = 0; p < bi; ++p) accl[q * bi + p] += (long double)pa[kk * bi + p] * bv;
                  }
              } else {
                for (int q = 0; q < bj; ++q)
                  for (int kk = 0; kk < bk; ++kk) {
                    const double bv = pb[q * bk + kk];
                    for (int p = 0; p < bi; ++p) acc[q * bi + p] = fma(pa[kk * bi + p], bv, acc[q * bi + p]);
                  }
              }
            }
            if (use_ld)
              for (int64_t e = 0; e < sz; ++e) acc[e] = (double)accl[e];
            if (filt_r && lamb_oracle_block_norm(acc, sz) < eps) { ++ndr; continue; }
            ro->cols[kept++] = cols[t];
            memcpy(ro->data + dpos, acc, sizeof(double) * (size_t)sz);
            dpos += sz;
          }
          ro->n_blks = kept;
          ro->n_data = dpos;
          for (int64_t t = 0; t < nc; ++t) marker[cols[t]] = -1;
          free(sorted);
          free(cstart);
        }
        free(marker);
        free(ents);
        free(cols);
        free(acc);
        free(accl);
      }
      R->n_products += np;
      R->n_skipped += nsk;
      R->n_dropped += ndr;
      R->flops += fl;
      /* merge rows into the sector */
      C->row_p = (int64_t*)calloc((size_t)C->nr + 1, sizeof(int64_t));
      C->pre_row_p = (int64_t*)calloc((size_t)C->nr + 1, sizeof(int64_t));
      int64_t nbk = 0, nd = 0, npre = 0, nent = 0;
      for (int32_t l = 0; l < C->nr; ++l) {
        nbk += rows[l].n_blks;
        nd += rows[l].n_data;
        npre += rows[l].n_pre;
        nent += rows[l].n_ent;
        C->row_p[l + 1] = nbk;
        C->pre_row_p[l + 1] = npre;
      }
      C->n_blks = nbk;
      C->data_len = nd;
      C->col_i = (int16_t*)malloc(sizeof(int16_t) * (size_t)(nbk > 0 ? nbk : 1));
      C->extents = (int64_t*)malloc(sizeof(int64_t) * 2 * (size_t)(nbk > 0 ? nbk : 1));
      C->data = (double*)malloc(sizeof(double) * (size_t)(nd > 0 ? nd : 1));
      C->pre_cols = (int64_t*)malloc(sizeof(int64_t) * (size_t)(npre > 0 ? npre : 1));
      C->n_ent = nent;
      C->ent = (int64_t*)malloc(sizeof(int64_t) * 6 * (size_t)(nent > 0 ? nent : 1));
      int64_t bpos = 0, dpos = 0, ppos = 0, epos = 0;
      for (int32_t l = 0; l < C->nr; ++l) {
        row_out* ro = &rows[l];
        const int bi = C->rbs[l];
        for (int64_t t = 0; t < ro->n_blks; ++t) {
          const int64_t sz = (int64_t)bi * C->cbs[ro->cols[t]];
          C->col_i[bpos] = (int16_t)(ro->cols[t] + 1);
          C->extents[2 * bpos] = dpos + 1;
          C->extents[2 * bpos + 1] = dpos + sz;
          ++bpos;
          dpos += sz;
        }
        if (ro->n_data) memcpy(C->data + (dpos - ro->n_data), ro->data, sizeof(double) * (size_t)ro->n_data);
        for (int64_t t = 0; t < ro->n_pre; ++t) C->pre_cols[ppos + t] = ro->pre_cols[t];
        for (int64_t e = 0; e < ro->n_ent; ++e) {
          for (int f = 0; f < 4; ++f) C->ent[6 * epos + f] = ro->ent[6 * e + f];
          C->ent[6 * epos + 4] = ppos + ro->ent[6 * e + 4];
          C->ent[6 * epos + 5] = ro->ent[6 * e + 5];
          ++epos;
        }
        ppos += ro->n_pre;
        free(ro->cols);
        free(ro->data);
        free(ro->pre_cols);
        free(ro->ent);
      }
      free(rows);
    }
  for (int i = 0; i < na; ++i) free(norm_a[i]);
  for (int i = 0; i < nb; ++i) free(norm_b[i]);
  free(norm_a);
  free(norm_b);
  *out = R;
  return 0;
}

int32_t lamb_oracle_n_sectors(const lamb_oracle_result* r) { return r ? r->n : -1; }

int32_t lamb_oracle_sector(const lamb_oracle_result* r, int32_t s, lamb_c_sector* o) {
  if (!r || !o || s < 0 || s >= r->n) return 1;
  const csec* c = &r->s[s];
  o->subset_row = c->sr;
  o->subset_col = c->sc;
  o->n_rows = c->nr;
  o->n_cols = c->nc;
  o->row_blk_sizes = c->rbs;
  o->col_blk_sizes = c->cbs;
  o->row_p = c->row_p;
  o->col_i = c->col_i;
  o->extents = c->extents;
  o->data = c->data;
  o->n_blks = c->n_blks;
  o->data_len = c->data_len;
  return 0;
}

int32_t lamb_oracle_stats(const lamb_oracle_result* r, int64_t* np, int64_t* nsk, double* fl, int64_t* ndr) {
  if (!r) return 1;
  if (np) *np = r->n_products;
  if (nsk) *nsk = r->n_skipped;
  if (fl) *fl = r->flops;
  if (ndr) *ndr = r->n_dropped;
  return 0;
}

typedef struct { int64_t key[4]; int64_t v[5]; } sent;

static int cmp_sent(const void* x, const void* y) {
  const sent* a = (const sent*)x;
  const sent* b = (const sent*)y;
  for (int i = 0; i < 4; ++i)
    if (a->key[i] != b->key[i]) return (a->key[i] > b->key[i]) - (a->key[i] < b->key[i]);
  return 0;
}

/* Canonical order per C sector: shape (m = b_i, n = b_j, k = b_k) ascending,
 * then (C block in CSR order, entry order), which is (C row, C col, k). */
int32_t lamb_oracle_stacks(const lamb_oracle_result* r, int64_t* entries, int64_t* n_entries) {
  if (!r || !n_entries || !r->has_stacks) return 1;
  int64_t tot = 0;
  for (int s = 0; s < r->n; ++s) tot += r->s[s].n_ent;
  if (!entries) { *n_entries = tot; return 0; }
  if (*n_entries < tot) return 2;
  int64_t out = 0;
  for (int s = 0; s < r->n; ++s) {
    const csec* c = &r->s[s];
    sent* v = (sent*)malloc(sizeof(sent) * (size_t)(c->n_ent > 0 ? c->n_ent : 1));
    /* row of each pre-filter block */
    int64_t* brow = (int64_t*)malloc(sizeof(int64_t) * (size_t)(c->pre_row_p[c->nr] > 0 ? c->pre_row_p[c->nr] : 1));
    for (int32_t l = 0; l < c->nr; ++l)
      for (int64_t t = c->pre_row_p[l]; t < c->pre_row_p[l + 1]; ++t) brow[t] = l;
    for (int64_t e = 0; e < c->n_ent; ++e) {
      const int64_t cblk = c->ent[6 * e + 4];
      v[e].key[0] = c->rbs[brow[cblk]];
      v[e].key[1] = c->cbs[c->pre_cols[cblk]];
      v[e].key[2] = c->ent[6 * e + 5];
      v[e].key[3] = e;
      for (int f = 0; f < 5; ++f) v[e].v[f] = c->ent[6 * e + f];
    }
    free(brow);
    qsort(v, (size_t)c->n_ent, sizeof(sent), cmp_sent);
    for (int64_t e = 0; e < c->n_ent; ++e) {
      for (int f = 0; f < 5; ++f) entries[5 * out + f] = v[e].v[f];
      ++out;
    }
    free(v);
  }
  *n_entries = out;
  return 0;
}

int32_t lamb_oracle_free(lamb_oracle_result* r) {
  if (!r) return 0;
  for (int s = 0; s < r->n; ++s) {
    csec* c = &r->s[s];
    free(c->rbs); free(c->cbs); free(c->row_p); free(c->col_i); free(c->extents); free(c->data);
    free(c->pre_row_p); free(c->pre_cols); free(c->ent);
  }
  free(r->s);
  free(r);
  return 0;
}

/* Compares a device result (downloaded sectors `got`) with an oracle result
 * computed WITHOUT the result filter: a reference block is expected in `got`
 * iff !(|C_ij|_F < eps) (all blocks when eps <= 0).  Counts pattern
 * mismatches (expected blocks missing, unexpected blocks present, block
 * sizes), sums |got - ref|^2 and |ref|^2 over the expected blocks, and returns
 * the smallest | |C_ij|_F - eps | / eps over all reference blocks (how close
 * any block sits to the filter threshold; +inf when eps <= 0). */
int32_t lamb_oracle_compare(const lamb_oracle_result* r, const lamb_c_sector* got, int32_t n_got, double eps,
                            int32_t n_threads, int64_t* n_mismatch, double* num, double* den, double* min_gap) {
  if (!r || (!got && n_got) || !n_mismatch || !num || !den || !min_gap) return 1;
  int nt = n_threads > 0 ? n_threads : omp_get_max_threads();
  int64_t mis = 0;
  double sn = 0.0, sd = 0.0, gap = INFINITY;
  for (int s = 0; s < r->n; ++s) {
    const csec* C = &r->s[s];
    const int g = find_sector(got, n_got, C->sr, C->sc);
    if (g < 0) {
      if (C->n_blks) mis += C->n_blks;
      continue;
    }
    const lamb_c_sector* G = &got[g];
    if (G->n_rows != C->nr || G->n_cols != C->nc) { mis += 1; continue; }
    int64_t m_loc = 0;
    double n_loc = 0.0, d_loc = 0.0, g_loc = INFINITY;
#pragma omp parallel for num_threads(nt) schedule(dynamic, 16) reduction(+ : m_loc, n_loc, d_loc) reduction(min : g_loc)
    for (int32_t l = 0; l < C->nr; ++l) {
      int64_t q = G->row_p[l];
      const int64_t qe = G->row_p[l + 1];
      const int bi = C->rbs[l];
      for (int64_t b = C->row_p[l]; b < C->row_p[l + 1]; ++b) {
        const int32_t col = C->col_i[b];
        const int64_t sz = (int64_t)bi * C->cbs[col - 1];
        const double* rv = C->data + C->extents[2 * b] - 1;
        const double nrm = lamb_oracle_block_norm(rv, sz);
        if (eps > 0) {
          const double gp = fabs(nrm - eps) / eps;
          if (gp < g_loc) g_loc = gp;
        }
        const int keep = !(eps > 0) || !(nrm < eps);
        while (q < qe && G->col_i[q] < col) { ++m_loc; ++q; }  /* unexpected block in got */
        const int present = q < qe && G->col_i[q] == col;
        if (keep != present) ++m_loc;
        if (present) {
          const int64_t glen = G->extents[2 * q + 1] - G->extents[2 * q] + 1;
          if (glen != sz) ++m_loc;
          else if (keep) {
            const double* gv = G->data + G->extents[2 * q] - 1;
            for (int64_t e = 0; e < sz; ++e) {
              const double d = gv[e] - rv[e];
              n_loc += d * d;
              d_loc += rv[e] * rv[e];
            }
          }
          ++q;
        }
      }
      m_loc += qe - q;  /* trailing unexpected blocks */
    }
    mis += m_loc;
    sn += n_loc;
    sd += d_loc;
    if (g_loc < gap) gap = g_loc;
  }
  for (int i = 0; i < n_got; ++i) {  /* sectors the reference does not have */
    int found = 0;
    for (int s = 0; s < r->n && !found; ++s) found = r->s[s].sr == got[i].subset_row && r->s[s].sc == got[i].subset_col;
    if (!found) mis += got[i].n_blks;
  }
  *n_mismatch = mis;
  *num = sn;
  *den = sd;
  *min_gap = gap;
  return 0;
}
