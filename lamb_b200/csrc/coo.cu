// Matrices from coordinate block lists on the GPU, and the DBCSR dump reader.
//
// lamb_gpu_matrix_from_coo is the device form of what the reference does
// after it has gathered a matrix's blocks as coordinates: lamb_dist_localize_index
// (global atom -> subset + local atom), internal_distribute (at one rank:
// every block is local) and fill_local_sectors + lamb_index_convert_to_csr
// (src/lamb_matrix_operations.F90:88-371, src/lamb_index_methods.F90:224-246).
// Blocks are sorted by (row, column) in sector order with a device radix sort,
// so the result is row-sorted CSR with sorted columns whatever the input
// order (the reference's convert_to_csr assumes rows already arrive sorted),
// and each block's data is gathered into the sector-major layout.
//
// lamb_dbcsr_scan / lamb_dbcsr_read parse a DBCSR dump as lamb_load_dbcsr and
// load_dbcsr_chunks do (src/lamb_io_operations.F90:267-756): sub-header 1
// (version, name, matrix type, numnodes, data type, block rows/columns and
// their sizes), one sub-header 2 per chunk (blocks, data area size), one
// sub-header 3 per chunk (row_p 0-based, col_i 1-based, blk_p 1-based) and
// the chunks' data areas, all 4-byte integers and 8-byte reals.
// lamb_gpu_matrix_load_dbcsr chains the reader, the single-rank subset rule
// and lamb_gpu_matrix_from_coo.
#include <cub/cub.cuh>

#include <cmath>
#include <cstdio>

#include "common.cuh"

namespace lamb {

enum CooErr : unsigned { kErrRange = 1u, kErrExtent = 2u, kErrDup = 4u };

__global__ void k_coo_keys(int64_t n, const int32_t* __restrict__ rows, const int32_t* __restrict__ cols,
                           const int64_t* __restrict__ ext, int32_t n_ar, int32_t n_ac,
                           const int32_t* __restrict__ rmap, const int32_t* __restrict__ cmap,
                           const int8_t* __restrict__ rbs, const int8_t* __restrict__ cbs, int64_t data_len,
                           unsigned long long* __restrict__ key, int64_t* __restrict__ val,
                           unsigned* __restrict__ err) {
  for (int64_t b = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; b < n; b += (int64_t)gridDim.x * blockDim.x) {
    const int r = rows[b], c = cols[b];
    if (r < 1 || r > n_ar || c < 1 || c > n_ac) {
      atomicOr(err, kErrRange);
      key[b] = ~0ull;
      val[b] = b;
      continue;
    }
    const int64_t e1 = ext[2 * b], e2 = ext[2 * b + 1];
    const int64_t len = (int64_t)rbs[r - 1] * cbs[c - 1];
    if (e2 - e1 + 1 != len || (len > 0 && (e1 < 1 || e2 > data_len))) atomicOr(err, kErrExtent);
    key[b] = ((unsigned long long)(uint32_t)rmap[r - 1] << 32) | (uint32_t)cmap[c - 1];
    val[b] = b;
  }
}

__global__ void k_coo_csr(int64_t n, const unsigned long long* __restrict__ key, int32_t* __restrict__ col,
                          int64_t* __restrict__ row_cnt, unsigned* __restrict__ err) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const unsigned long long k = key[i];
    if (k == ~0ull) continue;
    if (i > 0 && key[i - 1] == k) atomicOr(err, kErrDup);
    col[i] = (int32_t)(k & 0xffffffffull);
    atomicAdd(reinterpret_cast<unsigned long long*>(&row_cnt[k >> 32]), 1ull);
  }
}

// One warp per block: copies the block's elements from the caller's store.
__global__ void k_coo_gather(int64_t n, const int64_t* __restrict__ perm, const int64_t* __restrict__ ext,
                             const int64_t* __restrict__ off, const double* __restrict__ src,
                             double* __restrict__ dst) {
  const int lane = threadIdx.x & 31;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t i = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < n; i += nw) {
    const int64_t b = perm[i];
    const int64_t e1 = ext[2 * b], len = ext[2 * b + 1] - e1 + 1;
    const double* s = src + (e1 - 1);
    double* d = dst + off[i];
    for (int64_t e = lane; e < len; e += 32) d[e] = s[e];
  }
}

static int32_t from_coo_impl(Ctx* ctx, int32_t n_ar, int32_t n_ac, const int8_t* row_bs, const int8_t* col_bs,
                             const int32_t* row_subset, const int32_t* col_subset, int64_t n, const int32_t* rows,
                             const int32_t* cols, const int64_t* extents, const double* data, int64_t data_len,
                             lamb_gpu_matrix* handle) {
  if (n_ar < 0 || n_ac < 0 || n < 0 || data_len < 0 || (n_ar && (!row_bs || !row_subset)) ||
      (n_ac && (!col_bs || !col_subset)) || (n && (!rows || !cols || !extents)) || (data_len && !data))
    return fail(ctx, LAMB_LEVEL_FAILURE, LAMB_TYPE_WRONG_ARGS, "from_coo: bad arguments");
  if (n >= (1ll << 31)) return fail(ctx, LAMB_LEVEL_FAILURE, LAMB_TYPE_UNIMPLEMENTED, "from_coo: 2^31 blocks or more");
  auto m = std::make_unique<DevMatrix>();
  // Subsets and local atoms (global order inside a subset), as
  // lamb_dist_localize_index gives them at one rank.
  auto subsets = [&](int32_t na, const int32_t* sub, int32_t& ns, std::vector<int32_t>& cnt,
                     std::vector<int32_t>& base) -> int32_t {
    ns = na ? 1 : 0;
    for (int32_t a = 0; a < na; ++a) {
      if (sub[a] < 1) return fail(ctx, LAMB_LEVEL_FAILURE, LAMB_TYPE_WRONG_ARGS, "from_coo: subsets are 1-based");
      ns = std::max(ns, sub[a]);
    }
    cnt.assign(ns, 0);
    for (int32_t a = 0; a < na; ++a) ++cnt[sub[a] - 1];
    for (int32_t s = 0; s < ns; ++s)
      if (cnt[s] > 32767)
        return fail(ctx, LAMB_LEVEL_FAILURE, LAMB_TYPE_UNIMPLEMENTED, "from_coo: subset exceeds the int16 local range");
    base.assign(ns + 1, 0);
    for (int32_t s = 0; s < ns; ++s) base[s + 1] = base[s] + cnt[s];
    return LAMB_GPU_OK;
  };
  LAMB_TRY(subsets(n_ar, row_subset, m->n_rsub, m->rsub_cnt, m->rsub_base));
  LAMB_TRY(subsets(n_ac, col_subset, m->n_csub, m->csub_cnt, m->csub_base));
  if (n && (m->n_rsub == 0 || m->n_csub == 0))
    return fail(ctx, LAMB_LEVEL_FAILURE, LAMB_TYPE_WRONG_ARGS, "from_coo: blocks but no atoms");
  m->n_rows = n_ar;
  m->n_cols = n_ac;
  std::vector<int32_t> rmap(n_ar), cmap(n_ac);
  m->h_row_bs.resize(n_ar);
  m->h_col_bs.resize(n_ac);
  {
    std::vector<int32_t> next(m->rsub_base.begin(), m->rsub_base.end() - (m->n_rsub ? 1 : 0));
    for (int32_t a = 0; a < n_ar; ++a) {
      const int32_t p = next[row_subset[a] - 1]++;
      rmap[a] = p;
      m->h_row_bs[p] = row_bs[a];
    }
  }
  {
    std::vector<int32_t> next(m->csub_base.begin(), m->csub_base.end() - (m->n_csub ? 1 : 0));
    for (int32_t a = 0; a < n_ac; ++a) {
      const int32_t p = next[col_subset[a] - 1]++;
      cmap[a] = p;
      m->h_col_bs[p] = col_bs[a];
    }
  }
  for (int32_t a = 0; a < n_ar; ++a)
    if (row_bs[a] < 0) return fail(ctx, LAMB_LEVEL_FAILURE, LAMB_TYPE_WRONG_ARGS, "from_coo: negative block size");
  for (int32_t a = 0; a < n_ac; ++a)
    if (col_bs[a] < 0) return fail(ctx, LAMB_LEVEL_FAILURE, LAMB_TYPE_WRONG_ARGS, "from_coo: negative block size");
  LAMB_TRY(upload_block_sizes(ctx, m.get()));
  LAMB_TRY(dalloc(ctx, &m->row_p, (int64_t)n_ar + 1));
  m->nnz = n;
  // Temporaries: caller arrays on the device, sort keys and values.
  int32_t *d_rows = nullptr, *d_cols = nullptr, *d_rmap = nullptr, *d_cmap = nullptr;
  int8_t *d_rbs = nullptr, *d_cbs = nullptr;
  int64_t *d_ext = nullptr, *val = nullptr, *val2 = nullptr, *cnt = nullptr;
  unsigned long long *key = nullptr, *key2 = nullptr;
  unsigned* d_err = nullptr;
  double* d_src = nullptr;
  void* tmp = nullptr;
  struct Cleanup {
    Ctx* c;
    std::vector<void**> ps;
    ~Cleanup() {
      for (void** p : ps)
        if (*p) { cudaFreeAsync(*p, c->stream); *p = nullptr; }
    }
  } cleanup{ctx, {(void**)&d_rows, (void**)&d_cols, (void**)&d_rmap, (void**)&d_cmap, (void**)&d_rbs, (void**)&d_cbs,
                  (void**)&d_ext, (void**)&val, (void**)&val2, (void**)&cnt, (void**)&key, (void**)&key2,
                  (void**)&d_err, (void**)&d_src, &tmp}};
  const int64_t nb = std::max<int64_t>(n, 1);
  LAMB_TRY(dalloc(ctx, &d_rows, nb));
  LAMB_TRY(dalloc(ctx, &d_cols, nb));
  LAMB_TRY(dalloc(ctx, &d_ext, 2 * nb));
  LAMB_TRY(dalloc(ctx, &d_rmap, std::max(n_ar, 1)));
  LAMB_TRY(dalloc(ctx, &d_cmap, std::max(n_ac, 1)));
  LAMB_TRY(dalloc(ctx, &d_rbs, std::max(n_ar, 1)));
  LAMB_TRY(dalloc(ctx, &d_cbs, std::max(n_ac, 1)));
  LAMB_TRY(dalloc(ctx, &key, nb));
  LAMB_TRY(dalloc(ctx, &key2, nb));
  LAMB_TRY(dalloc(ctx, &val, nb));
  LAMB_TRY(dalloc(ctx, &val2, nb));
  LAMB_TRY(dalloc(ctx, &cnt, (int64_t)n_ar + 1));
  LAMB_TRY(dalloc(ctx, &d_err, 1));
  LAMB_TRY(dalloc(ctx, &d_src, std::max<int64_t>(data_len, 1)));
  auto h2d = [&](void* d, const void* h, size_t bytes) -> int32_t {
    if (bytes) LAMB_CUDA(ctx, cudaMemcpyAsync(d, h, bytes, cudaMemcpyHostToDevice, ctx->stream));
    return LAMB_GPU_OK;
  };
  LAMB_TRY(h2d(d_rows, rows, sizeof(int32_t) * n));
  LAMB_TRY(h2d(d_cols, cols, sizeof(int32_t) * n));
  LAMB_TRY(h2d(d_ext, extents, sizeof(int64_t) * 2 * n));
  LAMB_TRY(h2d(d_rmap, rmap.data(), sizeof(int32_t) * n_ar));
  LAMB_TRY(h2d(d_cmap, cmap.data(), sizeof(int32_t) * n_ac));
  LAMB_TRY(h2d(d_rbs, row_bs, n_ar));
  LAMB_TRY(h2d(d_cbs, col_bs, n_ac));
  LAMB_TRY(h2d(d_src, data, sizeof(double) * data_len));
  LAMB_CUDA(ctx, cudaMemsetAsync(d_err, 0, sizeof(unsigned), ctx->stream));
  LAMB_CUDA(ctx, cudaMemsetAsync(cnt, 0, sizeof(int64_t) * ((int64_t)n_ar + 1), ctx->stream));
  if (n) {
    k_coo_keys<<<grid_for(n), kThreads, 0, ctx->stream>>>(n, d_rows, d_cols, d_ext, n_ar, n_ac, d_rmap, d_cmap,
                                                          d_rbs, d_cbs, data_len, key, val, d_err);
    LAMB_LAUNCHED(ctx);
    size_t tmp_bytes = 0;
    LAMB_CUDA(ctx, cub::DeviceRadixSort::SortPairs(nullptr, tmp_bytes, key, key2, val, val2, (int)n, 0, 64,
                                                   ctx->stream));
    LAMB_TRY(dalloc_bytes(ctx, &tmp, std::max<size_t>(tmp_bytes, 16)));
    LAMB_CUDA(ctx, cub::DeviceRadixSort::SortPairs(tmp, tmp_bytes, key, key2, val, val2, (int)n, 0, 64, ctx->stream));
    LAMB_TRY(dalloc(ctx, &m->col, nb));
    k_coo_csr<<<grid_for(n), kThreads, 0, ctx->stream>>>(n, key2, m->col, cnt + 1, d_err);
    LAMB_LAUNCHED(ctx);
  } else {
    LAMB_TRY(dalloc(ctx, &m->col, 1));
  }
  unsigned h_err = 0;
  LAMB_CUDA(ctx, cudaMemcpyAsync(&h_err, d_err, sizeof(unsigned), cudaMemcpyDeviceToHost, ctx->stream));
  LAMB_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  if (h_err & kErrRange) return fail(ctx, LAMB_LEVEL_FAILURE, LAMB_TYPE_WRONG_ARGS, "from_coo: block atom out of range");
  if (h_err & kErrExtent)
    return fail(ctx, LAMB_LEVEL_FAILURE, LAMB_TYPE_WRONG_ARGS,
                "from_coo: an extent does not match its block size or lies outside the data");
  if (h_err & kErrDup) return fail(ctx, LAMB_LEVEL_FAILURE, LAMB_TYPE_WRONG_ARGS, "from_coo: duplicate block");
  LAMB_TRY(inclusive_scan_i64(ctx, cnt, m->row_p, (int64_t)n_ar + 1));
  LAMB_TRY(layout_sector_major(ctx, m.get(), nullptr));
  LAMB_TRY(dalloc(ctx, &m->data, std::max<int64_t>(m->data_len, 1)));
  if (n) {
    k_coo_gather<<<grid_for(n * 32), kThreads, 0, ctx->stream>>>(n, val2, d_ext, m->off, d_src, m->data);
    LAMB_LAUNCHED(ctx);
  }
  LAMB_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return register_matrix(ctx, std::move(m), handle);
}

// ---- DBCSR dump -----------------------------------------------------------------------
constexpr int kVersionLen = 10, kNameLen = 80;

struct DbcsrFile {
  FILE* f = nullptr;
  ~DbcsrFile() { if (f) fclose(f); }
};

struct DbcsrHeader {
  char name[kNameLen + 1] = {};
  char type = 0;
  int32_t numnodes = 0, data_type = 0, nbr = 0, nbc = 0;
  std::vector<int32_t> rbs, cbs;
  std::vector<int32_t> nblks, area;  // per chunk
  long h3_off = 0;                   // file offset of the first sub-header 3
};

// Reads sub-headers 1 and 2; msg gets the reason on failure.
static bool read_header(FILE* f, DbcsrHeader& h, std::string& msg) {
  char ver[kVersionLen];
  auto rd = [&](void* p, size_t sz, size_t n) { return fread(p, sz, n, f) == n; };
  int32_t meta[4];
  if (!rd(ver, 1, kVersionLen) || !rd(h.name, 1, kNameLen) || !rd(&h.type, 1, 1) || !rd(meta, 4, 4)) {
    msg = "truncated sub-header 1";
    return false;
  }
  h.numnodes = meta[0];
  h.data_type = meta[1];
  h.nbr = meta[2];
  h.nbc = meta[3];
  if (h.numnodes < 1 || h.nbr < 0 || h.nbc < 0) {
    msg = "bad sizes in sub-header 1";
    return false;
  }
  h.rbs.resize(h.nbr);
  h.cbs.resize(h.nbc);
  if ((h.nbr && !rd(h.rbs.data(), 4, h.nbr)) || (h.nbc && !rd(h.cbs.data(), 4, h.nbc))) {
    msg = "truncated block sizes";
    return false;
  }
  for (int32_t v : h.rbs)
    if (v < 0 || v > 127) { msg = "row block size outside 0..127 (int8 block sizes)"; return false; }
  for (int32_t v : h.cbs)
    if (v < 0 || v > 127) { msg = "column block size outside 0..127 (int8 block sizes)"; return false; }
  h.nblks.resize(h.numnodes);
  h.area.resize(h.numnodes);
  for (int c = 0; c < h.numnodes; ++c) {
    int32_t h2[2];
    if (!rd(h2, 4, 2)) { msg = "truncated sub-header 2"; return false; }
    if (h2[0] < 0 || h2[1] < 0) { msg = "negative sizes in sub-header 2"; return false; }
    h.nblks[c] = h2[0];
    h.area[c] = h2[1];
  }
  h.h3_off = ftell(f);
  for (int i = kNameLen - 1; i >= 0 && (h.name[i] == ' ' || h.name[i] == 0); --i) h.name[i] = 0;
  return true;
}

// Walks the chunks: per chunk its index (into rows/cols/ext at `first`) and,
// when data is given, its data area up to the largest extent, appended at
// `dpos`.  Extents are rebased onto the concatenated store.
static bool read_chunks(FILE* f, const DbcsrHeader& h, int32_t* rows, int32_t* cols, int64_t* ext, double* data,
                        int64_t data_cap, int64_t* n_blks_out, int64_t* data_len_out, std::string& msg) {
  const int64_t nbr = h.nbr;
  std::vector<int64_t> h3(h.numnodes), dat(h.numnodes);
  int64_t off = h.h3_off;
  for (int c = 0; c < h.numnodes; ++c) {
    h3[c] = off;
    off += 4 * (nbr + 1) + 8 * (int64_t)h.nblks[c];
  }
  for (int c = 0; c < h.numnodes; ++c) {
    dat[c] = off;
    off += 8 * (int64_t)h.area[c];
  }
  int64_t first = 0, dpos = 0;
  std::vector<int32_t> row_p, col_i, blk_p;
  for (int c = 0; c < h.numnodes; ++c) {
    const int64_t nb = h.nblks[c];
    row_p.resize(nbr + 1);
    col_i.resize(nb);
    blk_p.resize(nb);
    if (fseek(f, (long)h3[c], SEEK_SET) != 0 || fread(row_p.data(), 4, nbr + 1, f) != (size_t)(nbr + 1) ||
        (nb && (fread(col_i.data(), 4, nb, f) != (size_t)nb || fread(blk_p.data(), 4, nb, f) != (size_t)nb))) {
      msg = "truncated sub-header 3 of chunk " + std::to_string(c + 1);
      return false;
    }
    if (row_p[0] != 0 || row_p[nbr] != nb) {
      msg = "row_p of chunk " + std::to_string(c + 1) + " does not span its blocks";
      return false;
    }
    int64_t to_read = 0;
    for (int64_t r = 0; r < nbr; ++r) {
      if (row_p[r + 1] < row_p[r]) { msg = "row_p decreases"; return false; }
      for (int64_t b = row_p[r]; b < row_p[r + 1]; ++b) {
        const int32_t cc = col_i[b];
        if (cc < 1 || cc > h.nbc) { msg = "col_i out of range"; return false; }
        if (blk_p[b] < 1) { msg = "non-positive blk_p (transposed DBCSR blocks) is not supported"; return false; }
        const int64_t e1 = blk_p[b], e2 = e1 - 1 + (int64_t)h.rbs[r] * h.cbs[cc - 1];
        to_read = std::max(to_read, e2);
        if (rows) {
          rows[first + b] = (int32_t)(r + 1);
          cols[first + b] = cc;
          ext[2 * (first + b)] = e1 + dpos;
          ext[2 * (first + b) + 1] = e2 + dpos;
        }
      }
    }
    if (to_read > h.area[c]) {
      msg = "data block extent exceeds the data area of chunk " + std::to_string(c + 1);
      return false;
    }
    if (data) {
      if (dpos + to_read > data_cap) { msg = "data capacity too small"; return false; }
      if (to_read && (fseek(f, (long)dat[c], SEEK_SET) != 0 ||
                      fread(data + dpos, 8, to_read, f) != (size_t)to_read)) {
        msg = "truncated data area of chunk " + std::to_string(c + 1);
        return false;
      }
    }
    first += nb;
    dpos += to_read;
  }
  if (fseek(f, 0, SEEK_END) != 0 || ftell(f) != (long)off) {
    msg = "file size does not match its headers";
    return false;
  }
  *n_blks_out = first;
  *data_len_out = dpos;
  return true;
}

}  // namespace lamb

using namespace lamb;

extern "C" {

int32_t lamb_dbcsr_scan(const char* path, lamb_dbcsr_info* info, char* msg, int32_t msg_len) {
  std::string why;
  auto bad = [&](const std::string& s) {
    if (msg && msg_len > 0) snprintf(msg, (size_t)msg_len, "%s", s.c_str());
    return make_status(LAMB_LEVEL_FAILURE, LAMB_TYPE_EXTERNAL_ERROR);
  };
  if (!path || !info) return make_status(LAMB_LEVEL_FAILURE, LAMB_TYPE_WRONG_ARGS);
  DbcsrFile df;
  df.f = fopen(path, "rb");
  if (!df.f) return bad(std::string("cannot open ") + path);
  DbcsrHeader h;
  if (!read_header(df.f, h, why)) return bad(why);
  int64_t nb = 0, dl = 0;
  if (!read_chunks(df.f, h, nullptr, nullptr, nullptr, nullptr, 0, &nb, &dl, why)) return bad(why);
  memset(info, 0, sizeof(*info));
  memcpy(info->name, h.name, sizeof(info->name) - 1);
  info->matrix_type = h.type;
  info->n_chunks = h.numnodes;
  info->data_type = h.data_type;
  info->n_block_rows = h.nbr;
  info->n_block_cols = h.nbc;
  info->n_blks = nb;
  info->data_len = dl;
  return LAMB_GPU_OK;
}

int32_t lamb_dbcsr_read(const char* path, int32_t* row_blk_size, int32_t* col_blk_size, int32_t* rows, int32_t* cols,
                        int64_t* extents, double* data, int64_t data_cap, char* msg, int32_t msg_len) {
  std::string why;
  auto bad = [&](const std::string& s) {
    if (msg && msg_len > 0) snprintf(msg, (size_t)msg_len, "%s", s.c_str());
    return make_status(LAMB_LEVEL_FAILURE, LAMB_TYPE_EXTERNAL_ERROR);
  };
  if (!path || !row_blk_size || !col_blk_size || !rows || !cols || !extents || (data_cap && !data))
    return make_status(LAMB_LEVEL_FAILURE, LAMB_TYPE_WRONG_ARGS);
  DbcsrFile df;
  df.f = fopen(path, "rb");
  if (!df.f) return bad(std::string("cannot open ") + path);
  DbcsrHeader h;
  if (!read_header(df.f, h, why)) return bad(why);
  std::copy(h.rbs.begin(), h.rbs.end(), row_blk_size);
  std::copy(h.cbs.begin(), h.cbs.end(), col_blk_size);
  int64_t nb = 0, dl = 0;
  if (!read_chunks(df.f, h, rows, cols, extents, data, data_cap, &nb, &dl, why)) return bad(why);
  return LAMB_GPU_OK;
}

int32_t lamb_gpu_matrix_from_coo(lamb_gpu_ctx* c, int32_t n_atom_rows, int32_t n_atom_cols,
                                 const int8_t* row_blk_sizes, const int8_t* col_blk_sizes, const int32_t* row_subset,
                                 const int32_t* col_subset, int64_t n_blks, const int32_t* blk_row,
                                 const int32_t* blk_col, const int64_t* extents, const double* data, int64_t data_len,
                                 lamb_gpu_matrix* handle) {
  auto* ctx = reinterpret_cast<Ctx*>(c);
  if (!ctx) return make_status(LAMB_LEVEL_FAILURE, LAMB_TYPE_WRONG_ARGS);
  if (!handle) return fail(ctx, LAMB_LEVEL_FAILURE, LAMB_TYPE_WRONG_ARGS, "from_coo: no handle");
  *handle = 0;
  cudaSetDevice(ctx->device);
  return from_coo_impl(ctx, n_atom_rows, n_atom_cols, row_blk_sizes, col_blk_sizes, row_subset, col_subset, n_blks,
                       blk_row, blk_col, extents, data, data_len, handle);
}

int32_t lamb_gpu_matrix_load_dbcsr(lamb_gpu_ctx* c, const char* path, const float* xyz, int32_t n_x_cubes,
                                   lamb_gpu_matrix* handle) {
  auto* ctx = reinterpret_cast<Ctx*>(c);
  if (!ctx) return make_status(LAMB_LEVEL_FAILURE, LAMB_TYPE_WRONG_ARGS);
  if (!handle || !path || n_x_cubes < 1 || (n_x_cubes > 1 && !xyz))
    return fail(ctx, LAMB_LEVEL_FAILURE, LAMB_TYPE_WRONG_ARGS,
                "load_dbcsr: need a path, n_x_cubes >= 1 and coordinates when n_x_cubes > 1");
  *handle = 0;
  char msg[256] = {};
  lamb_dbcsr_info info;
  int32_t rc = lamb_dbcsr_scan(path, &info, msg, sizeof(msg));
  if (rc != LAMB_GPU_OK) return fail(ctx, LAMB_LEVEL_FAILURE, LAMB_TYPE_EXTERNAL_ERROR, std::string("load_dbcsr: ") + msg);
  if (info.matrix_type != 'N')
    return fail(ctx, LAMB_LEVEL_FAILURE, LAMB_TYPE_UNIMPLEMENTED,
                "load_dbcsr: only non-symmetric ('N') matrices are supported");
  const int32_t nbr = info.n_block_rows, nbc = info.n_block_cols;
  std::vector<int32_t> rbs(nbr), cbs(nbc), rows(info.n_blks), cols(info.n_blks);
  std::vector<int64_t> ext(2 * info.n_blks);
  std::vector<double> data(info.data_len);
  rc = lamb_dbcsr_read(path, rbs.data(), cbs.data(), rows.data(), cols.data(), ext.data(), data.data(),
                       info.data_len, msg, sizeof(msg));
  if (rc != LAMB_GPU_OK) return fail(ctx, LAMB_LEVEL_FAILURE, LAMB_TYPE_EXTERNAL_ERROR, std::string("load_dbcsr: ") + msg);
  // Subsets at one rank: 1 + mod(int(x * (n / h11)), n) in single precision,
  // h11 the largest row-atom x (src/lamb_io_operations.F90:448-457,
  // src/lamb_partition_methods.F90:85-96); columns share the row atoms'
  // coordinates (:472-480).
  auto subset_of = [&](int32_t na, std::vector<int32_t>& sub) {
    sub.assign(na, 1);
    if (n_x_cubes <= 1 || na == 0) return;
    float h11 = xyz[0];
    for (int32_t a = 1; a < nbr; ++a) h11 = std::max(h11, xyz[3 * a]);
    const float mult = (float)n_x_cubes / h11;
    for (int32_t a = 0; a < na; ++a) {
      const float x = xyz[3 * std::min(a, nbr - 1)];
      int cb = (int)(x * mult) % n_x_cubes;
      if (cb < 0) cb += n_x_cubes;
      sub[a] = cb + 1;
    }
  };
  if (n_x_cubes > 1 && nbc != nbr)
    return fail(ctx, LAMB_LEVEL_FAILURE, LAMB_TYPE_UNIMPLEMENTED,
                "load_dbcsr: coordinates split only square matrices (columns take the row atoms' coordinates)");
  std::vector<int32_t> rsub, csub;
  subset_of(nbr, rsub);
  subset_of(nbc, csub);
  std::vector<int8_t> rb8(rbs.begin(), rbs.end()), cb8(cbs.begin(), cbs.end());
  cudaSetDevice(ctx->device);
  return from_coo_impl(ctx, nbr, nbc, rb8.data(), cb8.data(), rsub.data(), csub.data(), info.n_blks, rows.data(),
                       cols.data(), ext.data(), data.data(), info.data_len, handle);
}

}  // extern "C"
