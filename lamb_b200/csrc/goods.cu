// Goods messages: one sector in the wire format of the reference's sector
// exchange (lamb_goods_X_create, src/lamb_goods_X_types.F90:79-268;
// lamb_goods_X_unpack, src/lamb_goods_X_methods.F90:166-218).
//
// The index is an int64 word array: 12 slots of 1-based (offset, size) for
// the index itself, the data, row_p, col_i, extents and flags
// (src/lamb_goods_X_types.F90:79-91), then row_p (int64 words), col_i
// (int16 values, four to a word, little-endian), extents (int64 pairs) and
// flags (zero); every section is at least one word.  The data travel as a
// separate float64 array: the sector's data store, which the extents index
// (1-based).  Followed by intent: row_p carries all n_rows + 1 offsets (the
// reference packs n_rows, :160-162, :196) and col_i is read back as int16.
//
// Pack and unpack accept host or device buffers (unified addressing), so a
// message can go straight from one GPU's memory to another's over NVLink
// (NCCL send/recv of the two arrays) or through the host.
#include <cstring>

#include "common.cuh"

namespace lamb {

constexpr int kSlots = 12;
enum GoodsSlot : int {
  kIdxOff = 0, kIdxSize, kDataOff, kDataSize, kRowPOff, kRowPSize, kColIOff, kColISize, kExtOff, kExtSize,
  kFlagsOff, kFlagsSize
};

static int64_t words_of(int64_t bytes) { return std::max<int64_t>(1, (bytes + 7) / 8); }

struct GoodsLayout {
  int64_t hdr[kSlots];
  int64_t w_rows, w_cols, w_ext, w_flags, n_words;
};

static GoodsLayout goods_layout(int64_t n_rows, int64_t n_blks, int64_t data_len) {
  GoodsLayout g{};
  g.w_rows = words_of(8 * (n_rows + 1));
  g.w_cols = words_of(2 * n_blks);
  g.w_ext = words_of(16 * n_blks);
  g.w_flags = words_of(n_blks);
  g.n_words = kSlots + g.w_rows + g.w_cols + g.w_ext + g.w_flags;
  int64_t off = 1 + kSlots;
  g.hdr[kIdxOff] = 1;
  g.hdr[kIdxSize] = g.n_words;
  g.hdr[kDataOff] = 1;
  g.hdr[kDataSize] = data_len;
  g.hdr[kRowPOff] = off; g.hdr[kRowPSize] = n_rows + 1; off += g.w_rows;
  g.hdr[kColIOff] = off; g.hdr[kColISize] = n_blks; off += g.w_cols;
  g.hdr[kExtOff] = off; g.hdr[kExtSize] = n_blks; off += g.w_ext;
  g.hdr[kFlagsOff] = off; g.hdr[kFlagsSize] = n_blks;
  return g;
}

}  // namespace lamb

using namespace lamb;

extern "C" {

int32_t lamb_gpu_goods_size(lamb_gpu_ctx* c, lamb_gpu_matrix h, int32_t sector, int64_t* index_words,
                            int64_t* data_len) {
  auto* ctx = reinterpret_cast<Ctx*>(c);
  if (!ctx || !index_words || !data_len) return make_status(LAMB_LEVEL_FAILURE, LAMB_TYPE_WRONG_ARGS);
  DevMatrix* m = get_matrix(ctx, h);
  if (!m) return fail(ctx, LAMB_LEVEL_FAILURE, LAMB_TYPE_WRONG_ARGS, "goods: invalid handle");
  const int n_sec = m->n_rsub * m->n_csub;
  if (sector < 0 || sector >= n_sec) return fail(ctx, LAMB_LEVEL_FAILURE, LAMB_TYPE_WRONG_ARGS, "goods: no such sector");
  const GoodsLayout g = goods_layout(m->rsub_cnt[sector / m->n_csub], m->sec_nblk[sector], m->sec_dlen[sector]);
  *index_words = g.n_words;
  *data_len = m->sec_dlen[sector];
  return LAMB_GPU_OK;
}

int32_t lamb_gpu_goods_pack(lamb_gpu_ctx* c, lamb_gpu_matrix h, int32_t sector, int64_t* index, double* data) {
  auto* ctx = reinterpret_cast<Ctx*>(c);
  if (!ctx) return make_status(LAMB_LEVEL_FAILURE, LAMB_TYPE_WRONG_ARGS);
  DevMatrix* m = get_matrix(ctx, h);
  if (!m) return fail(ctx, LAMB_LEVEL_FAILURE, LAMB_TYPE_WRONG_ARGS, "goods: invalid handle");
  const int S = m->n_csub, n_sec = m->n_rsub * S;
  if (sector < 0 || sector >= n_sec) return fail(ctx, LAMB_LEVEL_FAILURE, LAMB_TYPE_WRONG_ARGS, "goods: no such sector");
  cudaSetDevice(ctx->device);
  const int a = sector / S, b = sector % S;
  const int64_t n_rows = m->rsub_cnt[a], n_blks = m->sec_nblk[sector], dlen = m->sec_dlen[sector];
  if (!index || (dlen && !data)) return fail(ctx, LAMB_LEVEL_FAILURE, LAMB_TYPE_WRONG_ARGS, "goods: NULL buffer");
  const GoodsLayout g = goods_layout(n_rows, n_blks, dlen);
  SectorIndex si;
  LAMB_TRY(build_sector_index(ctx, m, &si));
  LAMB_CUDA(ctx, cudaStreamSynchronize(ctx->stream));  // h_bcnt
  // header, row_p and zeroed col_i / extents / flags words on the host
  std::vector<int64_t> host(g.n_words, 0);
  memcpy(host.data(), g.hdr, sizeof(g.hdr));
  {
    const int64_t base = (int64_t)m->rsub_base[a] * S + (int64_t)b * n_rows;
    int64_t* rp = host.data() + g.hdr[kRowPOff] - 1;
    rp[0] = 0;
    for (int64_t l = 0; l < n_rows; ++l) rp[l + 1] = rp[l] + (m->nnz ? si.h_bcnt[base + l] : 0);
  }
  LAMB_CUDA(ctx, cudaMemcpyAsync(index, host.data(), sizeof(int64_t) * g.n_words, cudaMemcpyDefault, ctx->stream));
  int64_t first = 0;
  for (int s = 0; s < sector; ++s) first += m->sec_nblk[s];
  if (n_blks) {
    LAMB_CUDA(ctx, cudaMemcpyAsync(index + g.hdr[kColIOff] - 1, si.col16 + first, sizeof(int16_t) * n_blks,
                                   cudaMemcpyDefault, ctx->stream));
    LAMB_CUDA(ctx, cudaMemcpyAsync(index + g.hdr[kExtOff] - 1, si.ext + 2 * first, sizeof(int64_t) * 2 * n_blks,
                                   cudaMemcpyDefault, ctx->stream));
  }
  if (dlen)
    LAMB_CUDA(ctx, cudaMemcpyAsync(data, m->data + m->sec_base[sector], sizeof(double) * dlen, cudaMemcpyDefault,
                                   ctx->stream));
  LAMB_CUDA(ctx, cudaStreamSynchronize(ctx->stream));  // host vector dies here
  free_sector_index(ctx, &si);
  return LAMB_GPU_OK;
}

int32_t lamb_gpu_goods_unpack(lamb_gpu_ctx* c, const int64_t* index, int64_t index_words, const double* data,
                              int32_t n_cols, const int8_t* row_blk_sizes, const int8_t* col_blk_sizes,
                              lamb_gpu_matrix* handle) {
  auto* ctx = reinterpret_cast<Ctx*>(c);
  if (!ctx) return make_status(LAMB_LEVEL_FAILURE, LAMB_TYPE_WRONG_ARGS);
  if (!index || !handle || index_words < kSlots || n_cols < 0 || (n_cols && !col_blk_sizes))
    return fail(ctx, LAMB_LEVEL_FAILURE, LAMB_TYPE_WRONG_ARGS, "goods: bad arguments");
  *handle = 0;
  cudaSetDevice(ctx->device);
  std::vector<int64_t> w(index_words);
  LAMB_CUDA(ctx, cudaMemcpyAsync(w.data(), index, sizeof(int64_t) * index_words, cudaMemcpyDefault, ctx->stream));
  LAMB_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  const int64_t n_rows = w[kRowPSize] - 1, n_blks = w[kColISize], dlen = w[kDataSize];
  if (w[kIdxOff] != 1 || w[kIdxSize] != index_words || n_rows < 0 || n_blks < 0 || w[kExtSize] != n_blks ||
      dlen < 0 || (dlen && !data) || (n_rows && !row_blk_sizes))
    return fail(ctx, LAMB_LEVEL_FAILURE, LAMB_TYPE_WRONG_ARGS, "goods: index header does not describe a sector");
  const GoodsLayout g = goods_layout(n_rows, n_blks, dlen);
  for (int k = 0; k < kSlots; ++k)
    if (g.hdr[k] != w[k]) return fail(ctx, LAMB_LEVEL_FAILURE, LAMB_TYPE_WRONG_ARGS, "goods: inconsistent index header");
  std::vector<int16_t> col(std::max<int64_t>(n_blks, 1));
  if (n_blks) memcpy(col.data(), w.data() + g.hdr[kColIOff] - 1, sizeof(int16_t) * n_blks);
  lamb_c_sector sec{};
  sec.subset_row = 1;
  sec.subset_col = 1;
  sec.n_rows = (int32_t)n_rows;
  sec.n_cols = n_cols;
  sec.row_blk_sizes = row_blk_sizes;
  sec.col_blk_sizes = col_blk_sizes;
  sec.row_p = w.data() + g.hdr[kRowPOff] - 1;
  sec.col_i = col.data();
  sec.extents = w.data() + g.hdr[kExtOff] - 1;
  sec.data = data;
  sec.n_blks = n_blks;
  sec.data_len = dlen;
  return lamb_gpu_matrix_upload(c, &sec, 1, handle);
}

}  // extern "C"
