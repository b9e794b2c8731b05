// Internal interfaces of the multiply (symbolic phase, numeric kernels, filters).
#pragma once
#include "common.cuh"

namespace lamb {

constexpr int64_t kOffMask = (1ll << 56) - 1;
constexpr int64_t kMask40 = (1ll << 40) - 1;

// One resolved stack entry: the two operand blocks of a block product.
//   a = data offset of operand 1 | (inner block size << 56)
//   b = data offset of operand 2
struct Ent {
  long long a;
  long long b;
};

// One unit of numeric work (a C block), in the processing order:
//   lo = C data offset (40 bits) | rows << 40 | cols << 48
//   hi = first stack entry (40 bits) | entry count << 40
struct Work {
  long long lo;
  long long hi;
};

// Output of the symbolic phase.  The stack of C block c is the entry range
// [stack_p[c], stack_p[c+1]), ordered by k ascending in sector order, i.e. by
// (k subset, local k): the canonical order of the build's stacks.  Entries are
// stored resolved (`ent`, for the numeric kernels) or as block-id pairs
// (`ids`, (A block, B block) of the global CSRs, for exporting stacks).
struct Symbolic {
  int64_t c_nnz = 0;
  int64_t n_ent = 0;
  int64_t n_pairs = 0;  // products before the product filter
  double flops = 0;     // sum of 2*b_i*b_k*b_j over the stack
  int64_t* stack_p = nullptr;  // [c_nnz+1]
  Ent* ent = nullptr;          // [n_ent] when resolved
  int2* ids = nullptr;         // [n_ent] when ids were requested
  int32_t* c_row = nullptr;    // [c_nnz] row of every C block
  std::vector<int64_t> h_row_len;  // C blocks per row (host)
  std::vector<int64_t> h_base;     // C data offset of every (row subset, column subset, rank) run
  bool use_scratch = false;    // set before symbolic_phase: ent lives in the context's scratch
  bool pattern_only = false;   // set before symbolic_phase: C's pattern and layout only, no stacks
  // set before symbolic_phase: C's pattern and layout now, the stacks later
  // one row chunk at a time (numeric_chunks); the fill's parameters are kept
  bool chunked_fill = false;
  std::vector<int64_t> h_row_ent;  // products per C row (host), with chunked_fill
  int32_t fill_n_words = 0, fill_na_max = 0, fill_nc_max = 0;
  double fill_eps = 0.0;
  size_t fill_smem = 0;
};
void free_symbolic(Ctx* ctx, Symbolic& s);

int32_t check_compatible(Ctx* ctx, const DevMatrix* A, const DevMatrix* B);
// Packs (data offset | column block size << 56) for every block of m.
int32_t pack_offk(Ctx* ctx, const DevMatrix* m, bool k_is_col, int64_t** offk);
// Builds C's pattern (row_p, col, sector-major off, data buffer) and the
// stacks; a_offk is required unless want_ids.
// b_meta: operand-2 offsets written into the entries (null: B's data offsets).
int32_t symbolic_phase(Ctx* ctx, DevMatrix* A, DevMatrix* B, DevMatrix* C, double eps, bool filt, bool want_ids,
                       const int64_t* a_offk, Symbolic* out, const int64_t* b_meta = nullptr);
// Work list of C blocks in the row processing order of `order_src` (its h_order).
// use_scratch: work and work_c come from the context's scratch (not to be freed).
int32_t build_work(Ctx* ctx, const DevMatrix* C, const Symbolic& sym, const DevMatrix* order_src, Work** work,
                   int32_t** work_c, bool use_scratch = false);
// Stacked small-GEMM kernels: out_c = sum_e op1_e . op2_e over the work list.
// TA/TB select transposed operands (used by the adjoint); see numeric.cu.
// max_inner: the largest inner block size of any entry (sizes the column table).
int32_t run_stacked(Ctx* ctx, int64_t n_work, const Work* work, const int32_t* work_c, const Ent* ent,
                    const double* d1, const double* d2, double* out, double* out_nrm, bool t1, bool t2,
                    int max_inner);
// Batched execution: operands of one instance, and a tunable launch shape.
struct BatchInst {
  const Ent* ent;
  const double* a;
  const double* b;
  double* c;
  double* nrm;
};
struct BatchConfig {
  int warps = 8;  // warps per CTA (4 or 8)
  int cap = 32;   // stack entries per column-table chunk
  int grab = 4;   // work items per queue fetch
};
int32_t launch_batch(Ctx* ctx, int64_t n_work, const Work* work, const int32_t* work_c, const int32_t* work_i,
                     const BatchInst* inst, unsigned long long* head, const BatchConfig& cfg, int max_inner);
inline int max_block(const std::vector<int8_t>& v) {
  int m = 0;
  for (int8_t x : v) m = x > m ? x : m;
  return m;
}
// int8 digit planes of A (rows scaled by 2^ea) and B (columns scaled by 2^eb).
struct MixedPlanes {
  int s = 0;
  int64_t *rbase = nullptr, *cbase = nullptr;  // element row / column bases
  int *ea = nullptr, *eb = nullptr;            // row / column exponents
  int64_t *a_soff = nullptr, *b_soff = nullptr;  // byte offset of every block in a plane
  int64_t a_plane = 0, b_plane = 0;              // bytes per plane
  int8_t *a_planes = nullptr, *b_planes = nullptr;
};
int mixed_slices_from_env();
// exps_only: only the row / column exponents (and element bases), no planes.
int32_t build_slices(Ctx* ctx, const DevMatrix* A, const DevMatrix* B, int s, MixedPlanes* mp, bool exps_only = false);
// Mixed path on tcgen05 (mixed_tc.cu): shape limits, and the numeric phase
// on cluster tiles (C's pattern set by a pattern-only symbolic phase).
bool mixed_tc_eligible(const DevMatrix* A, const DevMatrix* B);
constexpr int kMixedTcSlices = 6;
int32_t numeric_mixed_tc(Ctx* ctx, DevMatrix* A, DevMatrix* B, DevMatrix* C, const MixedPlanes& mp, double* c_nrm,
                         bool* ran, cudaEvent_t ev_prepared, double* tensor_ops);
void free_slices(Ctx* ctx, MixedPlanes* mp);
int32_t pack_plane_meta(Ctx* ctx, const DevMatrix* A, const MixedPlanes& mp, int64_t** a_meta);
int32_t numeric_mixed(Ctx* ctx, DevMatrix* A, DevMatrix* B, DevMatrix* C, const Symbolic& sym, const Work* work,
                      const int32_t* work_c, double* c_nrm, const MixedPlanes& mp);
// Drops C blocks with c_nrm < eps from the index (data stay in place), on the
// device; C's host block counts are updated by settle() (pending until then).
int32_t result_filter(Ctx* ctx, DevMatrix* C, const double* c_nrm, double eps);
// Full multiply on device handles (used by the C ABI, purification and batches).
int32_t multiply_impl(Ctx* ctx, DevMatrix* A, DevMatrix* B, DevMatrix* C, double eps, uint32_t flags,
                      lamb_gpu_mult_stats* stats);

}  // namespace lamb
