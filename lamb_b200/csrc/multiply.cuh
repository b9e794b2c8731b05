// Internal interfaces of the multiply (symbolic phase, numeric kernels, filters).
#pragma once
#include "common.cuh"

namespace lamb {

// Output of the symbolic phase.  The stack of C block c is
// stack[stack_p[c] .. stack_p[c+1]), pairs (A block id, B block id) of the
// global CSRs, ordered by k ascending in sector order, i.e. by (k subset,
// local k) -- the canonical order of the build's stacks.
struct Symbolic {
  int64_t c_nnz = 0;
  int64_t n_ent = 0;
  int64_t n_pairs = 0;  // products before the product filter
  double flops = 0;     // sum of 2*b_i*b_k*b_j over the stack
  int64_t* stack_p = nullptr;  // [c_nnz+1]
  int2* stack = nullptr;       // [n_ent]
  int32_t* c_row = nullptr;    // [c_nnz] row of every C block
  int32_t max_stack = 0;       // longest stack of one C block
};
void free_symbolic(Ctx* ctx, Symbolic& s);

int32_t check_compatible(Ctx* ctx, const DevMatrix* A, const DevMatrix* B);
// Builds C's pattern (row_p, col, sector-major off, data buffer) and the stacks.
int32_t symbolic_phase(Ctx* ctx, DevMatrix* A, DevMatrix* B, DevMatrix* C, double eps, bool filt, Symbolic* out);
// Packs (data offset | k block size << 56) for every A block.
int32_t pack_a_meta(Ctx* ctx, const DevMatrix* A, int64_t** a_offk);
int32_t numeric_fp64(Ctx* ctx, const DevMatrix* A, const DevMatrix* B, DevMatrix* C, const Symbolic& sym,
                     const int64_t* a_offk, double* c_nrm);
int32_t numeric_mixed(Ctx* ctx, DevMatrix* A, DevMatrix* B, DevMatrix* C, const Symbolic& sym,
                      const int64_t* a_offk, double* c_nrm, int* slices_used);
// Drops C blocks with c_nrm < eps from the index (data stay in place).
int32_t result_filter(Ctx* ctx, DevMatrix* C, const double* c_nrm, double eps, int64_t* dropped);
// Full multiply on device handles (used by the C ABI, purification and batches).
int32_t multiply_impl(Ctx* ctx, DevMatrix* A, DevMatrix* B, DevMatrix* C, double eps, uint32_t flags,
                      lamb_gpu_mult_stats* stats);

constexpr int64_t kOffMask = (1ll << 56) - 1;

}  // namespace lamb
