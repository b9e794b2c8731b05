// FP64 numeric phase: stacked small GEMMs on the FP64 tensor pipe (DMMA).
//
// This is the body of the reference's sector_multiply stub
// (src/lamb_multiplication.F90:206-225): every output block is owned by one
// warp (segment ownership, no atomics), which consumes the block's stack as
// ONE concatenated inner dimension,
//     C_ij = sum_e op1_e . op2_e = [op1_1 | op1_2 | ...] . [op2_1 ; op2_2 ; ...],
// padded once per chunk of entries instead of once per entry.
//
// Per chunk the warp writes a column table into shared memory: for every
// inner column kk of the concatenated panel, the address of op1(0,kk) and
// op2(kk,0) and their strides (so that op1(r,kk) = d1[a + r*sa] and
// op2(kk,c) = d2[b + c*sb]).  One 16-byte shared load per column then serves
// any operand transposition (forward product and both adjoint products).
//
// Products use mma.sync .f64 shapes (PTX ISA fragment layouts):
//   m16n8k16 (blocks with 9..16 rows): op1 a_i at (g + 8*(i%2), t + 4*(i/2)),
//     op2 b_i at (t + 4*i, g), out c_i at (g + 8*(i/2), 2t + i%2);
//   m8n8k4 (blocks with <= 8 rows): op1 at (g, t), op2 at (t, g),
//     out at (g, 2t + {0,1});
// with g = lane/4, t = lane%4.  Both run on the FP64 tensor pipe at the same
// peak; m16n8k16 does 16x the work per issued instruction.
//
// Scheduling: warps take work items one at a time from an atomic queue head,
// in the row processing order (Morton / Cuthill-McKee).  All warps then stay
// within a narrow window of neighbouring C rows, whose B rows stay resident in
// L2; a static grid-stride assignment lets warps drift hundreds of items apart
// and was 1.5x slower at 6,144 waters.
#include "multiply.cuh"

namespace lamb {

constexpr int kNumWarps = 8;
constexpr int kMaxChunk = 32;

// Column table entry: pointers to op1(0,kk) and op2(kk,0); the runtime
// stride (the entry's inner block size) sits in the top byte of `pbk`.
struct ColRef {
  const double* pa;
  unsigned long long pbk;
};

__device__ __forceinline__ void dmma884(double& c0, double& c1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
               : "+d"(c0), "+d"(c1)
               : "d"(a), "d"(b));
}

__device__ __forceinline__ void dmma16816(double (&c)[4], const double (&a)[8], const double (&b)[4]) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5,%6,%7,%8,%9,%10,%11}, "
      "{%12,%13,%14,%15}, {%0,%1,%2,%3};"
      : "+d"(c[0]), "+d"(c[1]), "+d"(c[2]), "+d"(c[3])
      : "d"(a[0]), "d"(a[1]), "d"(a[2]), "d"(a[3]), "d"(a[4]), "d"(a[5]), "d"(a[6]), "d"(a[7]), "d"(b[0]),
        "d"(b[1]), "d"(b[2]), "d"(b[3]));
}

// Loads up to `cap` entries starting at `first` and writes the column table;
// returns K, the number of inner columns.  TA/TB: op1/op2 stored transposed,
// i.e. op1(r,kk) = pa[r*ke] (else pa[r]) and op2(kk,c) = pb[c] (else pb[c*ke]).
template <bool TA, bool TB>
__device__ __forceinline__ int build_table(const double* __restrict__ d1, const double* __restrict__ d2,
                                           const Ent* __restrict__ ent, int64_t first, int m, int M, int N,
                                           ColRef* __restrict__ tbl, int lane) {
  Ent x{0, 0};
  if (lane < m) x = ent[first + lane];
  const int ke = lane < m ? (int)((unsigned long long)x.a >> 56) : 0;
  const int incl = warp_incl_scan(ke, lane);
  const int K = __shfl_sync(0xffffffffu, incl, 31);
  const double* pa = d1 + (x.a & kOffMask);
  const double* pb = d2 + x.b;
  const unsigned long long kb = (unsigned long long)ke << 56;
  for (int kc = 0, kk = incl - ke; kc < ke; ++kc, ++kk) {
    const double* ca = TA ? pa + kc : pa + (int64_t)kc * M;
    const double* cb = TB ? pb + (int64_t)kc * N : pb + kc;
    tbl[kk] = ColRef{ca, (unsigned long long)cb | kb};
  }
  __syncwarp();
  return K;
}

// op1(r, kk) and op2(kk, c) for one table column.
template <bool TA>
__device__ __forceinline__ double ld1(const ColRef& cr, int r, int ke, bool ok) {
  return ok ? __ldg(cr.pa + (TA ? (int64_t)r * ke : (int64_t)r)) : 0.0;
}
template <bool TB>
__device__ __forceinline__ double ld2(const double* pb, int c, int ke, bool ok) {
  return ok ? __ldg(pb + (TB ? (int64_t)c : (int64_t)c * ke)) : 0.0;
}
__device__ __forceinline__ const double* col_pb(const ColRef& cr) {
  return reinterpret_cast<const double*>(cr.pbk & kOffMask);
}
__device__ __forceinline__ int col_ke(const ColRef& cr) { return (int)(cr.pbk >> 56); }

// m16n8k16 on 16 output rows r0..r0+15 of a block with more than 8 rows.
// SWAP computes the transposed block (used when the block has <= 8 rows but
// more than 8 columns): tile rows are the block's columns.
template <int NF, bool TA, bool TB, bool SWAP>
__device__ __forceinline__ void block_m16(const double* __restrict__ d1, const double* __restrict__ d2,
                                          double* __restrict__ out, double* __restrict__ out_nrm, int64_t c, int M,
                                          int N, int r0, int c0, int64_t o_off, int64_t s0, int n,
                                          const Ent* __restrict__ ent, ColRef* __restrict__ tbl, int cap,
                                          bool last_slab) {
  const int lane = threadIdx.x & 31;
  const int g = lane >> 2, t = lane & 3;
  const int TM = SWAP ? N : M, TN = SWAP ? M : N;  // tile rows / columns
  double acc[NF][4];
#pragma unroll
  for (int j = 0; j < NF; ++j)
#pragma unroll
    for (int h = 0; h < 4; ++h) acc[j][h] = 0.0;
  const int ra = r0 + g, rb = r0 + g + 8;
  const bool rok0 = ra < TM, rok1 = rb < TM;
  bool cok[NF];
#pragma unroll
  for (int j = 0; j < NF; ++j) cok[j] = c0 + j * 8 + g < TN;
  for (int base = 0; base < n; base += cap) {
    const int m = min(cap, n - base);
    const int K = build_table<TA, TB>(d1, d2, ent, s0 + base, m, M, N, tbl, lane);
    for (int kw = 0; kw < K; kw += 16) {
      double a[8], b[NF][4];
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const int kk = kw + t + 4 * q;
        const bool kv = kk < K;
        const ColRef cr = tbl[kv ? kk : 0];
        const int ke = col_ke(cr);
        const double* pb = col_pb(cr);
        if (!SWAP) {
          a[2 * q] = ld1<TA>(cr, ra, ke, kv && rok0);
          a[2 * q + 1] = ld1<TA>(cr, rb, ke, kv && rok1);
#pragma unroll
          for (int j = 0; j < NF; ++j) b[j][q] = ld2<TB>(pb, c0 + j * 8 + g, ke, kv && cok[j]);
        } else {
          // tile op1(r', kk) = op2(kk, r'); tile op2(kk, c') = op1(c', kk)
          a[2 * q] = ld2<TB>(pb, ra, ke, kv && rok0);
          a[2 * q + 1] = ld2<TB>(pb, rb, ke, kv && rok1);
#pragma unroll
          for (int j = 0; j < NF; ++j) b[j][q] = ld1<TA>(cr, c0 + j * 8 + g, ke, kv && cok[j]);
        }
      }
#pragma unroll
      for (int j = 0; j < NF; ++j) dmma16816(acc[j], a, b[j]);
    }
    __syncwarp();
  }
  double sq = 0.0;
#pragma unroll
  for (int j = 0; j < NF; ++j)
#pragma unroll
    for (int h = 0; h < 4; ++h) {
      const int r = r0 + g + 8 * (h >> 1), cc = c0 + j * 8 + 2 * t + (h & 1);
      if (r < TM && cc < TN) {
        const double v = acc[j][h];
        if (SWAP)
          out[o_off + (int64_t)r * M + cc] = v;
        else
          out[o_off + (int64_t)cc * M + r] = v;
        sq = __fma_rn(v, v, sq);
      }
    }
  sq = warp_sum(sq);
  if (out_nrm) {
    // slabs of one block accumulate |C|^2 in order; the last slab takes the root
    const double prev = (r0 == 0 && c0 == 0) ? 0.0 : out_nrm[c];
    __syncwarp();
    if (lane == 0) out_nrm[c] = last_slab ? __dsqrt_rn(prev + sq) : prev + sq;
    __syncwarp();
  }
}

// Output blocks with at most 8 rows: m8n8k4.
template <int NF, bool TA, bool TB>
__device__ __forceinline__ void block_m8(const double* __restrict__ d1, const double* __restrict__ d2,
                                         double* __restrict__ out, double* __restrict__ out_nrm, int64_t c, int M,
                                         int N, int64_t o_off, int64_t s0, int n, const Ent* __restrict__ ent,
                                         ColRef* __restrict__ tbl, int cap) {
  const int lane = threadIdx.x & 31;
  const int g = lane >> 2, t = lane & 3;
  double acc[NF][2];
#pragma unroll
  for (int j = 0; j < NF; ++j) acc[j][0] = acc[j][1] = 0.0;
  const bool rok = g < M;
  bool cok[NF];
#pragma unroll
  for (int j = 0; j < NF; ++j) cok[j] = j * 8 + g < N;
  for (int base = 0; base < n; base += cap) {
    const int m = min(cap, n - base);
    const int K = build_table<TA, TB>(d1, d2, ent, s0 + base, m, M, N, tbl, lane);
    for (int kw = 0; kw < K; kw += 8) {
      double a[2], b[2][NF];
#pragma unroll
      for (int u = 0; u < 2; ++u) {
        const int kk = kw + 4 * u + t;
        const bool kv = kk < K;
        const ColRef cr = tbl[kv ? kk : 0];
        const int ke = col_ke(cr);
        const double* pb = col_pb(cr);
        a[u] = ld1<TA>(cr, g, ke, kv && rok);
#pragma unroll
        for (int j = 0; j < NF; ++j) b[u][j] = ld2<TB>(pb, j * 8 + g, ke, kv && cok[j]);
      }
#pragma unroll
      for (int u = 0; u < 2; ++u)
#pragma unroll
        for (int j = 0; j < NF; ++j) dmma884(acc[j][0], acc[j][1], a[u], b[u][j]);
    }
    __syncwarp();
  }
  double sq = 0.0;
#pragma unroll
  for (int j = 0; j < NF; ++j)
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int cc = j * 8 + 2 * t + h;
      if (g < M && cc < N) {
        const double v = acc[j][h];
        out[o_off + (int64_t)cc * M + g] = v;
        sq = __fma_rn(v, v, sq);
      }
    }
  sq = warp_sum(sq);
  if (lane == 0 && out_nrm) out_nrm[c] = __dsqrt_rn(sq);
}

// Blocks larger than 32 rows or 24 columns: plain FP64 FMAs, one output
// element per lane and step.
template <bool TA, bool TB>
__device__ void block_generic(const double* __restrict__ d1, const double* __restrict__ d2, double* __restrict__ out,
                              double* __restrict__ out_nrm, int64_t c, int M, int N, int64_t o_off, int64_t s0, int n,
                              const Ent* __restrict__ ent) {
  const int lane = threadIdx.x & 31;
  double sq = 0.0;
  for (int el = lane; el < M * N; el += 32) {
    const int r = el % M, cc = el / M;
    double acc = 0.0;
    for (int s = 0; s < n; ++s) {
      const Ent x = ent[s0 + s];
      const int ke = (int)((unsigned long long)x.a >> 56);
      const double* p1 = d1 + (x.a & kOffMask);
      const double* p2 = d2 + x.b;
      for (int kc = 0; kc < ke; ++kc) {
        const double u = TA ? p1[(int64_t)kc + (int64_t)r * ke] : p1[(int64_t)r + (int64_t)kc * M];
        const double v = TB ? p2[(int64_t)cc + (int64_t)kc * N] : p2[(int64_t)kc + (int64_t)cc * ke];
        acc = __fma_rn(u, v, acc);
      }
    }
    out[o_off + (int64_t)cc * M + r] = acc;
    sq = __fma_rn(acc, acc, sq);
  }
  sq = warp_sum(sq);
  if (lane == 0 && out_nrm) out_nrm[c] = __dsqrt_rn(sq);
}

// One work item: dispatch on the output block shape.
template <bool TA, bool TB>
__device__ __forceinline__ void process_item(const Work& it, int64_t c, const Ent* __restrict__ ent,
                                             const double* __restrict__ d1, const double* __restrict__ d2,
                                             double* __restrict__ out, double* __restrict__ out_nrm,
                                             ColRef* __restrict__ tbl, int cap) {
  const int64_t o_off = it.lo & kMask40;
  const int M = (int)((it.lo >> 40) & 0xff), N = (int)((it.lo >> 48) & 0xff);
  const int64_t s0 = it.hi & kMask40;
  const int n = (int)((unsigned long long)it.hi >> 40);
  if (M == 0 || N == 0) {
    if ((threadIdx.x & 31) == 0 && out_nrm) out_nrm[c] = 0.0;
    return;
  }
  if (M <= 8 && N <= 8) {
    block_m8<1, TA, TB>(d1, d2, out, out_nrm, c, M, N, o_off, s0, n, ent, tbl, cap);
  } else if (M <= 8 && N <= 32) {
    for (int r0 = 0; r0 < N; r0 += 16)
      block_m16<1, TA, TB, true>(d1, d2, out, out_nrm, c, M, N, r0, 0, o_off, s0, n, ent, tbl, cap, r0 + 16 >= N);
  } else if (M <= 32 && N <= 32) {
    // 16-row x 16-column slabs (the last may be 8 columns wide)
    for (int r0 = 0; r0 < M; r0 += 16)
      for (int c0 = 0; c0 < N; c0 += 16) {
        const bool last = r0 + 16 >= M && c0 + 16 >= N;
        if (N - c0 > 8)
          block_m16<2, TA, TB, false>(d1, d2, out, out_nrm, c, M, N, r0, c0, o_off, s0, n, ent, tbl, cap, last);
        else
          block_m16<1, TA, TB, false>(d1, d2, out, out_nrm, c, M, N, r0, c0, o_off, s0, n, ent, tbl, cap, last);
      }
  } else {
    block_generic<TA, TB>(d1, d2, out, out_nrm, c, M, N, o_off, s0, n, ent);
  }
}

template <bool TA, bool TB>
__global__ void __launch_bounds__(kNumWarps * 32, 3)
    k_stacked(int64_t n_work, const Work* __restrict__ work, const int32_t* __restrict__ work_c,
              const Ent* __restrict__ ent, const double* __restrict__ d1, const double* __restrict__ d2,
              double* __restrict__ out, double* __restrict__ out_nrm, int cap, int tbl_cols,
              unsigned long long* __restrict__ head) {
  extern __shared__ ColRef tbl_all[];
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  ColRef* tbl = tbl_all + (size_t)w * tbl_cols;
  while (true) {
    unsigned long long v = 0;
    if (lane == 0) v = atomicAdd(head, 1ull);
    v = __shfl_sync(0xffffffffu, v, 0);
    if (v >= (unsigned long long)n_work) break;
    process_item<TA, TB>(work[v], work_c[v], ent, d1, d2, out, out_nrm, tbl, cap);
  }
}

// Persistent kernel over the global queue of a batch: warps take `grab`
// consecutive items per atomic on `head` (reset before every launch); each
// item names its instance, whose operands come from the instance table.
template <int NW>
__global__ void __launch_bounds__(NW * 32, 24 / NW)
    k_stacked_batch(int64_t n_work, const Work* __restrict__ work, const int32_t* __restrict__ work_c,
                    const int32_t* __restrict__ work_i, const BatchInst* __restrict__ inst,
                    unsigned long long* __restrict__ head, int grab, int cap, int tbl_cols) {
  extern __shared__ ColRef tbl_all[];
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  ColRef* tbl = tbl_all + (size_t)w * tbl_cols;
  while (true) {
    unsigned long long start = 0;
    if (lane == 0) start = atomicAdd(head, (unsigned long long)grab);
    start = __shfl_sync(0xffffffffu, start, 0);
    if (start >= (unsigned long long)n_work) break;
    const int64_t end = min((int64_t)start + grab, n_work);
    for (int64_t v = (int64_t)start; v < end; ++v) {
      const BatchInst I = inst[work_i[v]];
      process_item<false, false>(work[v], work_c[v], I.ent, I.a, I.b, I.c, I.nrm, tbl, cap);
    }
  }
}

// Stack entries per column-table chunk: at most `want`, and few enough that
// the tables of `warps` warps (cap x max_inner columns each) fit the device's
// opt-in shared memory per CTA (227 KB on B200; blocks of 127 rows allow 14
// entries per chunk).
static int table_cap(Ctx* ctx, int want, int max_inner, int warps) {
  int optin = 0;
  if (cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, ctx->device) != cudaSuccess || optin <= 0)
    optin = 48 * 1024;
  const int fit = optin / (int)(sizeof(ColRef) * (size_t)max_inner * warps);
  return std::max(1, std::min(want, std::min(8192 / max_inner, fit)));
}

template <int NW>
static int32_t launch_batch_nw(Ctx* ctx, int64_t n_work, const Work* work, const int32_t* work_c,
                               const int32_t* work_i, const BatchInst* inst, unsigned long long* head, int grab,
                               int cap, int max_inner) {
  const int mi = std::max(1, std::min(max_inner, 127));
  cap = table_cap(ctx, cap, mi, NW);
  const int tbl_cols = cap * mi;
  const size_t smem = sizeof(ColRef) * (size_t)tbl_cols * NW;
  auto kern = k_stacked_batch<NW>;
  if (smem > 48 * 1024)
    LAMB_CUDA(ctx, cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  int sms = 148, per_sm = 1;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx->device);
  LAMB_CUDA(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, NW * 32, smem));
  const int grid = sms * std::max(per_sm, 1);
  kern<<<grid, NW * 32, smem, ctx->stream>>>(n_work, work, work_c, work_i, inst, head, grab, cap, tbl_cols);
  LAMB_LAUNCHED(ctx);
  return LAMB_GPU_OK;
}

int32_t launch_batch(Ctx* ctx, int64_t n_work, const Work* work, const int32_t* work_c, const int32_t* work_i,
                     const BatchInst* inst, unsigned long long* head, const BatchConfig& cfg, int max_inner) {
  if (n_work == 0) return LAMB_GPU_OK;
  if (cfg.warps == 4) return launch_batch_nw<4>(ctx, n_work, work, work_c, work_i, inst, head, cfg.grab, cfg.cap, max_inner);
  return launch_batch_nw<8>(ctx, n_work, work, work_c, work_i, inst, head, cfg.grab, cfg.cap, max_inner);
}

template <bool TA, bool TB>
static int32_t launch_stacked(Ctx* ctx, int64_t n_work, const Work* work, const int32_t* work_c, const Ent* ent,
                              const double* d1, const double* d2, double* out, double* out_nrm, int max_inner) {
  // Column table per warp: `cap` entries of up to max_inner columns each.
  const int mi = std::max(1, std::min(max_inner, 127));
  const int cap = table_cap(ctx, kMaxChunk, mi, kNumWarps);
  const int tbl_cols = cap * mi;
  const size_t smem = sizeof(ColRef) * (size_t)tbl_cols * kNumWarps;
  auto kern = k_stacked<TA, TB>;
  if (smem > 48 * 1024)
    LAMB_CUDA(ctx, cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  int sms = 148, per_sm = 1;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx->device);
  LAMB_CUDA(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kNumWarps * 32, smem));
  const int64_t need = (n_work + kNumWarps - 1) / kNumWarps;
  const int grid = (int)std::max<int64_t>(1, std::min<int64_t>(need, (int64_t)sms * std::max(per_sm, 1)));
  unsigned long long* head = nullptr;
  LAMB_TRY(dalloc(ctx, &head, 1));
  LAMB_CUDA(ctx, cudaMemsetAsync(head, 0, sizeof(unsigned long long), ctx->stream));
  kern<<<grid, kNumWarps * 32, smem, ctx->stream>>>(n_work, work, work_c, ent, d1, d2, out, out_nrm, cap, tbl_cols, head);
  LAMB_LAUNCHED(ctx);
  dfree(ctx, head);
  return LAMB_GPU_OK;
}

int32_t run_stacked(Ctx* ctx, int64_t n_work, const Work* work, const int32_t* work_c, const Ent* ent,
                    const double* d1, const double* d2, double* out, double* out_nrm, bool t1, bool t2,
                    int max_inner) {
  if (n_work == 0) return LAMB_GPU_OK;
  if (!t1 && !t2) return launch_stacked<false, false>(ctx, n_work, work, work_c, ent, d1, d2, out, out_nrm, max_inner);
  if (!t1 && t2) return launch_stacked<false, true>(ctx, n_work, work, work_c, ent, d1, d2, out, out_nrm, max_inner);
  if (t1 && !t2) return launch_stacked<true, false>(ctx, n_work, work, work_c, ent, d1, d2, out, out_nrm, max_inner);
  return fail(ctx, LAMB_LEVEL_FAILURE, LAMB_TYPE_INTERNAL_ERROR, "unsupported operand transposition");
}

}  // namespace lamb
