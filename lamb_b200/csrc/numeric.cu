// FP64 numeric phase: stacked small GEMMs on the FP64 tensor pipe (DMMA).
//
// This is the body of the reference's sector_multiply stub
// (src/lamb_multiplication.F90:206-225): every C block is owned by one warp
// (segment ownership, no atomics), which consumes the block's stack as ONE
// concatenated inner dimension,
//     C_ij = sum_e A_ik(e) . B_k(e)j = [A_ik1 | A_ik2 | ...] . [B_k1j ; B_k2j ; ...],
// padded to a multiple of 4 once per 64 entries instead of once per entry.
// The product runs as mma.m8n8k4.f64: MF x NF fragments of 8x8 cover the
// M x N output block.  Fragment layouts (PTX ISA, mma.m8n8k4 with .f64):
//   op1 (8x4, row): lane holds op1[lane/4][lane%4]
//   op2 (4x8, col): lane holds op2[lane%4][lane/4]
//   out (8x8):      lane holds out[lane/4][2*(lane%4) + {0,1}]
// Operand fragments are loaded two windows (8 inner columns) ahead of the
// mma that consumes them, and warps take work items in the row processing
// order (Morton / Cuthill-McKee), so that the B rows of neighbouring C rows
// stay resident in L2.
#include "multiply.cuh"

namespace lamb {

constexpr int kNumWarps = 8;
constexpr int kChunk = 64;

struct WarpBuf {
  long long ao[kChunk];
  long long bo[kChunk];
  int pre[kChunk + 1];
};

__device__ __forceinline__ void dmma884(double& c0, double& c1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
               : "+d"(c0), "+d"(c1)
               : "d"(a), "d"(b));
}

// Loads one chunk of <= 64 entries into the warp buffer; returns K (sum of
// inner sizes).  Entries beyond m contribute nothing.
__device__ __forceinline__ int load_chunk(const Ent* __restrict__ ent, int64_t first, int m, WarpBuf& wb,
                                          int lane) {
  Ent x0{0, 0}, x1{0, 0};
  if (lane < m) x0 = ent[first + lane];
  if (lane + 32 < m) x1 = ent[first + lane + 32];
  const int k0 = lane < m ? (int)((unsigned long long)x0.a >> 56) : 0;
  const int k1 = lane + 32 < m ? (int)((unsigned long long)x1.a >> 56) : 0;
  const int i0 = warp_incl_scan(k0, lane);
  const int t0 = __shfl_sync(0xffffffffu, i0, 31);
  const int i1 = warp_incl_scan(k1, lane) + t0;
  wb.ao[lane] = x0.a & kOffMask;
  wb.bo[lane] = x0.b;
  wb.ao[lane + 32] = x1.a & kOffMask;
  wb.bo[lane + 32] = x1.b;
  wb.pre[lane] = i0 - k0;
  wb.pre[lane + 32] = i1 - k1;
  if (lane == 31) wb.pre[kChunk] = i1;
  __syncwarp();
  return wb.pre[kChunk];
}

template <int MF, int NF, bool TA, bool TB>
struct Window {
  double a[MF], b[NF];
  __device__ __forceinline__ void load(const double* __restrict__ d1, const double* __restrict__ d2,
                                       const WarpBuf& wb, int m, int K, int M, int N, int kw, int g, int t, int& e) {
    const int colk = kw + t;
    while (e < m - 1 && colk >= wb.pre[e + 1]) ++e;
    const bool valid = colk < K;
    const int kc = colk - wb.pre[e];
    const int ke = wb.pre[e + 1] - wb.pre[e];
    const double* p1 = d1 + wb.ao[e];
    const double* p2 = d2 + wb.bo[e];
#pragma unroll
    for (int i = 0; i < MF; ++i) {
      const int r = i * 8 + g;
      a[i] = (valid && r < M) ? __ldg(p1 + (TA ? (int64_t)kc + (int64_t)r * ke : (int64_t)r + (int64_t)kc * M)) : 0.0;
    }
#pragma unroll
    for (int j = 0; j < NF; ++j) {
      const int cc = j * 8 + g;
      b[j] = (valid && cc < N) ? __ldg(p2 + (TB ? (int64_t)cc + (int64_t)kc * N : (int64_t)kc + (int64_t)cc * ke)) : 0.0;
    }
  }
};

template <int MF, int NF, bool TA, bool TB>
__device__ __forceinline__ void stacked_block(const double* __restrict__ d1, const double* __restrict__ d2,
                                              double* __restrict__ out, double* __restrict__ out_nrm, int64_t c,
                                              int M, int N, int64_t o_off, int64_t s0, int n,
                                              const Ent* __restrict__ ent, WarpBuf& wb) {
  const int lane = threadIdx.x & 31;
  const int g = lane >> 2, t = lane & 3;
  double acc[MF][NF][2];
#pragma unroll
  for (int i = 0; i < MF; ++i)
#pragma unroll
    for (int j = 0; j < NF; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;
  for (int base = 0; base < n; base += kChunk) {
    const int m = min(kChunk, n - base);
    const int K = load_chunk(ent, s0 + base, m, wb, lane);
    int e = 0;
    Window<MF, NF, TA, TB> w0, w1;
    w0.load(d1, d2, wb, m, K, M, N, 0, g, t, e);
    for (int kw = 0; kw < K; kw += 8) {
      w1.load(d1, d2, wb, m, K, M, N, kw + 4, g, t, e);
#pragma unroll
      for (int i = 0; i < MF; ++i)
#pragma unroll
        for (int j = 0; j < NF; ++j) dmma884(acc[i][j][0], acc[i][j][1], w0.a[i], w0.b[j]);
      w0.load(d1, d2, wb, m, K, M, N, kw + 8, g, t, e);
      if (kw + 4 < K) {
#pragma unroll
        for (int i = 0; i < MF; ++i)
#pragma unroll
          for (int j = 0; j < NF; ++j) dmma884(acc[i][j][0], acc[i][j][1], w1.a[i], w1.b[j]);
      }
    }
    __syncwarp();
  }
  double sq = 0.0;
#pragma unroll
  for (int i = 0; i < MF; ++i)
#pragma unroll
    for (int j = 0; j < NF; ++j)
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int r = i * 8 + g, cc = j * 8 + 2 * t + h;
        if (r < M && cc < N) {
          const double v = acc[i][j][h];
          out[o_off + (int64_t)cc * M + r] = v;
          sq = __fma_rn(v, v, sq);
        }
      }
  sq = warp_sum(sq);
  if (lane == 0 && out_nrm) out_nrm[c] = __dsqrt_rn(sq);
}

// Blocks larger than 24 in a dimension: plain FP64 FMAs, one output element
// per lane and step.
template <bool TA, bool TB>
__device__ void stacked_block_generic(const double* __restrict__ d1, const double* __restrict__ d2,
                                      double* __restrict__ out, double* __restrict__ out_nrm, int64_t c, int M,
                                      int N, int64_t o_off, int64_t s0, int n, const Ent* __restrict__ ent) {
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

template <bool TA, bool TB>
__global__ void __launch_bounds__(kNumWarps * 32, 3)
    k_stacked(int64_t n_work, const Work* __restrict__ work, const int32_t* __restrict__ work_c,
              const Ent* __restrict__ ent, const double* __restrict__ d1, const double* __restrict__ d2,
              double* __restrict__ out, double* __restrict__ out_nrm) {
  __shared__ WarpBuf wbs[kNumWarps];
  const int w = threadIdx.x >> 5;
  WarpBuf& wb = wbs[w];
  const int64_t nwarps = (int64_t)gridDim.x * kNumWarps;
  for (int64_t v = (int64_t)blockIdx.x * kNumWarps + w; v < n_work; v += nwarps) {
    const Work it = work[v];
    const int64_t c = work_c[v];
    const int64_t o_off = it.lo & kMask40;
    const int M = (int)((it.lo >> 40) & 0xff), N = (int)((it.lo >> 48) & 0xff);
    const int64_t s0 = it.hi & kMask40;
    const int n = (int)((unsigned long long)it.hi >> 40);
    const int mf = (M + 7) >> 3, nf = (N + 7) >> 3;
    if (mf == 0 || nf == 0) {
      if ((threadIdx.x & 31) == 0 && out_nrm) out_nrm[c] = 0.0;
      continue;
    }
    switch (mf * 4 + nf) {
      case 1 * 4 + 1: stacked_block<1, 1, TA, TB>(d1, d2, out, out_nrm, c, M, N, o_off, s0, n, ent, wb); break;
      case 1 * 4 + 2: stacked_block<1, 2, TA, TB>(d1, d2, out, out_nrm, c, M, N, o_off, s0, n, ent, wb); break;
      case 1 * 4 + 3: stacked_block<1, 3, TA, TB>(d1, d2, out, out_nrm, c, M, N, o_off, s0, n, ent, wb); break;
      case 2 * 4 + 1: stacked_block<2, 1, TA, TB>(d1, d2, out, out_nrm, c, M, N, o_off, s0, n, ent, wb); break;
      case 2 * 4 + 2: stacked_block<2, 2, TA, TB>(d1, d2, out, out_nrm, c, M, N, o_off, s0, n, ent, wb); break;
      case 2 * 4 + 3: stacked_block<2, 3, TA, TB>(d1, d2, out, out_nrm, c, M, N, o_off, s0, n, ent, wb); break;
      case 3 * 4 + 1: stacked_block<3, 1, TA, TB>(d1, d2, out, out_nrm, c, M, N, o_off, s0, n, ent, wb); break;
      case 3 * 4 + 2: stacked_block<3, 2, TA, TB>(d1, d2, out, out_nrm, c, M, N, o_off, s0, n, ent, wb); break;
      case 3 * 4 + 3: stacked_block<3, 3, TA, TB>(d1, d2, out, out_nrm, c, M, N, o_off, s0, n, ent, wb); break;
      default: stacked_block_generic<TA, TB>(d1, d2, out, out_nrm, c, M, N, o_off, s0, n, ent); break;
    }
  }
}

template <bool TA, bool TB>
static int32_t launch_stacked(Ctx* ctx, int64_t n_work, const Work* work, const int32_t* work_c, const Ent* ent,
                              const double* d1, const double* d2, double* out, double* out_nrm) {
  int sms = 148, per_sm = 1;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx->device);
  LAMB_CUDA(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_stacked<TA, TB>, kNumWarps * 32, 0));
  const int64_t need = (n_work + kNumWarps - 1) / kNumWarps;
  const int grid = (int)std::max<int64_t>(1, std::min<int64_t>(need, (int64_t)sms * std::max(per_sm, 1)));
  k_stacked<TA, TB><<<grid, kNumWarps * 32, 0, ctx->stream>>>(n_work, work, work_c, ent, d1, d2, out, out_nrm);
  LAMB_LAUNCHED(ctx);
  return LAMB_GPU_OK;
}

int32_t run_stacked(Ctx* ctx, int64_t n_work, const Work* work, const int32_t* work_c, const Ent* ent,
                    const double* d1, const double* d2, double* out, double* out_nrm, bool t1, bool t2) {
  if (n_work == 0) return LAMB_GPU_OK;
  if (!t1 && !t2) return launch_stacked<false, false>(ctx, n_work, work, work_c, ent, d1, d2, out, out_nrm);
  if (!t1 && t2) return launch_stacked<false, true>(ctx, n_work, work, work_c, ent, d1, d2, out, out_nrm);
  if (t1 && !t2) return launch_stacked<true, false>(ctx, n_work, work, work_c, ent, d1, d2, out, out_nrm);
  return fail(ctx, LAMB_LEVEL_FAILURE, LAMB_TYPE_INTERNAL_ERROR, "unsupported operand transposition");
}

}  // namespace lamb
