// Mixed-precision numeric phase: FP64 block products as exact int8 slice
// products on the tensor cores with FP64 recombination (the split-and-sum
// scheme of Ozaki, Ogita, Oishi and Rump, Numer. Algorithms 59 (2012), with
// int8 digits).  No reference counterpart.
//
// Every element row r of A gets a power-of-two scale 2^ea_r >= max_k |A(r,k)|
// and every element column c of B a scale 2^eb_c >= max_k |B(k,c)|.  A scaled
// value x in [-1, 1] is written as x = sum_p d_p w_p + rest with integer
// digits d_p in [-64, 64], w_1 = 2^-6 and w_p = 2^-6-7(p-1) (each digit takes
// the next 7 bits; |rest| <= w_s / 2).  Then
//   C(r,c) = 2^(ea_r + eb_c) * sum_{p+q <= s+1} w_p w_q (D_p . E_q)(r,c),
// where D_p, E_q are the digit planes of A and B.  Each plane product is an
// exact int32 sum (|d| <= 64, so 2^19 inner terms fit) computed with
// mma.m16n8k32 .s8.s8.s32; the recombination runs in FP64.  Pairs with
// p + q > s+1 are dropped: their weight is below 2^-(12+7s).
//
// Plane layout: A block (M x ke) as M rows of pad4(ke) inner indices, B block
// (ke x N) as N columns of pad4(ke) inner indices; every 32-bit word holds
// four consecutive inner indices of one row (A) or one column (B) of one
// digit plane -- the operand words of the m16n8k32 fragments -- and the
// words of all 8 planes (planes >= s are zero) of one (row, word) position
// are interleaved in 32 bytes, so one lane fetches every plane of its
// fragment word with two 16-byte loads:
//   byte(row ln, inner kc, plane p) = 8*soff + (ln*pad4(ke)/4 + kc/4)*32 + 4p + kc%4
// (soff: the block's offset in a single plane).  Fragment words:
//   op1 a0,a1,a2,a3 = words (g, t), (g+8, t), (g, 4+t), (g+8, 4+t)
//   op2 b0,b1       = words (col g, t), (col g, 4+t)
//   out c0..c3      = (g, 2t), (g, 2t+1), (g+8, 2t), (g+8, 2t+1)
// with g = lane/4, t = lane%4 (PTX ISA fragment layout of mma.m16n8k32 for
// 8-bit integer types).
#include <cub/cub.cuh>

#include <algorithm>
#include <climits>
#include <cstdlib>

#include "algebra.cuh"
#include "multiply.cuh"

namespace lamb {

constexpr int kMixWarps = 4;
constexpr int kMaxSlices = 8;
// Largest inner length (bytes of a padded plane row) for which the level
// accumulators of 7 slices stay exact: 7 products of |digit| <= 64 per index.
constexpr int64_t kLevelInnerMax7 = (int64_t)INT_MAX / (7 * 64 * 64);

__device__ __forceinline__ int pad4(int x) { return (x + 3) & ~3; }

// ---- scales ----------------------------------------------------------------------------
// Row exponents of A: one CTA per block row, its warps taking every 8th
// block of the row (memory parallelism across the row's blocks).  For
// bi <= 32 lane l keeps the running max of element row l % bi over the
// columns l / bi, l / bi + 32 / bi, ... of its blocks; all lanes of one
// element row then merge through a shared-memory atomic max (non-negative
// doubles order like their bit patterns).  Larger blocks merge every element.
__global__ void k_row_exp(int32_t n_rows, const int64_t* __restrict__ row_p, const int32_t* __restrict__ col,
                          const int64_t* __restrict__ off, const int8_t* __restrict__ row_bs,
                          const int8_t* __restrict__ col_bs, const double* __restrict__ d,
                          const int64_t* __restrict__ ebase, int* __restrict__ ea) {
  __shared__ unsigned long long pm[128];
  const int lane = threadIdx.x & 31, wl = threadIdx.x >> 5, nwl = blockDim.x >> 5;
  for (int64_t r = blockIdx.x; r < n_rows; r += gridDim.x) {
    const int bi = row_bs[r];
    for (int p = threadIdx.x; p < bi; p += blockDim.x) pm[p] = 0ull;
    __syncthreads();
    if (bi <= 32) {
      const int G = 32 / bi, pe = lane % bi, g = lane / bi;
      double m = 0.0;
      if (g < G)
        for (int64_t b = row_p[r] + wl; b < row_p[r + 1]; b += nwl) {
          const int bk = col_bs[col[b]];
          const double* x = d + off[b];
#pragma unroll 4
          for (int kc = g; kc < bk; kc += G) m = fmax(m, fabs(x[pe + kc * bi]));
        }
      if (g < G) atomicMax(&pm[pe], (unsigned long long)__double_as_longlong(m));
    } else {
      for (int64_t b = row_p[r] + wl; b < row_p[r + 1]; b += nwl) {
        const int ne = bi * col_bs[col[b]];
        const double* x = d + off[b];
        Walk w(bi, lane);
        for (int e = lane; e < ne; e += 32, w.next())
          atomicMax(&pm[w.minor], (unsigned long long)__double_as_longlong(fabs(x[e])));
      }
    }
    __syncthreads();
    for (int p = threadIdx.x; p < bi; p += blockDim.x) {
      int e = 0;
      frexp(__longlong_as_double((long long)pm[p]), &e);
      ea[ebase[r] + p] = e;
    }
    __syncthreads();
  }
}

// Column exponents of B: one CTA per block row, its warps taking every 8th
// block of the row.  For bj <= 32 lane l keeps the max of element column
// l % bj over the rows l / bj, l / bj + 32 / bj, ...; the lanes of one
// column merge through a shared-memory atomic max, then one global atomic
// max per block column element.
__global__ void k_col_exp(int32_t n_rows, const int64_t* __restrict__ row_p, const int32_t* __restrict__ col,
                          const int64_t* __restrict__ off, const int8_t* __restrict__ row_bs,
                          const int8_t* __restrict__ col_bs, const double* __restrict__ d,
                          const int64_t* __restrict__ ebase, int* __restrict__ eb) {
  __shared__ unsigned long long cm[8][128];
  const int lane = threadIdx.x & 31, wl = threadIdx.x >> 5, nwl = blockDim.x >> 5;
  for (int64_t r = blockIdx.x; r < n_rows; r += gridDim.x) {
    const int bk = row_bs[r];
    for (int64_t b = row_p[r] + wl; b < row_p[r + 1]; b += nwl) {
      const int j = col[b], bj = col_bs[j];
      const double* x = d + off[b];
      for (int c = lane; c < bj; c += 32) cm[wl][c] = 0ull;
      __syncwarp();
      if (bj <= 32) {
        const int H = 32 / bj, c = lane % bj, h = lane / bj;
        if (h < H) {
          double m = 0.0;
#pragma unroll 4
          for (int kr = h; kr < bk; kr += H) m = fmax(m, fabs(x[kr + c * bk]));
          atomicMax(&cm[wl][c], (unsigned long long)__double_as_longlong(m));
        }
      } else {
        Walk w(bj, lane);
        for (int e = lane; e < bk * bj; e += 32, w.next())
          atomicMax(&cm[wl][w.minor], (unsigned long long)__double_as_longlong(fabs(x[w.major + w.minor * bk])));
      }
      __syncwarp();
      for (int c = lane; c < bj; c += 32) {
        int e = 0;
        frexp(__longlong_as_double((long long)cm[wl][c]), &e);
        atomicMax(&eb[ebase[j] + c], e);
      }
      __syncwarp();
    }
  }
}

// Plane block sizes: A block (M x ke) -> M*pad4(ke); B block (ke x N) -> N*pad4(ke).
__global__ void k_plane_sizes(int32_t n_rows, const int64_t* __restrict__ row_p, const int32_t* __restrict__ col,
                              const int8_t* __restrict__ row_bs, const int8_t* __restrict__ col_bs, int a_side,
                              int64_t* __restrict__ sz) {
  for (int64_t r = global_warp(); r < n_rows; r += grid_warps())
    for (int64_t b = row_p[r] + (threadIdx.x & 31); b < row_p[r + 1]; b += 32) {
      const int rb = row_bs[r], cb = col_bs[col[b]];
      sz[b] = a_side ? (int64_t)rb * pad4(cb) : (int64_t)cb * pad4(rb);
    }
}

// Digits of one block into the interleaved planes.  a_side: line p holds
// x(p, kc) = A(p,kc) 2^-ea_p; else line c holds x(c, kc) = B(kc,c) 2^-eb_c.
__global__ void k_digits(int32_t n_rows, const int64_t* __restrict__ row_p, const int32_t* __restrict__ col,
                         const int64_t* __restrict__ off, const int8_t* __restrict__ row_bs,
                         const int8_t* __restrict__ col_bs, const double* __restrict__ d,
                         const int64_t* __restrict__ rbase, const int64_t* __restrict__ cbase,
                         const int* __restrict__ e_row, const int* __restrict__ e_col, int a_side,
                         const int64_t* __restrict__ soff, int s, int8_t* __restrict__ planes) {
  const int lane = threadIdx.x & 31;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t r = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; r < n_rows; r += nw) {
    const int rb = row_bs[r];
    for (int64_t b = row_p[r]; b < row_p[r + 1]; ++b) {
      const int j = col[b], cb = col_bs[j];
      const double* x = d + off[b];
      const int lines = a_side ? rb : cb;  // stored rows
      const int ke = a_side ? cb : rb;     // inner size
      const int kp = pad4(ke);
      // one lane per (line, word): 4 inner indices x 8 planes = 32 bytes, two 16-byte stores
      const int nwl = kp >> 2;
      for (int e = lane; e < lines * nwl; e += 32) {
        const int ln = e / nwl, w = e % nwl;
        const int e_sc = a_side ? e_row[rbase[r] + ln] : e_col[cbase[j] + ln];
        unsigned word[kMaxSlices];
#pragma unroll
        for (int p = 0; p < kMaxSlices; ++p) word[p] = 0u;
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          const int kc = 4 * w + q;
          double v = 0.0;
          if (kc < ke) v = ldexp(a_side ? x[(int64_t)kc * rb + ln] : x[(int64_t)ln * rb + kc], -e_sc);
          // digits: 2^6 v, then 7 bits per step; every step is exact in FP64
          double t = ldexp(v, 6);
#pragma unroll
          for (int p = 0; p < kMaxSlices; ++p) {
            const double dg = p < s ? rint(t) : 0.0;
            word[p] |= (unsigned)(uint8_t)(int8_t)dg << (8 * q);
            t = ldexp(t - dg, 7);
          }
        }
        int4* dst = reinterpret_cast<int4*>(planes + 8 * soff[b] + ((int64_t)ln * nwl + w) * 32);
        dst[0] = make_int4((int)word[0], (int)word[1], (int)word[2], (int)word[3]);
        dst[1] = make_int4((int)word[4], (int)word[5], (int)word[6], (int)word[7]);
      }
    }
  }
}

// ---- numeric kernel ---------------------------------------------------------------------
struct WordRef {
  const int4* pa;           // A word group (row 0, this word): 8 plane words, 32 bytes
  unsigned long long pbk;   // B word group (column 0, this word) | row stride in int4 units << 56
};

__device__ __forceinline__ void imma16832(int (&c)[4], const int (&a)[4], const int (&b)[2]) {
  asm volatile(
      "mma.sync.aligned.m16n8k32.row.col.s32.s8.s8.s32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};"
      : "+r"(c[0]), "+r"(c[1]), "+r"(c[2]), "+r"(c[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

// Word table of one chunk: the word groups of every entry's blocks, concatenated.
__device__ __forceinline__ int build_words(const int4* __restrict__ pa0, const int4* __restrict__ pb0,
                                           const Ent* __restrict__ ent, int64_t first, int m,
                                           WordRef* __restrict__ tbl, int lane) {
  Ent x{0, 0};
  if (lane < m) x = ent[first + lane];
  const int ke = lane < m ? (int)((unsigned long long)x.a >> 56) : 0;
  const int nw = (ke + 3) >> 2;
  const int incl = warp_incl_scan(nw, lane);
  const int W = __shfl_sync(0xffffffffu, incl, 31);
  // 8 * soff bytes = soff / 2 int4 (soff is a multiple of 4)
  const int4* pa = pa0 + ((x.a & kOffMask) >> 1);
  const int4* pb = pb0 + (x.b >> 1);
  const unsigned long long sb = (unsigned long long)(2 * nw) << 56;
  for (int w = 0, k = incl - nw; w < nw; ++w, ++k)
    tbl[k] = WordRef{pa + 2 * w, (unsigned long long)(pb + 2 * w) | sb};
  __syncwarp();
  return W;
}

// The 8 plane words of one fragment word (two 16-byte loads), zero when absent.
__device__ __forceinline__ void ld_group(const int4* p, bool ok, int (&w)[8]) {
  int4 lo = make_int4(0, 0, 0, 0), hi = make_int4(0, 0, 0, 0);
  if (ok) {
    lo = __ldg(p);
    hi = __ldg(p + 1);
  }
  w[0] = lo.x; w[1] = lo.y; w[2] = lo.z; w[3] = lo.w;
  w[4] = hi.x; w[5] = hi.y; w[6] = hi.z; w[7] = hi.w;
}

// Fragment words of one 8-word window for every plane: op1 (16 tile rows:
// A rows, or B columns when SWAP) and op2 (8 tile columns).
template <bool SWAP>
__device__ __forceinline__ void load_window(const WordRef* __restrict__ tbl, int W, int w0, int t, int ra, int rb,
                                            int cc, bool ok_a, bool ok_b, bool ok_c, int (&a)[4][8],
                                            int (&bw)[2][8]) {
  const int wa = w0 + t, wb = w0 + 4 + t;
  const bool va = wa < W, vb = wb < W;
  const WordRef ta = tbl[va ? wa : 0], tb = tbl[vb ? wb : 0];
  const int sa = (int)(ta.pbk >> 56), sbw = (int)(tb.pbk >> 56);
  const int4* pba = reinterpret_cast<const int4*>(ta.pbk & kOffMask);
  const int4* pbb = reinterpret_cast<const int4*>(tb.pbk & kOffMask);
  const int4* o1a = SWAP ? pba : ta.pa;
  const int4* o1b = SWAP ? pbb : tb.pa;
  const int4* o2a = SWAP ? ta.pa : pba;
  const int4* o2b = SWAP ? tb.pa : pbb;
  ld_group(o1a + (int64_t)ra * sa, va && ok_a, a[0]);
  ld_group(o1a + (int64_t)rb * sa, va && ok_b, a[1]);
  ld_group(o1b + (int64_t)ra * sbw, vb && ok_a, a[2]);
  ld_group(o1b + (int64_t)rb * sbw, vb && ok_b, a[3]);
  ld_group(o2a + (int64_t)cc * sa, va && ok_c, bw[0]);
  ld_group(o2b + (int64_t)cc * sbw, vb && ok_c, bw[1]);
}

// 16 tile rows (r0..) x 8 tile columns (c0..) of one C block, any s <= 8
// slices, one int32 accumulator per digit pair and table chunk, added into
// the FP64 result after every chunk (a chunk has at most 4,096 inner
// indices; an int32 sum of |digit| <= 64 products is exact up to 2^19), so
// stacks of any length stay exact.  SWAP: tile rows are the block's columns
// (B side), tile columns the block's rows (A side).
template <bool SWAP>
__device__ __forceinline__ void mixed_tile(const int4* __restrict__ pa0, const int4* __restrict__ pb0, int s,
                                           const Ent* __restrict__ ent, int64_t s0, int n, int cap,
                                           WordRef* __restrict__ tbl, int TM, int TN, int r0, int c0,
                                           double (&out)[4]) {
  const int lane = threadIdx.x & 31;
  const int g = lane >> 2, t = lane & 3;
  const int ra = r0 + g, rb = r0 + g + 8, cc = c0 + g;
  const bool ok_a = ra < TM, ok_b = rb < TM, ok_c = cc < TN;
#pragma unroll
  for (int h = 0; h < 4; ++h) out[h] = 0.0;
  for (int p = 0; p < s; ++p) {
    for (int base = 0; base < n; base += cap) {
      int acc[kMaxSlices][4];
#pragma unroll
      for (int q = 0; q < kMaxSlices; ++q)
#pragma unroll
        for (int h = 0; h < 4; ++h) acc[q][h] = 0;
      const int m = min(cap, n - base);
      const int W = build_words(pa0, pb0, ent, s0 + base, m, tbl, lane);
      for (int w0 = 0; w0 < W; w0 += 8) {
        int aw[4][8], bw[2][8];
        load_window<SWAP>(tbl, W, w0, t, ra, rb, cc, ok_a, ok_b, ok_c, aw, bw);
        int a[4];
#pragma unroll
        for (int pp = 0; pp < kMaxSlices; ++pp)
          if (pp == p) { a[0] = aw[0][pp]; a[1] = aw[1][pp]; a[2] = aw[2][pp]; a[3] = aw[3][pp]; }
#pragma unroll
        for (int q = 0; q < kMaxSlices; ++q)
          if (q < s - p) {
            const int bq[2] = {bw[0][q], bw[1][q]};
            imma16832(acc[q], a, bq);
          }
      }
      __syncwarp();
      // flushed per chunk: a chunk has at most cap x 128 inner indices
#pragma unroll
      for (int q = 0; q < kMaxSlices; ++q)
        if (q < s - p) {
          const int sh = -12 - 7 * (p + q);
#pragma unroll
          for (int h = 0; h < 4; ++h) out[h] += ldexp((double)acc[q][h], sh);
        }
    }
  }
}

// One 16 x 8 tile for S digits with one int32 accumulator per weight level
// d = p + q (every pair of a level has the weight 2^(-12-7d)).  A level sums
// at most S products of |digit| <= 64 per inner index, so it stays exact while
// the tile's inner length is at most (2^31 - 1) / (S * 4096) (74,898 for
// S = 7); callers check that bound.  Per window of 8 words every plane of
// both operands is loaded once (12 16-byte loads per lane) and all
// S(S+1)/2 pairs run.
template <int S, bool SWAP>
__device__ __forceinline__ void mixed_tile_levels(const int4* __restrict__ pa0, const int4* __restrict__ pb0,
                                                  const Ent* __restrict__ ent, int64_t s0, int n, int cap,
                                                  WordRef* __restrict__ tbl, int TM, int TN, int r0, int c0,
                                                  double (&out)[4]) {
  const int lane = threadIdx.x & 31;
  const int g = lane >> 2, t = lane & 3;
  const int ra = r0 + g, rb = r0 + g + 8, cc = c0 + g;
  const bool ok_a = ra < TM, ok_b = rb < TM, ok_c = cc < TN;
  int acc[S][4];
#pragma unroll
  for (int d = 0; d < S; ++d)
#pragma unroll
    for (int h = 0; h < 4; ++h) acc[d][h] = 0;
  for (int base = 0; base < n; base += cap) {
    const int m = min(cap, n - base);
    const int W = build_words(pa0, pb0, ent, s0 + base, m, tbl, lane);
    for (int w0 = 0; w0 < W; w0 += 8) {
      int aw[4][8], bw[2][8];
      load_window<SWAP>(tbl, W, w0, t, ra, rb, cc, ok_a, ok_b, ok_c, aw, bw);
#pragma unroll
      for (int p = 0; p < S; ++p) {
        const int a[4] = {aw[0][p], aw[1][p], aw[2][p], aw[3][p]};
#pragma unroll
        for (int q = 0; q < S - p; ++q) {
          const int bq[2] = {bw[0][q], bw[1][q]};
          imma16832(acc[p + q], a, bq);
        }
      }
    }
    __syncwarp();
  }
#pragma unroll
  for (int h = 0; h < 4; ++h) {
    double v = 0.0;
#pragma unroll
    for (int d = S - 1; d >= 0; --d) v += ldexp((double)acc[d][h], -12 - 7 * d);
    out[h] = v;
  }
}

// Five CTAs per SM (96 registers a thread, a small spill) run the 6,144-water
// multiply 1.8 % faster than the 128-register build at four.
__global__ void __launch_bounds__(kMixWarps * 32, 5) k_mixed(
    int64_t n_work, const Work* __restrict__ work, const int32_t* __restrict__ work_c,
    const int32_t* __restrict__ c_row, const int32_t* __restrict__ c_col, const Ent* __restrict__ ent,
    const int4* __restrict__ pa0, const int4* __restrict__ pb0, int s,
    const int64_t* __restrict__ rbase, const int64_t* __restrict__ cbase, const int* __restrict__ ea,
    const int* __restrict__ eb, double* __restrict__ out, double* __restrict__ out_nrm, int cap, int tbl_words,
    int kmax4, unsigned long long* __restrict__ head) {
  extern __shared__ WordRef wtbl[];
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int g = lane >> 2, t = lane & 3;
  WordRef* tbl = wtbl + (size_t)w * tbl_words;
  while (true) {
    unsigned long long vv = 0;
    if (lane == 0) vv = atomicAdd(head, 1ull);
    vv = __shfl_sync(0xffffffffu, vv, 0);
    if (vv >= (unsigned long long)n_work) break;
    const int64_t v = (int64_t)vv;
    const Work it = work[v];
    const int64_t c = work_c[v];
    const int64_t o_off = it.lo & kMask40;
    const int M = (int)((it.lo >> 40) & 0xff), N = (int)((it.lo >> 48) & 0xff);
    const int64_t s0 = it.hi & kMask40;
    const int n = (int)((unsigned long long)it.hi >> 40);
    const int64_t rb0 = rbase[c_row[c]], cb0 = cbase[c_col[c]];
    const bool swap = M <= 8 && N > 8;
    const int TM = swap ? N : M, TN = swap ? M : N;
    double sq = 0.0;
    for (int r0 = 0; r0 < TM; r0 += 16)
      for (int c0 = 0; c0 < TN; c0 += 8) {
        double o[4];
        if (s == 7 && (int64_t)n * kmax4 <= kLevelInnerMax7) {
          if (swap)
            mixed_tile_levels<7, true>(pa0, pb0, ent, s0, n, cap, tbl, TM, TN, r0, c0, o);
          else
            mixed_tile_levels<7, false>(pa0, pb0, ent, s0, n, cap, tbl, TM, TN, r0, c0, o);
        } else if (swap) {
          mixed_tile<true>(pa0, pb0, s, ent, s0, n, cap, tbl, TM, TN, r0, c0, o);
        } else {
          mixed_tile<false>(pa0, pb0, s, ent, s0, n, cap, tbl, TM, TN, r0, c0, o);
        }
#pragma unroll
        for (int h = 0; h < 4; ++h) {
          const int tr = r0 + g + 8 * (h >> 1), tc = c0 + 2 * t + (h & 1);
          if (tr < TM && tc < TN) {
            const int r = swap ? tc : tr, cl = swap ? tr : tc;
            const double val = ldexp(o[h], ea[rb0 + r] + eb[cb0 + cl]);
            out[o_off + (int64_t)cl * M + r] = val;
            sq = __fma_rn(val, val, sq);
          }
        }
      }
    sq = warp_sum(sq);
    if (lane == 0 && out_nrm) out_nrm[c] = __dsqrt_rn(sq);
  }
}

// ---- host side ----------------------------------------------------------------------------
int mixed_slices_from_env() {
  const char* v = getenv("LAMB_GPU_MIXED_SLICES");
  int s = v ? atoi(v) : 7;
  return std::max(2, std::min(s, kMaxSlices));
}

static std::vector<int64_t> elem_base(const std::vector<int8_t>& bs) {
  std::vector<int64_t> b(bs.size() + 1, 0);
  for (size_t i = 0; i < bs.size(); ++i) b[i + 1] = b[i] + bs[i];
  return b;
}

int32_t build_slices(Ctx* ctx, const DevMatrix* A, const DevMatrix* B, int s, MixedPlanes* mp, bool exps_only) {
  if (max_block(A->h_row_bs) > 127 || max_block(B->h_col_bs) > 127)
    return fail(ctx, LAMB_LEVEL_FAILURE, LAMB_TYPE_UNIMPLEMENTED, "mixed: block too large");
  static_assert(kThreads <= 256, "k_col_exp keeps 8 warps x 128 columns of maxima in shared memory");
  mp->s = s;
  const auto ra = elem_base(A->h_row_bs), cbv = elem_base(B->h_col_bs);
  LAMB_TRY(dalloc(ctx, &mp->rbase, (int64_t)ra.size()));
  LAMB_TRY(dalloc(ctx, &mp->cbase, (int64_t)cbv.size()));
  LAMB_CUDA(ctx, cudaMemcpyAsync(mp->rbase, ra.data(), sizeof(int64_t) * ra.size(), cudaMemcpyHostToDevice, ctx->stream));
  LAMB_CUDA(ctx, cudaMemcpyAsync(mp->cbase, cbv.data(), sizeof(int64_t) * cbv.size(), cudaMemcpyHostToDevice, ctx->stream));
  LAMB_TRY(dalloc(ctx, &mp->ea, std::max<int64_t>(ra.back(), 1)));
  LAMB_TRY(dalloc(ctx, &mp->eb, std::max<int64_t>(cbv.back(), 1)));
  // eb starts at 0x80808080 (byte fill), below any frexp exponent, for the atomic max
  LAMB_CUDA(ctx, cudaMemsetAsync(mp->eb, 0x80, sizeof(int) * std::max<int64_t>(cbv.back(), 1), ctx->stream));
  if (A->nnz) {
    k_row_exp<<<grid_for((int64_t)A->n_rows * kThreads), kThreads, 0, ctx->stream>>>(
        A->n_rows, A->row_p, A->col, A->off, A->row_bs, A->col_bs, A->data, mp->rbase, mp->ea);
    LAMB_LAUNCHED(ctx);
  }
  if (B->nnz) {
    k_col_exp<<<grid_for((int64_t)B->n_rows * kThreads), kThreads, 0, ctx->stream>>>(
        B->n_rows, B->row_p, B->col, B->off, B->row_bs, B->col_bs, B->data, mp->cbase, mp->eb);
    LAMB_LAUNCHED(ctx);
  }
  trace_mark(ctx, "slice exponents");
  if (exps_only) return LAMB_GPU_OK;
  // plane offsets
  int64_t* sz = nullptr;
  LAMB_TRY(dalloc(ctx, &mp->a_soff, std::max<int64_t>(A->nnz, 1) + 1));
  LAMB_TRY(dalloc(ctx, &mp->b_soff, std::max<int64_t>(B->nnz, 1) + 1));
  LAMB_TRY(dalloc(ctx, &sz, std::max(A->nnz, B->nnz) + 1));
  auto plane = [&](const DevMatrix* m, int a_side, int64_t* soff, int64_t* bytes) -> int32_t {
    LAMB_CUDA(ctx, cudaMemsetAsync(sz + m->nnz, 0, sizeof(int64_t), ctx->stream));
    if (m->nnz) {
      k_plane_sizes<<<grid_for(32ll * m->n_rows, 256), 256, 0, ctx->stream>>>(m->n_rows, m->row_p, m->col, m->row_bs,
                                                                         m->col_bs, a_side, sz);
      LAMB_LAUNCHED(ctx);
    }
    LAMB_TRY(exclusive_scan_i64(ctx, sz, soff, m->nnz + 1));
    LAMB_CUDA(ctx, cudaMemcpyAsync(bytes, soff + m->nnz, sizeof(int64_t), cudaMemcpyDeviceToHost, ctx->stream));
    LAMB_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    *bytes = std::max<int64_t>((*bytes + 15) & ~15ll, 16);
    return LAMB_GPU_OK;
  };
  LAMB_TRY(plane(A, 1, mp->a_soff, &mp->a_plane));
  LAMB_TRY(plane(B, 0, mp->b_soff, &mp->b_plane));
  dfree(ctx, sz);
  trace_mark(ctx, "plane sizes");
  // 8 interleaved planes (those >= s are zero): 8 bytes per element
  LAMB_TRY(scratch(ctx, kScrPlaneA, mp->a_plane * kMaxSlices, &mp->a_planes));
  LAMB_TRY(scratch(ctx, kScrPlaneB, mp->b_plane * kMaxSlices, &mp->b_planes));
  if (A->nnz) {
    k_digits<<<grid_for((int64_t)A->n_rows * 32), kThreads, 0, ctx->stream>>>(
        A->n_rows, A->row_p, A->col, A->off, A->row_bs, A->col_bs, A->data, mp->rbase, nullptr, mp->ea, nullptr, 1,
        mp->a_soff, s, mp->a_planes);
    LAMB_LAUNCHED(ctx);
  }
  if (B->nnz) {
    k_digits<<<grid_for((int64_t)B->n_rows * 32), kThreads, 0, ctx->stream>>>(
        B->n_rows, B->row_p, B->col, B->off, B->row_bs, B->col_bs, B->data, nullptr, mp->cbase, nullptr, mp->eb, 0,
        mp->b_soff, s, mp->b_planes);
    LAMB_LAUNCHED(ctx);
  }
  return LAMB_GPU_OK;
}

void free_slices(Ctx* ctx, MixedPlanes* mp) {
  dfree(ctx, mp->rbase); dfree(ctx, mp->cbase); dfree(ctx, mp->ea); dfree(ctx, mp->eb);
  dfree(ctx, mp->a_soff); dfree(ctx, mp->b_soff);
  mp->a_planes = mp->b_planes = nullptr;  // context scratch
}

// (plane offset | inner size << 56) for every A block; plane offsets of B.
__global__ void k_pack_plane_meta(int32_t n_rows, const int64_t* __restrict__ row_p, const int32_t* __restrict__ col,
                                  const int8_t* __restrict__ col_bs, const int64_t* __restrict__ soff,
                                  int64_t* __restrict__ out) {
  for (int64_t r = global_warp(); r < n_rows; r += grid_warps())
    for (int64_t b = row_p[r] + (threadIdx.x & 31); b < row_p[r + 1]; b += 32)
      out[b] = soff[b] | ((int64_t)col_bs[col[b]] << 56);
}

int32_t pack_plane_meta(Ctx* ctx, const DevMatrix* A, const MixedPlanes& mp, int64_t** a_meta) {
  LAMB_TRY(dalloc(ctx, a_meta, std::max<int64_t>(A->nnz, 1)));
  if (A->nnz) {
    k_pack_plane_meta<<<grid_for(32ll * A->n_rows, 256), 256, 0, ctx->stream>>>(A->n_rows, A->row_p, A->col, A->col_bs,
                                                                           mp.a_soff, *a_meta);
    LAMB_LAUNCHED(ctx);
  }
  return LAMB_GPU_OK;
}

int32_t numeric_mixed(Ctx* ctx, DevMatrix* A, DevMatrix* B, DevMatrix* C, const Symbolic& sym, const Work* work,
                      const int32_t* work_c, double* c_nrm, const MixedPlanes& mp) {
  if (sym.c_nnz == 0) return LAMB_GPU_OK;
  const int mi = std::max(1, std::min(max_block(A->h_col_bs), 127));
  const int wpe = (mi + 3) / 4;  // words per entry at most
  const int cap = std::max(1, std::min(32, 4096 / wpe));
  const int tbl_words = cap * wpe;
  const size_t smem = sizeof(WordRef) * (size_t)tbl_words * kMixWarps;
  if (smem > 48 * 1024)
    LAMB_CUDA(ctx, cudaFuncSetAttribute(k_mixed, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  int sms = 148, per_sm = 1;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx->device);
  LAMB_CUDA(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_mixed, kMixWarps * 32, smem));
  const int64_t need = (sym.c_nnz + kMixWarps - 1) / kMixWarps;
  const int grid = (int)std::max<int64_t>(1, std::min<int64_t>(need, (int64_t)sms * std::max(per_sm, 1)));
  unsigned long long* head = nullptr;
  LAMB_TRY(dalloc(ctx, &head, 1));
  LAMB_CUDA(ctx, cudaMemsetAsync(head, 0, sizeof(unsigned long long), ctx->stream));
  k_mixed<<<grid, kMixWarps * 32, smem, ctx->stream>>>(
      sym.c_nnz, work, work_c, sym.c_row, C->col, sym.ent, reinterpret_cast<const int4*>(mp.a_planes),
      reinterpret_cast<const int4*>(mp.b_planes), mp.s, mp.rbase, mp.cbase, mp.ea,
      mp.eb, C->data, c_nrm, cap, tbl_words, 4 * wpe, head);
  LAMB_LAUNCHED(ctx);
  dfree(ctx, head);
  return LAMB_GPU_OK;
}

}  // namespace lamb
