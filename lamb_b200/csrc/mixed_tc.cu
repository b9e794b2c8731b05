// Mixed-precision numeric phase on the 5th-generation tensor cores
// (tcgen05.mma kind::i8, accumulators in tensor memory).  No reference
// counterpart: the reference's sector_multiply (src/lamb_multiplication.F90:
// 206-225) is a stub; this computes the same C = A.B as the FP64 path from
// exact int8 digit products (the split-and-sum idea of Ozaki, Ogita, Oishi
// and Rump, Numer. Algorithms 59 (2012), with fixed-point int8 digits).
//
// Digits.  Every element row r of A gets a power-of-two scale 2^ea_r >=
// max_k |A(r,k)|, every element column c of B 2^eb_c >= max_k |B(k,c)|; a
// scaled value x in (-1, 1) is written x = sum_p d_p / (127 * 254^p) + rest
// with integer digits |d_p| <= 127 (t = 127 x; d_p = rint(t);
// t = 254 (t - d_p)), i.e. almost 8 bits a digit: six digits carry 47 bits.
// For S digits,
//   C(r,c) = 2^(ea_r + eb_c) sum_{L=0}^{S-1} sum_{p+q=L} (D_p E_q)(r,c) / (127^2 254^L),
// every D_p E_q is an exact int32 sum (S * 127^2 per inner index keeps
// 22,190 inner indices exact for S = 6), and the recombination runs in FP64.
// Pairs with p + q >= S are dropped (weight below 127^-2 254^-S).
//
// Tiles.  Block rows are too small for tcgen05 (M = 128), so the multiply is
// done on spatial clusters: row atoms (in the row processing order, a Morton
// curve over the atoms' coordinates) are cut into clusters of at most 128
// rows, column atoms into clusters of at most 64 columns.  A cluster pair
// (I, J) holding at least one C block is one tile; its inner dimension is the
// concatenation of every inner atom k that couples to both clusters (some
// A_ik with i in I and some B_kj with j in J), so only M and N are padded.
// Operands live in "panels" built once per multiply: for row cluster I and
// every inner atom k it touches, b_k panel rows of 128 bytes (the cluster's
// rows, zero where A_ik is absent), one array per digit plane; B likewise
// with 64-byte rows.  A K-row of a tile is thus one 128-byte A panel row and
// one 64-byte B panel row, which the producer warps gather into shared memory
// (cp.async, 16 bytes a thread) in the canonical MN-major layouts of UMMA
// (128B swizzle for A, 64B swizzle for B).  Products that the product filter
// would skip are included (they are bounded by eps each); the C pattern is
// the filtered one, so only C blocks of the pattern are written.
//
// Kernel roles (one CTA of 352 threads per SM, persistent over the tiles):
//   warps 0-5  producers: gather the tile's K rows, 32 per pipeline stage
//              (four warps the A chunks, two warps the B chunks);
//   warp 6     loads each tile's inner-atom list one tile ahead, allocates
//              the tensor memory (6 levels x 64 columns in 512) and from one
//              lane issues nine MMAs (M=128, K=32, N=64..256) per stage,
//              one per A digit plane and run of up to four B digit planes;
//   warps 7-10 epilogue: tensor memory -> FP64 staging tile in shared
//              memory (the six levels of a column recombined exactly in two
//              int64 sums), then column scaling and per-row partial sums of
//              squares per column atom; every C block of the tile copied out
//              in its storage order (contiguous stores, one warp a block)
//              and its norm summed from the row partials.  The tile's block
//              list (built before the kernel) and exponents are loaded one
//              tile ahead into registers.
// Every wait on an mbarrier is bounded (2 s of %globaltimer); on a timeout
// the kernel records an error code, every role stops, and the host returns
// an error status.
#include <cub/cub.cuh>

#include <algorithm>
#include <climits>
#include <numeric>

#include "lamb_probe.h"
#include "multiply.cuh"

namespace lamb {
namespace tc {

constexpr int kS = 6;                 // digits per operand
constexpr int kM = 128, kN = 64, kK = 32;
constexpr int kStages = 3;
constexpr int kPlaneA = kK * kM;      // bytes of one digit plane of one stage (A)
constexpr int kPlaneB = kK * kN;
constexpr int kStageA = kS * kPlaneA;
constexpr int kStageB = kS * kPlaneB;
constexpr int kStageBytes = kStageA + kStageB;  // 36,864: a multiple of 1,024
constexpr int kMaxEnt = 1024;         // inner-list entries of one tile (runs of consecutive atoms)
constexpr int kMaxRowAtoms = 32;      // atoms of one row cluster
constexpr int kMaxColAtoms = 16;      // atoms of one column cluster
constexpr int kMaxBlocks = kMaxRowAtoms * kMaxColAtoms;  // C blocks of one tile
constexpr int kPartStride = kMaxColAtoms + 1;  // padded: the rows of a warp hit distinct banks
// An integer x with |x| < 2^51 added to the bit pattern of 2^52 + 2^51 gives
// the double 2^52 + 2^51 + x exactly; subtracting that constant leaves x.
constexpr long long kBias = 0x4338000000000000LL;
constexpr double kBiasD = 6755399441055744.0;
// Exponents up to this size scale by multiplying with exact powers of two
// (no intermediate can under- or overflow); larger ones go through ldexp.
constexpr int kExactExp = 500;
constexpr int kProdWarps = 6;                 // warps 0-5: producers
constexpr int kProducers = 32 * kProdWarps;
constexpr int kMmaWarp = kProdWarps;          // warp 6: entry loader and MMA issuer
constexpr int kEpiWarp0 = kMmaWarp + 1;       // warps 7-10: epilogue
constexpr int kTileThreads = 32 * (kEpiWarp0 + 4);
constexpr int kUnits = 32 * (8 + 4);          // 16-byte (row, chunk) copies of a stage and plane
static_assert(kUnits % kProducers == 0, "units split evenly over the producers");
constexpr int kTmemCols = 512;
constexpr int64_t kRowMask = (1 << 25) - 1;  // panel row of an entry (its row count in the top 7 bits)
// Level accumulators stay exact while (K rows) * S * 127^2 < 2^31.
constexpr int64_t kMaxKRows = (int64_t)INT_MAX / (kS * 127 * 127);
constexpr double kFirst = 127.0, kBase = 254.0;
// Weight of level L: 1 / (127^2 254^L).
__device__ constexpr double kLevelW[kS] = {1.0 / 16129.0, 1.0 / (16129.0 * 254.0), 1.0 / (16129.0 * 64516.0),
                                          1.0 / (16129.0 * 16387064.0), 1.0 / (16129.0 * 4162314256.0),
                                          1.0 / (16129.0 * 1057227821024.0)};

enum : int { kErrTimeoutFull = 1, kErrTimeoutEmpty = 2, kErrTimeoutTmemFull = 4, kErrTimeoutTmemEmpty = 8,
             kErrTimeoutEnt = 16, kErrTimeoutDone = 32, kErrEntries = 64 };

// ---- shared-memory layout of the tile kernel --------------------------------------------
struct __align__(16) TileSmem {
  // the tile's scaled FP64 values: element (m, n) at m * kN + (n ^ (m % 16))
  double stg[kM * kN];
  // sum of squares of row m over the columns of column atom b, at m * kPartStride + b
  double part[kM * kPartStride];
  // entries of two tiles (the loader fills one while the producers use the other)
  int32_t ent_a[2][kMaxEnt];
  int32_t ent_b[2][kMaxEnt];
  uint16_t ent_pre[2][kMaxEnt + 8];  // first K row of every entry (K rows < 2^16)
  int32_t ent_n[2];
  int32_t ent_k[2];  // K rows of the tile
  // epilogue tables of the current tile
  long long boff[kMaxBlocks];     // data offset of C block (row atom a, column atom b) at a * 16 + b, or -1
  int32_t blk_id[kMaxBlocks];     // C blocks of the tile in list order: index in C
  int32_t blk_geom[kMaxBlocks];   // and geometry (first tile row | bi << 7 | row atom << 14 | column atom << 19)
  double col_scale[kN];           // 2^exponent of every tile column (when not wide)
  int32_t col_exp[kN];
  int32_t col_atom[kMaxColAtoms]; // first tile column | width << 8 of every column atom
  int32_t n_blk;
  int32_t n_col_atoms;
  unsigned long long bar_full[kStages], bar_empty[kStages];
  unsigned long long bar_tmem_full, bar_tmem_empty, bar_ent_full[2], bar_ent_empty[2], bar_done;
  uint32_t tmem_base;
  int abort;
};

constexpr size_t kSmemBytes = (size_t)kStages * kStageBytes + sizeof(TileSmem) + 1024;  // + alignment slack
static_assert(kSmemBytes <= 232448, "tile kernel exceeds the shared memory of one CTA");
static_assert(kMaxKRows < 65536, "entry starts are stored as 16-bit K rows");

struct TcArgs {
  const int2* tiles;
  int64_t n_tiles;
  const int64_t* ent_base;
  const int64_t* ent_cnt;
  const int32_t* krows;
  const uint2* ent;
  const int8_t* pan_a;
  int64_t plane_a;  // bytes between digit planes of the A panels
  const int8_t* pan_b;
  int64_t plane_b;
  const int32_t* rc_first;
  const int32_t* rc_atoms;
  const int32_t* cc_first;
  const int32_t* cc_atoms;
  const int8_t* row_bs;  // C (= A) row block sizes
  const int8_t* col_bs;  // C (= B) column block sizes
  const int64_t* rbase;  // first element row of every A row atom
  const int64_t* cbase;  // first element column of every B column atom
  const int* ea;
  const int* eb;
  // C blocks of every tile: tile t owns blist[lbase[t] .. lbase[t + 1]),
  // each (C block index, geometry, data offset low, high word)
  const int4* blist;
  const int64_t* lbase;
  // per row cluster and tile row m: the row's exponent (0 for padding) and
  // (row atom << 16 | element << 8 | block size) or -1 for padding
  const int32_t* rc_exp;
  const int32_t* rc_row;
  // per column cluster and tile column n the column's exponent; per column
  // atom (first tile column | width << 8)
  const int32_t* cc_exp;
  const int32_t* cc_ab;
  double* c_data;
  double* c_nrm;
  int* err;
};

// ---- PTX helpers -----------------------------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}
// x * 2^e for any e, out of line: the scatter loop is unrolled 64 times and
// only exponents beyond kExactExp (not met in practice) take this path.
__device__ __noinline__ double scale_wide(double x, int e) { return ldexp(x, e); }
// 2^e for -1022 <= e <= 1023, exactly.
__device__ __forceinline__ double pow2(int e) { return __longlong_as_double((long long)(e + 1023) << 52); }
__device__ __forceinline__ uint64_t now_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
__device__ __forceinline__ void bar_init(unsigned long long* b, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(b)), "r"(count) : "memory");
}
__device__ __forceinline__ void bar_arrive(unsigned long long* b) {
  asm volatile("{\n\t.reg .b64 st;\n\tmbarrier.arrive.shared::cta.b64 st, [%0];\n\t}" ::"r"(smem_u32(b)) : "memory");
}
__device__ __forceinline__ bool bar_try(unsigned long long* b, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(b)), "r"(parity)
      : "memory");
  return ok != 0;
}
// try_wait with a suspend-time hint: a waiting thread sleeps in hardware
// (issuing nothing) until the phase completes or about `ns` nanoseconds pass.
__device__ __forceinline__ bool bar_try_sleep(unsigned long long* b, uint32_t parity, uint32_t ns) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\tselp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(b)), "r"(parity), "r"(ns)
      : "memory");
  return ok != 0;
}
// Waits until the phase with the given parity has completed; gives up after
// 2 s (or when another role aborted), recording `code`.  The waiting thread
// sleeps between checks, leaving the issue slots to the other warps of its
// SM sub-partition.
__device__ __forceinline__ bool bar_wait(unsigned long long* b, uint32_t parity, TileSmem* sm, int* err, int code) {
  if (bar_try(b, parity)) return true;
  const uint64_t t0 = now_ns();
  for (;;) {
    if (bar_try_sleep(b, parity, 200000u)) return true;
    if (*(volatile int*)&sm->abort) return false;
    if (now_ns() - t0 > 2000000000ull) {
      atomicOr(err, code);
      *(volatile int*)&sm->abort = 1;
      return false;
    }
  }
}
__device__ __forceinline__ void cp16(uint32_t dst, const void* src, uint32_t bytes) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(dst), "l"(src), "r"(bytes) : "memory");
}
// Arrive on the mbarrier once every cp.async this thread issued so far has
// landed (counts as one of the barrier's expected arrivals).
__device__ __forceinline__ void cp_arrive(unsigned long long* b) {
  asm volatile("cp.async.mbarrier.arrive.noinc.shared::cta.b64 [%0];" ::"r"(smem_u32(b)) : "memory");
}
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void named_sync(int id, int n) { asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(n) : "memory"); }
// Named barrier that also returns the OR of every participant's predicate.
__device__ __forceinline__ bool named_sync_or(int id, int n, bool pred) {
  uint32_t r;
  asm volatile(
      "{\n\t.reg .pred p, q;\n\tsetp.ne.u32 p, %1, 0;\n\tbar.red.or.pred q, %2, %3, p;\n\tselp.u32 %0, 1, 0, q;\n\t}"
      : "=r"(r)
      : "r"((uint32_t)pred), "r"(id), "r"(n)
      : "memory");
  return r != 0;
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// Shared-memory matrix descriptor (tcgen05): start address, leading / stride
// byte offsets (16-byte units), version 1, swizzle mode.
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo, uint32_t swizzle) {
  uint64_t d = 0;
  d |= (uint64_t)((addr >> 4) & 0x3fff);
  d |= (uint64_t)((lbo >> 4) & 0x3fff) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3fff) << 32;
  d |= (uint64_t)1 << 46;              // descriptor version (Blackwell)
  d |= (uint64_t)(swizzle & 7) << 61;  // 2: 128-byte swizzle, 4: 64-byte swizzle
  return d;
}
// Instruction descriptor: kind::i8, signed A and B, int32 accumulator, both
// operands MN-major, M = 128, the given N (a multiple of 16 up to 256).
constexpr uint32_t idesc_i8(int n) {
  return (2u << 4) | (1u << 7) | (1u << 10) | (1u << 15) | (1u << 16) | ((uint32_t)(n >> 3) << 17) |
         ((uint32_t)(kM >> 4) << 24);
}

__device__ __forceinline__ void mma_i8(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem),
      "l"(a), "l"(b), "r"(idesc), "r"(acc)
      : "memory");
}
__device__ __forceinline__ void mma_commit(unsigned long long* b) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(b))
               : "memory");
}
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, int (&v)[32]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16,%17,%18,"
      "%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
      : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]), "=r"(v[8]),
        "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15]), "=r"(v[16]),
        "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]), "=r"(v[22]), "=r"(v[23]), "=r"(v[24]),
        "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]), "=r"(v[30]), "=r"(v[31])
      : "r"(taddr));
}
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, int (&v)[16]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]), "=r"(v[8]),
        "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
      : "r"(taddr));
}
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// Byte offset of (inner row kk, 16-byte chunk c) of one digit plane of a
// stage: A rows are 128 bytes, 128-byte swizzle (chunk ^= row % 8); B rows
// are 64 bytes, 64-byte swizzle (chunk ^= (row / 2) % 4).
__device__ __forceinline__ uint32_t a_swz(int kk, int c) { return (uint32_t)(kk * 128 + ((c ^ (kk & 7)) << 4)); }
__device__ __forceinline__ uint32_t b_swz(int kk, int c) { return (uint32_t)(kk * 64 + ((c ^ ((kk >> 1) & 3)) << 4)); }

// ---- the tile kernel ------------------------------------------------------------------------
__global__ void __launch_bounds__(kTileThreads, 1) k_tc_tiles(TcArgs g) {
  extern __shared__ unsigned char smem_raw[];
  // 1024-byte aligned base by pointer arithmetic on the shared array, so that
  // the compiler keeps the shared state space (shared loads and stores, not
  // generic ones)
  unsigned char* base = smem_raw + ((1024u - (smem_u32(smem_raw) & 1023u)) & 1023u);
  unsigned char* stages = base;
  TileSmem* sm = reinterpret_cast<TileSmem*>(base + (size_t)kStages * kStageBytes);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

  if (tid == 0) {
    for (int s = 0; s < kStages; ++s) {
      bar_init(&sm->bar_full[s], kProducers);
      bar_init(&sm->bar_empty[s], 1);
    }
    bar_init(&sm->bar_tmem_full, 1);
    bar_init(&sm->bar_tmem_empty, 128);
    for (int b = 0; b < 2; ++b) {
      bar_init(&sm->bar_ent_full[b], 32);
      bar_init(&sm->bar_ent_empty[b], kProducers);
    }
    bar_init(&sm->bar_done, 1);
    sm->abort = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == kMmaWarp) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&sm->tmem_base)),
                 "r"(kTmemCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = sm->tmem_base;
  const int64_t n_tiles = g.n_tiles;

  if (warp < kProdWarps) {
    // ================= producers =================
    const int pt = tid;  // 0..kProducers-1
    // A stage is 32 inner rows x (8 A chunks + 4 B chunks) of 16 bytes per
    // digit plane: 384 (row, chunk) units, two per producer thread.  Units
    // 0..255 are A (row u / 8, chunk u % 8), 256..383 are B (row v / 4,
    // chunk v % 4): consecutive lanes copy consecutive chunks of one panel
    // row, so a warp reads whole 128-byte (A) or 64-byte (B) rows.
    int64_t gs = 0;      // stages issued by this CTA so far
    int64_t local = 0;
    for (int64_t t = blockIdx.x; t < n_tiles && !sm->abort; t += gridDim.x, ++local) {
      const int buf = (int)(local & 1);
      if (!bar_wait(&sm->bar_ent_full[buf], (uint32_t)((local >> 1) & 1), sm, g.err, kErrTimeoutEnt)) break;
      const int n = sm->ent_n[buf];
      const int K = sm->ent_k[buf];
      const int nst = K > 0 ? (K + kK - 1) / kK : 1;
      const uint16_t* pre = sm->ent_pre[buf];
      // last entry e with pre[e] <= kk (a binary search; only for stages
      // where more than 31 entries start)
      auto find = [&](int kk) {
        int lo = 0, hi = n - 1;
        while (lo < hi) {
          const int mid = (lo + hi + 1) >> 1;
          if (pre[mid] <= kk) lo = mid; else hi = mid - 1;
        }
        return lo;
      };
      int e0 = 0;  // the entry holding the stage's first inner row
      for (int s = 0; s < nst; ++s, ++gs) {
        const int stg = (int)(gs % kStages);
        if (!bar_wait(&sm->bar_empty[stg], (uint32_t)(((gs / kStages) & 1) ^ 1), sm, g.err, kErrTimeoutEmpty)) break;
        const uint32_t sa = smem_u32(stages + (size_t)stg * kStageBytes);
        const uint32_t sb = sa + kStageA;
        // lane r of every producer warp finds the panel rows of the stage's
        // inner row r; the units take them by shuffle.  Lane j reads the
        // start of entry e0 + j: the entries starting inside the stage set
        // one bit each (starts are distinct, every entry has rows), and the
        // entry of row r is e0 plus the starts at or before it.
        int my_a = 0, my_b = 0;
        {
          const int r0 = s * kK, kk = r0 + lane;
          const int j = e0 + lane;
          const int P = j <= n ? (int)pre[j] : 0x10000;
          const uint32_t mask = __reduce_or_sync(0xffffffffu, lane >= 1 && P < r0 + kK ? 1u << (P - r0) : 0u);
          const bool at_end = __any_sync(0xffffffffu, lane >= 1 && P == r0 + kK);
          const bool crowded = __shfl_sync(0xffffffffu, P, 31) < r0 + kK;  // starts beyond the 32 read
          int e;
          if (!crowded) {
            e = e0 + __popc(mask & (0xffffffffu >> (31 - lane)));
            e0 += __popc(mask) + (at_end ? 1 : 0);
          } else {
            e = find(kk < K ? kk : K - 1);
            e0 = find(r0 + kK < K ? r0 + kK : K - 1);
          }
          if (kk < K) {
            my_a = sm->ent_a[buf][e] + (kk - pre[e]);
            my_b = sm->ent_b[buf][e] + (kk - pre[e]);
          }
        }
#pragma unroll
        for (int i = 0; i < kUnits / kProducers; ++i) {
          const int u = pt + kProducers * i;
          const bool is_a = u < 256;  // uniform over the warp
          const int row = is_a ? (u >> 3) : ((u - 256) >> 2);
          const int ch = is_a ? (u & 7) : ((u - 256) & 3);
          const bool valid = s * kK + row < K;
          const int64_t prow = __shfl_sync(0xffffffffu, is_a ? my_a : my_b, row);
          const uint32_t bytes = valid ? 16u : 0u;
          if (is_a) {
            const int8_t* src = g.pan_a + prow * 128 + 16 * ch;
#pragma unroll
            for (int p = 0; p < kS; ++p) cp16(sa + p * kPlaneA + a_swz(row, ch), src + p * g.plane_a, bytes);
          } else {
            const int8_t* src = g.pan_b + prow * 64 + 16 * ch;
#pragma unroll
            for (int p = 0; p < kS; ++p) cp16(sb + p * kPlaneB + b_swz(row, ch), src + p * g.plane_b, bytes);
          }
        }
        cp_arrive(&sm->bar_full[stg]);
      }
      // the entry buffer of this tile may be refilled once every producer is past it
      bar_arrive(&sm->bar_ent_empty[buf]);
    }
  } else if (warp >= kEpiWarp0) {
    // ================= epilogue =================
    const int ew = warp & 3;        // tensor-memory lane quarter (warp id mod 4)
    const int et = 32 * ew + lane;  // tile row m
    // Tables of the next tile, loaded into registers while the current tile
    // is written out: this thread's row exponent and row descriptor, the
    // column exponents (threads < kN), column atoms (threads < 16) and
    // count, block count and up to kMaxBlocks / 128 block-list entries per
    // thread.  The list bounds and clusters of the tile after next are
    // loaded one tile earlier still, so no load waits on another.
    constexpr int kBlkRegs = kMaxBlocks / 128;
    int nx_er = 0, nx_ri = -1, nx_ec = 0, nx_cab = 0, nx_nca = 0, nx_nb = 0;
    int4 nx_b[kBlkRegs];
    int64_t lb_lo = 0, lb_hi = 0;  // list bounds of the tile being prefetched
    int2 lb_tile = make_int2(0, 0);  // and its clusters
    auto bounds = [&](int64_t t) {
      lb_lo = t < n_tiles ? g.lbase[t] : 0;
      lb_hi = t < n_tiles ? g.lbase[t + 1] : 0;
      lb_tile = t < n_tiles ? g.tiles[t] : make_int2(0, 0);
    };
    auto prefetch = [&]() {
      const int I = lb_tile.x, J = lb_tile.y;
      nx_er = g.rc_exp[(int64_t)I * kM + et];
      nx_ri = g.rc_row[(int64_t)I * kM + et];
      if (et < kN) nx_ec = g.cc_exp[(int64_t)J * kN + et];
      if (et < kMaxColAtoms) nx_cab = g.cc_ab[(int64_t)J * kMaxColAtoms + et];
      nx_nca = g.cc_first[J + 1] - g.cc_first[J];
      nx_nb = (int)(lb_hi - lb_lo);
#pragma unroll
      for (int j = 0; j < kBlkRegs; ++j) {
        const int k = et + 128 * j;
        nx_b[j] = k < nx_nb ? g.blist[lb_lo + k] : make_int4(0, 0, 0, 0);
      }
    };
    // Writes the prefetched tables to shared memory; returns whether some
    // exponent of the tile lies beyond kExactExp (the same for every thread).
    auto publish = [&]() -> bool {
#pragma unroll
      for (int j = 0; j < kBlkRegs; ++j) sm->boff[et + 128 * j] = -1;
      if (et < kN) {
        sm->col_exp[et] = nx_ec;
        sm->col_scale[et] = pow2(nx_ec < -kExactExp || nx_ec > kExactExp ? 0 : nx_ec);
      }
      if (et < kMaxColAtoms) sm->col_atom[et] = nx_cab;
      if (et == 0) {
        sm->n_blk = nx_nb;
        sm->n_col_atoms = nx_nca;
      }
      named_sync(2, 128);  // every slot reset before the blocks are entered
#pragma unroll
      for (int j = 0; j < kBlkRegs; ++j) {
        const int k = et + 128 * j;
        if (k < nx_nb) {
          const int geo = nx_b[j].y;
          sm->blk_id[k] = nx_b[j].x;
          sm->blk_geom[k] = geo;
          sm->boff[((geo >> 14) & 31) * kMaxColAtoms + ((geo >> 19) & 15)] =
              (long long)(((uint64_t)(uint32_t)nx_b[j].w << 32) | (uint32_t)nx_b[j].z);
        }
      }
      const bool w = nx_er < -kExactExp || nx_er > kExactExp || (et < kN && (nx_ec < -kExactExp || nx_ec > kExactExp));
      return named_sync_or(2, 128, w);
    };
    int64_t local = 0;
    bool wide = false;
    int er = 0, ri = -1;  // this thread's row: exponent and descriptor
    if ((int64_t)blockIdx.x < n_tiles) {
      bounds(blockIdx.x);
      prefetch();
      bounds(blockIdx.x + (int64_t)gridDim.x);
      er = nx_er;
      ri = nx_ri;
      wide = publish();
    }
    for (int64_t t = blockIdx.x; t < n_tiles && !sm->abort; t += gridDim.x, ++local) {
      const bool has_next = t + gridDim.x < n_tiles;
      // ---- accumulators: tensor memory -> staging tile, 16 columns a round
      // (a rolled loop: the epilogue's code stays small next to the other
      // roles' in the instruction cache).  Per column the six level sums v_L
      // recombine as (v0 254^2 + v1 254 + v2) w_2 + (v3 254^2 + v4 254 + v5) w_5
      // with w_L = 1 / (127^2 254^L): both brackets are exact in int64
      // (|v_L| < 2^31), below 2^51 in magnitude, and convert exactly to FP64
      // by the 2^52 + 2^51 bias.  The row's power of two is folded into w_2
      // and w_5 (exact: |er| <= kExactExp).  Tensor memory is released as
      // soon as the tile is staged: the next tile's MMAs wait for nothing else. ----
      if (!bar_wait(&sm->bar_tmem_full, (uint32_t)(local & 1), sm, g.err, kErrTimeoutTmemFull)) break;
      tc_fence_after();
      double* row = sm->stg + et * kN;
      const int sw = et & 15;
      {
        const double rs = wide ? 1.0 : pow2(er);
        const double w2 = kLevelW[2] * rs, w5 = kLevelW[5] * rs;
        const uint32_t lane_base = tmem + ((uint32_t)(32 * ew) << 16);
#pragma unroll 1
        for (int c0 = 0; c0 < kN; c0 += 16) {
          int v[kS][16];
#pragma unroll
          for (int L = 0; L < kS; ++L) tmem_ld16(lane_base + (uint32_t)(64 * L + c0), v[L]);
          tmem_wait_ld();
#pragma unroll
          for (int c = 0; c < 16; ++c) {
            const long long hi = kBias + (long long)v[0][c] * 64516 + (long long)v[1][c] * 254 + v[2][c];
            const long long lo = kBias + (long long)v[3][c] * 64516 + (long long)v[4][c] * 254 + v[5][c];
            const double hd = __longlong_as_double(hi) - kBiasD, ld = __longlong_as_double(lo) - kBiasD;
            row[(c0 + c) ^ sw] = __fma_rn(hd, w2, ld * w5);
          }
        }
        tc_fence_before();
        bar_arrive(&sm->bar_tmem_empty);  // the MMAs of the next tile may start
      }
      if (has_next) {
        prefetch();
        bounds(t + 2 * (int64_t)gridDim.x);
      }
      // ---- write-out: each thread writes its tile row into the C blocks of
      // its row atom, one column atom after the other (a block's column is
      // bi consecutive doubles, so a warp's store covers its rows' runs),
      // scaling by the column's power of two, and keeps the row's sum of
      // squares per column atom for the block norms ----
      if (ri >= 0) {
        const int a = ri >> 16, pe = (ri >> 8) & 0xff, bi = ri & 0xff;
        const int nca = sm->n_col_atoms;
        double* part = sm->part + et * kPartStride;
        for (int b = 0; b < nca; ++b) {
          const int cab = sm->col_atom[b];
          const int c0 = cab & 0xff, bj = cab >> 8;
          const long long bo = sm->boff[a * kMaxColAtoms + b];
          double sq = 0.0;
          if (bo >= 0) {
            double* __restrict__ dst = g.c_data + bo + pe;
            if (!wide) {
#pragma unroll 4
              for (int q = 0; q < bj; ++q) {
                const int n = c0 + q;
                const double v = row[n ^ sw] * sm->col_scale[n];
                dst[q * bi] = v;
                sq = __fma_rn(v, v, sq);
              }
            } else {  // rare: exponents beyond kExactExp, scaled out of line
              for (int q = 0; q < bj; ++q) {
                const int n = c0 + q;
                const double v = scale_wide(row[n ^ sw], er + sm->col_exp[n]);
                dst[q * bi] = v;
                sq = __fma_rn(v, v, sq);
              }
            }
          }
          part[b] = sq;
        }
      }
      named_sync(2, 128);
      // ---- block norms: rows of the block in ascending order ----
      const int nb = sm->n_blk;
      for (int k = et; k < nb; k += 128) {
        const int geo = sm->blk_geom[k];
        const int r0 = geo & 127, bi = (geo >> 7) & 127, cb = (geo >> 19) & 15;
        double sq = 0.0;
        for (int pe = 0; pe < bi; ++pe) sq += sm->part[(r0 + pe) * kPartStride + cb];
        g.c_nrm[sm->blk_id[k]] = __dsqrt_rn(sq);
      }
      named_sync(2, 128);  // the staging tile and the tables are free again
      if (has_next) {
        er = nx_er;
        ri = nx_ri;
        wide = publish();
      }
    }
  } else {
    // ================= entry loader (all lanes) and MMA issuer (lane 0) =================
    // Entries of tile `local` go to buffer local % 2.  The next tile's
    // entries are loaded into registers when a tile starts and written to
    // shared memory once the tile's tensor memory is free (the loads fly
    // meanwhile), before its first MMA, so the producers can move on to the
    // next tile as soon as they have issued this one.
    int64_t gs = 0, local_mma = 0;
    bool ok = true;
    constexpr int kEntRegs = kMaxEnt / 32;
    uint2 pre_x[kEntRegs];
    int pre_n = 0, pre_k = 0, cur_k = 0;
    // entry count, base and K rows of the tile to prefetch next, loaded one
    // tile earlier so that the entry loads wait on nothing
    int64_t nb_cnt = 0, nb_base = 0;
    int nb_k = 0;
    auto bounds = [&](int64_t t) {
      nb_cnt = t < n_tiles ? g.ent_cnt[t] : 0;
      nb_base = t < n_tiles ? g.ent_base[t] : 0;
      nb_k = t < n_tiles ? g.krows[t] : 0;
    };
    auto prefetch = [&]() {
      pre_n = (int)nb_cnt;
      pre_k = nb_k;
#pragma unroll
      for (int j = 0; j < kEntRegs; ++j) {
        const int e = lane + 32 * j;
        pre_x[j] = e < pre_n ? g.ent[nb_base + e] : make_uint2(0u, 0u);
      }
    };
    auto publish = [&](int64_t lidx) -> bool {
      const int buf = (int)(lidx & 1);
      if (!bar_wait(&sm->bar_ent_empty[buf], (uint32_t)(((lidx >> 1) & 1) ^ 1), sm, g.err, kErrTimeoutEnt))
        return false;
      if (pre_n > kMaxEnt) {
        atomicOr(g.err, kErrEntries);
        sm->abort = 1;
        return false;
      }
      int carry = 0;
#pragma unroll
      for (int j = 0; j < kEntRegs; ++j) {
        if (32 * j >= pre_n) break;
        const int e = lane + 32 * j;
        const uint2 x = pre_x[j];
        const int bk = (int)(x.x >> 25);
        const int incl = warp_incl_scan(bk, lane);
        if (e < pre_n) {
          sm->ent_a[buf][e] = (int32_t)(x.x & kRowMask);
          sm->ent_b[buf][e] = (int32_t)x.y;
          sm->ent_pre[buf][e] = (uint16_t)(carry + incl - bk);
        }
        carry += __shfl_sync(0xffffffffu, incl, 31);
      }
      if (lane == 0) {
        sm->ent_pre[buf][pre_n] = (uint16_t)carry;
        sm->ent_n[buf] = pre_n;
        sm->ent_k[buf] = pre_k;
      }
      __syncwarp();
      bar_arrive(&sm->bar_ent_full[buf]);
      return true;
    };
    if ((int64_t)blockIdx.x < n_tiles) {
      bounds(blockIdx.x);
      prefetch();
      bounds(blockIdx.x + (int64_t)gridDim.x);
      ok = publish(0);
    }
    for (int64_t t = blockIdx.x; ok && t < n_tiles && !sm->abort; t += gridDim.x, ++local_mma) {
      const bool has_next = t + gridDim.x < n_tiles;
      cur_k = pre_k;  // K rows of tile t (published with its entries)
      if (has_next) {
        prefetch();
        bounds(t + 2 * (int64_t)gridDim.x);
      }
      bool published = !has_next;
      const int K = cur_k;
      const int nst = K > 0 ? (K + kK - 1) / kK : 1;
      // tensor memory is free once the epilogue has read the previous tile
      if (!bar_wait(&sm->bar_tmem_empty, (uint32_t)((local_mma & 1) ^ 1), sm, g.err, kErrTimeoutTmemEmpty)) break;
      tc_fence_after();
      for (int s = 0; s < nst; ++s, ++gs) {
        const int stg = (int)(gs % kStages);
        if (!bar_wait(&sm->bar_full[stg], (uint32_t)((gs / kStages) & 1), sm, g.err, kErrTimeoutFull)) { ok = false; break; }
        tc_fence_after();
        if (lane == 0) {
          fence_async_smem();
          const uint32_t sa = smem_u32(stages + (size_t)stg * kStageBytes);
          const uint32_t sb = sa + kStageA;
          // A plane p times B planes q0 .. q0 + nq - 1 in one MMA of N = 64 nq:
          // the B planes lie kPlaneB apart, which the descriptor's leading
          // byte offset steps through as consecutive 64-column chunks of N,
          // and their products land on consecutive level accumulators
          // 64 (p + q) of tensor memory.  Nine MMAs per stage cover the 21
          // pairs p + q < 6 (N <= 256 per instruction), reading A nine times
          // instead of 21.
#pragma unroll
          for (int p = 0; p < kS; ++p) {
            const uint64_t da = smem_desc(sa + p * kPlaneA, 128, 1024, 2);
#pragma unroll
            for (int q0 = 0; q0 < kS - p; q0 += 4) {
              const int nq = (kS - p - q0) < 4 ? (kS - p - q0) : 4;
              const uint64_t db = smem_desc(sb + q0 * kPlaneB, kPlaneB, 512, 4);
              mma_i8(tmem + (uint32_t)(64 * (p + q0)), da, db, idesc_i8(64 * nq), (s > 0 || p > 0) ? 1u : 0u);
            }
          }
          mma_commit(&sm->bar_empty[stg]);
        }
        __syncwarp();
        if (!published) {  // after the tile's first MMAs: the next tile's entries (loaded meanwhile)
          published = true;
          if (!(ok = publish(local_mma + 1))) break;
        }
      }
      if (!ok) break;
      if (lane == 0) mma_commit(&sm->bar_tmem_full);
      __syncwarp();
    }
    // every MMA issued by this CTA has completed before tensor memory is released
    if (lane == 0) mma_commit(&sm->bar_done);
    __syncwarp();
    bar_wait(&sm->bar_done, 0, sm, g.err, kErrTimeoutDone);
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (warp == kMmaWarp)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols) : "memory");
}

}  // namespace tc
}  // namespace lamb

// ============================================================================================
// Preparation: clusters, inner-atom bitmaps, digit panels, tiles and their inner lists.
// ============================================================================================
namespace lamb {
namespace tc {

// Bitmap bit (cluster, inner atom k): A (by_row): cluster of row r, k = column;
// B (!by_row): cluster of column c, k = row r.
__global__ void k_tc_bitmap(int32_t n_rows, const int64_t* __restrict__ row_p, const int32_t* __restrict__ col,
                            const int32_t* __restrict__ clus, int by_row, int32_t W, uint32_t* __restrict__ bm) {
  const int lane = threadIdx.x & 31;
  for (int64_t r = global_warp(); r < n_rows; r += grid_warps())
    for (int64_t b = row_p[r] + lane; b < row_p[r + 1]; b += 32) {
      const int c = col[b];
      const int cl = by_row ? clus[r] : clus[c];
      const int k = by_row ? c : (int)r;
      atomicOr(&bm[(int64_t)cl * W + (k >> 5)], 1u << (k & 31));
    }
}

// Per cluster and bitmap word: inner atoms and panel rows (sum of their block
// sizes) before the word; per cluster the totals.  One warp per cluster.
__global__ void k_tc_word_prefix(int32_t n_cl, int32_t W, const uint32_t* __restrict__ bm,
                                 const int8_t* __restrict__ kbs, int32_t* __restrict__ wrow,
                                 int64_t* __restrict__ tot_row) {
  const int lane = threadIdx.x & 31;
  for (int64_t c = global_warp(); c < n_cl; c += grid_warps()) {
    int carry = 0;
    for (int w0 = 0; w0 < W; w0 += 32) {
      const int w = w0 + lane;
      uint32_t bits = w < W ? bm[c * W + w] : 0u;
      int rows = 0;
      while (bits) {
        const int bit = __ffs(bits) - 1;
        bits &= bits - 1u;
        rows += kbs[32 * w + bit];
      }
      const int incl = warp_incl_scan(rows, lane);
      if (w < W) wrow[c * W + w] = carry + incl - rows;
      carry += __shfl_sync(0xffffffffu, incl, 31);
    }
    if (lane == 0) tot_row[c] = carry;
  }
}

// Panel row of inner atom k within cluster c's panel (relative to its
// base), by the whole warp: lane b adds the rows of atom 32 (k / 32) + b
// when its bit is set and below k's.
__device__ __forceinline__ int64_t panel_row_warp(const uint32_t* __restrict__ bm, const int32_t* __restrict__ wrow,
                                                  const int8_t* __restrict__ kbs, int64_t c, int32_t W, int k,
                                                  int lane) {
  const int w = k >> 5;
  const uint32_t word = bm[c * W + w];
  const int add = lane < (k & 31) && ((word >> lane) & 1u) ? kbs[32 * w + lane] : 0;
  return wrow[c * W + w] + __reduce_add_sync(0xffffffffu, add);
}

// Writes the S digits of x (|x| < 1) to S planes: |127 x| < 127 and every
// later t lies in [-127, 127], so each digit fits int8.
__device__ __forceinline__ void put_digits(int8_t* __restrict__ pan, int64_t plane, int64_t pos, double x) {
  double t = x * kFirst;
#pragma unroll
  for (int p = 0; p < kS; ++p) {
    const double dg = rint(t);
    pan[p * plane + pos] = (int8_t)dg;
    t = (t - dg) * kBase;
  }
}

// x * 2^-e: an exact power-of-two multiply where 2^-e is a normal double
// (the result rounds once either way), ldexp outside that range.
__device__ __forceinline__ double scale_down(double x, int e) {
  return e > -1000 && e < 1000 ? x * __longlong_as_double((long long)(1023 - e) << 52) : ldexp(x, -e);
}

// Warps per block row in the digit kernels (memory parallelism across the
// row's blocks).
constexpr int kDigitWays = 8;

// A panels: element (pe, kc) of block (i, k) goes to panel row
// base[I] + row(I, k) + kc, byte roff[i] + pe of that 128-byte row.  Lanes
// walk the block in storage order (pe fastest), so they write consecutive
// bytes of a panel row.
__global__ void k_tc_digits_a(int32_t n_rows, const int64_t* __restrict__ row_p, const int32_t* __restrict__ col,
                              const int64_t* __restrict__ off, const int8_t* __restrict__ row_bs,
                              const int8_t* __restrict__ kbs, const double* __restrict__ data,
                              const int32_t* __restrict__ rcl, const int32_t* __restrict__ roff, int32_t W,
                              const uint32_t* __restrict__ bm, const int32_t* __restrict__ wrow,
                              const int64_t* __restrict__ base, const int64_t* __restrict__ rbase,
                              const int* __restrict__ ea, int64_t plane, int8_t* __restrict__ pan) {
  const int lane = threadIdx.x & 31;
  // kDigitWays warps per block row, each every kDigitWays-th block of it
  for (int64_t gw = global_warp(); gw < (int64_t)n_rows * kDigitWays; gw += grid_warps()) {
    const int64_t i = gw / kDigitWays;
    const int I = rcl[i], m0 = roff[i], bi = row_bs[i];
    const int64_t e0 = rbase[i];
    for (int64_t b = row_p[i] + gw % kDigitWays; b < row_p[i + 1]; b += kDigitWays) {
      const int k = col[b], bk = kbs[k];
      const int64_t prow = base[I] + panel_row_warp(bm, wrow, kbs, I, W, k, lane);
      const double* x = data + off[b];
      Walk w(bi, lane);
      for (int e = lane; e < bi * bk; e += 32, w.next())
        put_digits(pan, plane, (prow + w.major) * 128 + m0 + w.minor, scale_down(x[e], ea[e0 + w.minor]));
    }
  }
}

// B panels: element (kr, q) of block (k, j) goes to panel row
// base[J] + row(J, k) + kr, byte coff[j] + q of that 64-byte row.  Lanes
// walk the block row by row (q fastest), so they write consecutive bytes of
// a panel row (the strided reads stay within the block).
__global__ void k_tc_digits_b(int32_t n_rows, const int64_t* __restrict__ row_p, const int32_t* __restrict__ col,
                              const int64_t* __restrict__ off, const int8_t* __restrict__ kbs,
                              const int8_t* __restrict__ col_bs, const double* __restrict__ data,
                              const int32_t* __restrict__ ccl, const int32_t* __restrict__ coff, int32_t W,
                              const uint32_t* __restrict__ bm, const int32_t* __restrict__ wrow,
                              const int64_t* __restrict__ base, const int64_t* __restrict__ cbase,
                              const int* __restrict__ eb, int64_t plane, int8_t* __restrict__ pan) {
  const int lane = threadIdx.x & 31;
  for (int64_t gw = global_warp(); gw < (int64_t)n_rows * kDigitWays; gw += grid_warps()) {
    const int64_t k = gw / kDigitWays;
    const int bk = kbs[k];
    for (int64_t b = row_p[k] + gw % kDigitWays; b < row_p[k + 1]; b += kDigitWays) {
      const int j = col[b], J = ccl[j], n0 = coff[j], bj = col_bs[j];
      const int64_t prow = base[J] + panel_row_warp(bm, wrow, kbs, J, W, (int)k, lane);
      const double* x = data + off[b];
      const int64_t e0 = cbase[j];
      Walk w(bj, lane);
      for (int e = lane; e < bk * bj; e += 32, w.next()) {
        const int q = w.minor, kr = w.major;
        put_digits(pan, plane, (prow + kr) * 64 + n0 + q, scale_down(x[kr + q * bk], eb[e0 + q]));
      }
    }
  }
}

// Tile flags: (row cluster, column cluster) pairs holding a C block.
__global__ void k_tc_tile_flags(int32_t n_rows, const int64_t* __restrict__ row_p, const int32_t* __restrict__ col,
                                const int32_t* __restrict__ rcl, const int32_t* __restrict__ ccl, int32_t n_cc,
                                int64_t* __restrict__ flag) {
  const int lane = threadIdx.x & 31;
  for (int64_t i = global_warp(); i < n_rows; i += grid_warps()) {
    const int64_t I = rcl[i];
    for (int64_t b = row_p[i] + lane; b < row_p[i + 1]; b += 32) flag[I * n_cc + ccl[col[b]]] = 1;
  }
}

__global__ void k_tc_tile_list(int64_t n_map, int32_t n_cc, const int64_t* __restrict__ flag,
                               const int64_t* __restrict__ pos, int2* __restrict__ tiles) {
  for (int64_t x = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; x < n_map; x += (int64_t)gridDim.x * blockDim.x)
    if (flag[x]) tiles[pos[x]] = make_int2((int)(x / n_cc), (int)(x % n_cc));
}

// C blocks of every tile.  Count pass: blocks per tile.  Fill pass: one
// list entry per block at lbase[t] + (arrival order within the tile), each
// (block index, geometry, data offset) with geometry = first tile row |
// bi << 7 | row atom << 14 | column atom << 19.  The order within a tile
// decides nothing but which thread computes which norm.
template <bool FILL>
__global__ void k_tc_tile_blocks(int32_t n_rows, const int64_t* __restrict__ row_p, const int32_t* __restrict__ col,
                                 const int64_t* __restrict__ off, const int8_t* __restrict__ row_bs,
                                 const int32_t* __restrict__ rcl, const int32_t* __restrict__ roff,
                                 const int32_t* __restrict__ ratom, const int32_t* __restrict__ ccl,
                                 const int32_t* __restrict__ catom, int32_t n_cc,
                                 const int64_t* __restrict__ pos, int64_t* __restrict__ cnt,
                                 const int64_t* __restrict__ lbase, int4* __restrict__ blist) {
  const int lane = threadIdx.x & 31;
  for (int64_t i = global_warp(); i < n_rows; i += grid_warps()) {
    const int64_t I = rcl[i];
    const int geo_r = roff[i] | ((int)row_bs[i] << 7) | (ratom[i] << 14);
    for (int64_t b = row_p[i] + lane; b < row_p[i + 1]; b += 32) {
      const int j = col[b];
      const int64_t t = pos[I * n_cc + ccl[j]];
      const int64_t slot = (int64_t)atomicAdd(reinterpret_cast<unsigned long long*>(&cnt[t]), 1ull);
      if (FILL) {
        const int geo = geo_r | (catom[j] << 19);
        const uint64_t o = (uint64_t)off[b];
        blist[lbase[t] + slot] = make_int4((int)b, geo, (int)(uint32_t)o, (int)(uint32_t)(o >> 32));
      }
    }
  }
}

// Inner atoms of every tile: k with A_ik for some i in I and B_kj for some j
// in J (and b_k > 0), in increasing k.  Consecutive such atoms whose panel
// rows follow on in both panels (no atom of only one cluster between them)
// merge into one entry of up to 127 rows, within one 32-atom bitmap word.
// Count pass: entries and panel rows per tile.  Fill pass: (A panel row |
// rows << 25, B panel row) per entry.  One warp per tile, a lane per word.
template <bool FILL>
__device__ __forceinline__ int tile_word_entries(uint32_t xa, uint32_t xb, int w, const int8_t* __restrict__ kbs,
                                                 int64_t ar, int64_t br, uint2* __restrict__ out, int* nrows,
                                                 int* slot) {
  const uint32_t x = xa & xb;
  int n = 0, open = 0;  // rows of the open entry (0: none)
  int64_t oa = 0, ob = 0;
  for (uint32_t y = xa | xb; y;) {
    const int bit = __ffs(y) - 1;
    y &= y - 1u;
    const uint32_t mb = 1u << bit;
    const int bk = kbs[32 * w + bit];
    if (bk > 0) {
      if (x & mb) {
        *nrows += bk;
        if (open > 0 && open + bk <= 127) {
          open += bk;
        } else {
          if (open > 0) {
            if (FILL) out[atomicAdd(slot, 1)] = make_uint2((uint32_t)oa | ((uint32_t)open << 25), (uint32_t)ob);
            ++n;
          }
          oa = ar;
          ob = br;
          open = bk;
        }
      } else if (open > 0) {  // rows of one panel only: the next entry starts apart
        if (FILL) out[atomicAdd(slot, 1)] = make_uint2((uint32_t)oa | ((uint32_t)open << 25), (uint32_t)ob);
        ++n;
        open = 0;
      }
    }
    if (xa & mb) ar += bk;
    if (xb & mb) br += bk;
  }
  if (open > 0) {
    if (FILL) out[atomicAdd(slot, 1)] = make_uint2((uint32_t)oa | ((uint32_t)open << 25), (uint32_t)ob);
    ++n;
  }
  return n;
}

template <bool FILL>
__global__ void __launch_bounds__(256) k_tc_tile_k(int64_t n_tiles, const int2* __restrict__ tiles, int32_t W,
                                                   const uint32_t* __restrict__ bma, const uint32_t* __restrict__ bmb,
                                                   const int32_t* __restrict__ wra, const int32_t* __restrict__ wrb,
                                                   const int64_t* __restrict__ basea, const int64_t* __restrict__ baseb,
                                                   const int8_t* __restrict__ kbs, int64_t* __restrict__ cnt,
                                                   int32_t* __restrict__ rows, const int64_t* __restrict__ ebase,
                                                   uint2* __restrict__ ent) {
  // Fill pass: entries take the next free slot of their tile (a per-warp
  // counter); the K-row order inside a tile does not change the exact int32
  // level sums, and the producers' row prefix follows the stored order.
  __shared__ int slot[8];
  const int lane = threadIdx.x & 31, wl = threadIdx.x >> 5;
  for (int64_t t = global_warp(); t < n_tiles; t += grid_warps()) {
    const int64_t I = tiles[t].x, J = tiles[t].y;
    int64_t carry = 0;
    int nrows = 0;
    if (FILL && lane == 0) slot[wl] = 0;
    __syncwarp();
    uint2* out = FILL ? ent + ebase[t] : nullptr;
    for (int w0 = 0; w0 < W; w0 += 32) {
      const int w = w0 + lane;
      const uint32_t xa = w < W ? bma[I * W + w] : 0u, xb = w < W ? bmb[J * W + w] : 0u;
      int c = 0;
      if (xa & xb) {
        const int64_t ar = basea[I] + wra[I * W + w], br = baseb[J] + wrb[J * W + w];
        c = tile_word_entries<FILL>(xa, xb, w, kbs, ar, br, out, &nrows, &slot[wl]);
      }
      if (!FILL) carry += warp_sum_ll(c);
    }
    if (!FILL) {
      nrows = (int)warp_sum_ll(nrows);
      if (lane == 0) {
        cnt[t] = carry;
        rows[t] = nrows;
      }
    }
    __syncwarp();
  }
}

// Largest inner-atom count and K of any tile, and the pipeline stages of
// all tiles (ceil(K / 32), at least one), into out[0..2].
__global__ void k_tc_tile_stats(int64_t n_tiles, const int64_t* __restrict__ cnt, const int32_t* __restrict__ rows,
                                unsigned long long* __restrict__ out) {
  long long me = 0, mr = 0, st = 0;
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < n_tiles; t += (int64_t)gridDim.x * blockDim.x) {
    me = max(me, (long long)cnt[t]);
    mr = max(mr, (long long)rows[t]);
    st += rows[t] > 0 ? (rows[t] + kK - 1) / kK : 1;
  }
  for (int o = 16; o; o >>= 1) {
    me = max(me, __shfl_xor_sync(0xffffffffu, me, o));
    mr = max(mr, __shfl_xor_sync(0xffffffffu, mr, o));
    st += __shfl_xor_sync(0xffffffffu, st, o);
  }
  if ((threadIdx.x & 31) == 0) {
    atomicMax(&out[0], (unsigned long long)me);
    atomicMax(&out[1], (unsigned long long)mr);
    atomicAdd(&out[2], (unsigned long long)st);
  }
}

// Exponent of every tile row / column of every cluster (0 for padding).
__global__ void k_tc_cluster_exp(int64_t n, const int64_t* __restrict__ elem, const int* __restrict__ e,
                                 int32_t* __restrict__ out) {
  for (int64_t x = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; x < n; x += (int64_t)gridDim.x * blockDim.x)
    out[x] = elem[x] >= 0 ? e[elem[x]] : 0;
}

// ---- host ----------------------------------------------------------------------------------
struct Clusters {
  int32_t n = 0;
  std::vector<int32_t> of, idx, off, first, atoms;
};

// Greedy cut of `order` into clusters of at most max_rows rows and max_atoms atoms.
static Clusters make_clusters(const std::vector<int32_t>& order, const std::vector<int8_t>& bs, int max_rows,
                              int max_atoms) {
  Clusters c;
  const size_t n = bs.size();
  c.of.assign(n, 0);
  c.idx.assign(n, 0);
  c.off.assign(n, 0);
  int rows = 0, atoms = 0;
  for (size_t t = 0; t < order.size(); ++t) {
    const int a = order[t], b = bs[a];
    if (c.first.empty() || rows + b > max_rows || atoms == max_atoms) {
      c.first.push_back((int32_t)c.atoms.size());
      rows = 0;
      atoms = 0;
    }
    c.of[a] = (int32_t)c.first.size() - 1;
    c.idx[a] = atoms;
    c.off[a] = rows;
    c.atoms.push_back(a);
    rows += b;
    ++atoms;
  }
  c.n = (int32_t)c.first.size();
  c.first.push_back((int32_t)c.atoms.size());
  return c;
}

template <typename T>
static int32_t upload_vec(Ctx* ctx, const std::vector<T>& v, T** d) {
  LAMB_TRY(dalloc(ctx, d, std::max<int64_t>((int64_t)v.size(), 1)));
  if (!v.empty()) LAMB_CUDA(ctx, cudaMemcpyAsync(*d, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice, ctx->stream));
  return LAMB_GPU_OK;
}

// Device buffers of one call, released (stream-ordered) when it returns.
struct Bufs {
  Ctx* ctx;
  std::vector<void*> p;
  ~Bufs() {
    for (void* x : p)
      if (x) cudaFreeAsync(x, ctx->stream);
  }
  template <typename T>
  int32_t alloc(T** d, int64_t n) {
    LAMB_TRY(dalloc(ctx, d, std::max<int64_t>(n, 1)));
    p.push_back(*d);
    return LAMB_GPU_OK;
  }
  template <typename T>
  int32_t up(const std::vector<T>& v, T** d) {
    LAMB_TRY(upload_vec(ctx, v, d));
    p.push_back(*d);
    return LAMB_GPU_OK;
  }
};

}  // namespace tc

bool mixed_tc_eligible(const DevMatrix* A, const DevMatrix* B) {
  return max_block(A->h_row_bs) <= tc::kM && max_block(B->h_col_bs) <= tc::kN && A->n_rows > 0 && B->n_cols > 0 &&
         A->nnz > 0 && B->nnz > 0;
}

// Numeric phase of a mixed multiply on tcgen05 (C's pattern, layout and data
// buffer already set by a pattern-only symbolic phase).  Sets *ran = false,
// leaving C untouched, when a tile exceeds the kernel's limits (inner atoms
// or rows); the caller then uses the mma.sync path.
int32_t numeric_mixed_tc(Ctx* ctx, DevMatrix* A, DevMatrix* B, DevMatrix* C, const MixedPlanes& mp, double* c_nrm,
                         bool* ran, cudaEvent_t ev_prepared, double* tensor_ops) {
  using namespace tc;
  *ran = false;
  *tensor_ops = 0.0;
  if (C->nnz == 0) { *ran = true; return LAMB_GPU_OK; }
  // ---- clusters (host, from the row processing order) ----
  if ((int)A->h_order.size() != A->n_rows) return fail(ctx, LAMB_LEVEL_FAILURE, LAMB_TYPE_INTERNAL_ERROR, "mixed: row order missing");
  const Clusters rc = make_clusters(A->h_order, A->h_row_bs, kM, kMaxRowAtoms);
  std::vector<int32_t> corder(B->n_cols);
  if (B->n_cols == A->n_rows && B->h_col_bs == A->h_row_bs)
    corder = A->h_order;
  else
    std::iota(corder.begin(), corder.end(), 0);
  const Clusters cc = make_clusters(corder, B->h_col_bs, kN, kMaxColAtoms);
  const int32_t nk = A->n_cols, W = (nk + 31) / 32;
  Bufs m{ctx, {}};
  int32_t *d_rcl, *d_ratom, *d_roff, *d_rcf, *d_rca, *d_ccl, *d_catom, *d_coff, *d_ccf, *d_cca;
  LAMB_TRY(m.up(rc.of, &d_rcl)); LAMB_TRY(m.up(rc.idx, &d_ratom)); LAMB_TRY(m.up(rc.off, &d_roff));
  LAMB_TRY(m.up(rc.first, &d_rcf)); LAMB_TRY(m.up(rc.atoms, &d_rca));
  LAMB_TRY(m.up(cc.of, &d_ccl)); LAMB_TRY(m.up(cc.idx, &d_catom)); LAMB_TRY(m.up(cc.off, &d_coff));
  LAMB_TRY(m.up(cc.first, &d_ccf)); LAMB_TRY(m.up(cc.atoms, &d_cca));
  // per-cluster tables of the epilogue: row and column-atom descriptors, row and column exponents
  std::vector<int32_t> h_rc_row((size_t)rc.n * kM, -1), h_cc_ab((size_t)cc.n * kMaxColAtoms, 0);
  std::vector<int64_t> h_rc_elem((size_t)rc.n * kM, -1), h_cc_elem((size_t)cc.n * kN, -1);
  {
    std::vector<int64_t> rb(A->n_rows + 1, 0), cb(B->n_cols + 1, 0);
    for (int i = 0; i < A->n_rows; ++i) rb[i + 1] = rb[i] + A->h_row_bs[i];
    for (int j = 0; j < B->n_cols; ++j) cb[j + 1] = cb[j] + B->h_col_bs[j];
    for (int I = 0; I < rc.n; ++I)
      for (int a = 0; a < rc.first[I + 1] - rc.first[I]; ++a) {
        const int atom = rc.atoms[rc.first[I] + a], b = A->h_row_bs[atom], o = rc.off[atom];
        for (int pe = 0; pe < b; ++pe) {
          h_rc_row[(size_t)I * kM + o + pe] = (a << 16) | (pe << 8) | b;
          h_rc_elem[(size_t)I * kM + o + pe] = rb[atom] + pe;
        }
      }
    for (int J = 0; J < cc.n; ++J)
      for (int b = 0; b < cc.first[J + 1] - cc.first[J]; ++b) {
        const int atom = cc.atoms[cc.first[J] + b], w = B->h_col_bs[atom], o = cc.off[atom];
        h_cc_ab[(size_t)J * kMaxColAtoms + b] = o | (w << 8);
        for (int q = 0; q < w; ++q) h_cc_elem[(size_t)J * kN + o + q] = cb[atom] + q;
      }
  }
  int32_t *d_rc_row, *d_cc_ab, *d_rc_exp, *d_cc_exp;
  int64_t *d_rc_elem, *d_cc_elem;
  LAMB_TRY(m.up(h_rc_row, &d_rc_row));
  LAMB_TRY(m.up(h_cc_ab, &d_cc_ab));
  LAMB_TRY(m.up(h_rc_elem, &d_rc_elem)); LAMB_TRY(m.up(h_cc_elem, &d_cc_elem));
  LAMB_TRY(m.alloc(&d_rc_exp, (int64_t)rc.n * kM)); LAMB_TRY(m.alloc(&d_cc_exp, (int64_t)cc.n * kN));
  k_tc_cluster_exp<<<grid_for((int64_t)rc.n * kM), 256, 0, ctx->stream>>>((int64_t)rc.n * kM, d_rc_elem, mp.ea, d_rc_exp);
  LAMB_LAUNCHED(ctx);
  k_tc_cluster_exp<<<grid_for((int64_t)cc.n * kN), 256, 0, ctx->stream>>>((int64_t)cc.n * kN, d_cc_elem, mp.eb, d_cc_exp);
  LAMB_LAUNCHED(ctx);
  // ---- inner-atom bitmaps and panel row offsets ----
  uint32_t *bma, *bmb;
  int32_t *wra, *wrb;
  int64_t *tra, *trb, *basea, *baseb;
  LAMB_TRY(m.alloc(&bma, (int64_t)rc.n * W)); LAMB_TRY(m.alloc(&bmb, (int64_t)cc.n * W));
  LAMB_TRY(m.alloc(&wra, (int64_t)rc.n * W)); LAMB_TRY(m.alloc(&wrb, (int64_t)cc.n * W));
  LAMB_TRY(m.alloc(&tra, rc.n + 1)); LAMB_TRY(m.alloc(&trb, cc.n + 1));
  LAMB_TRY(m.alloc(&basea, rc.n + 1)); LAMB_TRY(m.alloc(&baseb, cc.n + 1));
  LAMB_CUDA(ctx, cudaMemsetAsync(bma, 0, sizeof(uint32_t) * (size_t)rc.n * W, ctx->stream));
  LAMB_CUDA(ctx, cudaMemsetAsync(bmb, 0, sizeof(uint32_t) * (size_t)cc.n * W, ctx->stream));
  LAMB_CUDA(ctx, cudaMemsetAsync(tra + rc.n, 0, sizeof(int64_t), ctx->stream));
  LAMB_CUDA(ctx, cudaMemsetAsync(trb + cc.n, 0, sizeof(int64_t), ctx->stream));
  k_tc_bitmap<<<grid_for(32ll * A->n_rows, 256), 256, 0, ctx->stream>>>(A->n_rows, A->row_p, A->col, d_rcl, 1, W, bma);
  LAMB_LAUNCHED(ctx);
  k_tc_bitmap<<<grid_for(32ll * B->n_rows, 256), 256, 0, ctx->stream>>>(B->n_rows, B->row_p, B->col, d_ccl, 0, W, bmb);
  LAMB_LAUNCHED(ctx);
  k_tc_word_prefix<<<grid_for(32ll * rc.n, 256), 256, 0, ctx->stream>>>(rc.n, W, bma, A->col_bs, wra, tra);
  LAMB_LAUNCHED(ctx);
  k_tc_word_prefix<<<grid_for(32ll * cc.n, 256), 256, 0, ctx->stream>>>(cc.n, W, bmb, B->row_bs, wrb, trb);
  LAMB_LAUNCHED(ctx);
  LAMB_TRY(exclusive_scan_i64(ctx, tra, basea, rc.n + 1));
  LAMB_TRY(exclusive_scan_i64(ctx, trb, baseb, cc.n + 1));
  // ---- tiles: cluster pairs holding a C block ----
  const int64_t n_map = (int64_t)rc.n * cc.n;
  int64_t *flag, *pos;
  LAMB_TRY(m.alloc(&flag, n_map + 1)); LAMB_TRY(m.alloc(&pos, n_map + 1));
  LAMB_CUDA(ctx, cudaMemsetAsync(flag, 0, sizeof(int64_t) * (size_t)(n_map + 1), ctx->stream));
  k_tc_tile_flags<<<grid_for(32ll * C->n_rows, 256), 256, 0, ctx->stream>>>(C->n_rows, C->row_p, C->col, d_rcl, d_ccl,
                                                                         cc.n, flag);
  LAMB_LAUNCHED(ctx);
  LAMB_TRY(exclusive_scan_i64(ctx, flag, pos, n_map + 1));
  // panel rows of A and B and the tile count in one read-back
  int64_t h_sizes[3] = {0, 0, 0};
  LAMB_CUDA(ctx, cudaMemcpyAsync(&h_sizes[0], basea + rc.n, sizeof(int64_t), cudaMemcpyDeviceToHost, ctx->stream));
  LAMB_CUDA(ctx, cudaMemcpyAsync(&h_sizes[1], baseb + cc.n, sizeof(int64_t), cudaMemcpyDeviceToHost, ctx->stream));
  LAMB_CUDA(ctx, cudaMemcpyAsync(&h_sizes[2], pos + n_map, sizeof(int64_t), cudaMemcpyDeviceToHost, ctx->stream));
  LAMB_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  const int64_t ra = h_sizes[0], rb = h_sizes[1], n_tiles = h_sizes[2];
  if (ra + 1 > kRowMask || rb + 1 > INT_MAX) return LAMB_GPU_OK;  // panel rows beyond the entry format: not run
  // ---- digit panels (one zero row at the end of each plane for padding reads) ----
  const int64_t plane_a = ((ra + 1) * 128 + 255) & ~255ll, plane_b = ((rb + 1) * 64 + 255) & ~255ll;
  int8_t *pan_a = nullptr, *pan_b = nullptr;
  LAMB_TRY(scratch(ctx, kScrPlaneA, plane_a * kS, &pan_a));
  LAMB_TRY(scratch(ctx, kScrPlaneB, plane_b * kS, &pan_b));
  LAMB_CUDA(ctx, cudaMemsetAsync(pan_a, 0, (size_t)(plane_a * kS), ctx->stream));
  LAMB_CUDA(ctx, cudaMemsetAsync(pan_b, 0, (size_t)(plane_b * kS), ctx->stream));
  k_tc_digits_a<<<grid_for(32ll * kDigitWays * A->n_rows, 256), 256, 0, ctx->stream>>>(
      A->n_rows, A->row_p, A->col, A->off, A->row_bs, A->col_bs, A->data, d_rcl, d_roff, W, bma, wra, basea, mp.rbase,
      mp.ea, plane_a, pan_a);
  LAMB_LAUNCHED(ctx);
  k_tc_digits_b<<<grid_for(32ll * kDigitWays * B->n_rows, 256), 256, 0, ctx->stream>>>(
      B->n_rows, B->row_p, B->col, B->off, B->row_bs, B->col_bs, B->data, d_ccl, d_coff, W, bmb, wrb, baseb, mp.cbase,
      mp.eb, plane_b, pan_b);
  LAMB_LAUNCHED(ctx);
  // ---- tile list, C block lists, inner lists ----
  int2* tiles;
  int32_t* krows;
  int64_t *ecnt, *ebase, *lcnt, *lbase;
  int4* blist;
  LAMB_TRY(m.alloc(&tiles, n_tiles));
  LAMB_TRY(m.alloc(&lcnt, n_tiles + 1));
  LAMB_TRY(m.alloc(&lbase, n_tiles + 1));
  LAMB_TRY(m.alloc(&blist, C->nnz));
  LAMB_TRY(m.alloc(&krows, n_tiles));
  LAMB_TRY(m.alloc(&ecnt, n_tiles + 1));
  LAMB_TRY(m.alloc(&ebase, n_tiles + 1));
  k_tc_tile_list<<<grid_for(n_map, 256), 256, 0, ctx->stream>>>(n_map, cc.n, flag, pos, tiles);
  LAMB_LAUNCHED(ctx);
  LAMB_CUDA(ctx, cudaMemsetAsync(lcnt, 0, sizeof(int64_t) * (size_t)(n_tiles + 1), ctx->stream));
  k_tc_tile_blocks<false><<<grid_for(32ll * C->n_rows, 256), 256, 0, ctx->stream>>>(
      C->n_rows, C->row_p, C->col, C->off, C->row_bs, d_rcl, d_roff, d_ratom, d_ccl, d_catom, cc.n, pos, lcnt, nullptr,
      nullptr);
  LAMB_LAUNCHED(ctx);
  LAMB_TRY(exclusive_scan_i64(ctx, lcnt, lbase, n_tiles + 1));
  LAMB_CUDA(ctx, cudaMemsetAsync(lcnt, 0, sizeof(int64_t) * (size_t)(n_tiles + 1), ctx->stream));
  k_tc_tile_blocks<true><<<grid_for(32ll * C->n_rows, 256), 256, 0, ctx->stream>>>(
      C->n_rows, C->row_p, C->col, C->off, C->row_bs, d_rcl, d_roff, d_ratom, d_ccl, d_catom, cc.n, pos, lcnt, lbase,
      blist);
  LAMB_LAUNCHED(ctx);
  LAMB_CUDA(ctx, cudaMemsetAsync(ecnt + n_tiles, 0, sizeof(int64_t), ctx->stream));
  k_tc_tile_k<false><<<grid_for(32ll * n_tiles, 256), 256, 0, ctx->stream>>>(
      n_tiles, tiles, W, bma, bmb, wra, wrb, basea, baseb, A->col_bs, ecnt, krows, nullptr, nullptr);
  LAMB_LAUNCHED(ctx);
  LAMB_TRY(exclusive_scan_i64(ctx, ecnt, ebase, n_tiles + 1));
  // {largest entry count, largest K, stages, entries} in one read-back
  unsigned long long* d_stats;
  LAMB_TRY(m.alloc(&d_stats, 4));
  LAMB_CUDA(ctx, cudaMemsetAsync(d_stats, 0, 4 * sizeof(unsigned long long), ctx->stream));
  k_tc_tile_stats<<<grid_for(n_tiles, 256), 256, 0, ctx->stream>>>(n_tiles, ecnt, krows, d_stats);
  LAMB_LAUNCHED(ctx);
  LAMB_CUDA(ctx, cudaMemcpyAsync(d_stats + 3, ebase + n_tiles, sizeof(int64_t), cudaMemcpyDeviceToDevice, ctx->stream));
  unsigned long long h_stats[4] = {0, 0, 0, 0};
  LAMB_CUDA(ctx, cudaMemcpyAsync(h_stats, d_stats, sizeof(h_stats), cudaMemcpyDeviceToHost, ctx->stream));
  LAMB_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  const int64_t max_ent = (int64_t)h_stats[0], max_rows = (int64_t)h_stats[1], n_ent = (int64_t)h_stats[3];
  *tensor_ops = (double)h_stats[2] * (kS * (kS + 1) / 2) * 2.0 * kM * kN * kK;
  if (max_ent > kMaxEnt || max_rows > kMaxKRows) return LAMB_GPU_OK;  // outside the kernel's limits: not run
  uint2* ent;
  LAMB_TRY(m.alloc(&ent, n_ent));
  k_tc_tile_k<true><<<grid_for(32ll * n_tiles, 256), 256, 0, ctx->stream>>>(
      n_tiles, tiles, W, bma, bmb, wra, wrb, basea, baseb, A->col_bs, nullptr, nullptr, ebase, ent);
  LAMB_LAUNCHED(ctx);
  if (ev_prepared) LAMB_CUDA(ctx, cudaEventRecord(ev_prepared, ctx->stream));
  // ---- the tile kernel ----
  int* d_err;
  LAMB_TRY(m.alloc(&d_err, 1));
  LAMB_CUDA(ctx, cudaMemsetAsync(d_err, 0, sizeof(int), ctx->stream));
  TcArgs g{};
  g.tiles = tiles; g.n_tiles = n_tiles; g.ent_base = ebase; g.ent_cnt = ecnt; g.krows = krows; g.ent = ent;
  g.pan_a = pan_a; g.plane_a = plane_a; g.pan_b = pan_b; g.plane_b = plane_b;
  g.rc_first = d_rcf; g.rc_atoms = d_rca; g.cc_first = d_ccf; g.cc_atoms = d_cca;
  g.row_bs = C->row_bs; g.col_bs = C->col_bs; g.rbase = mp.rbase; g.cbase = mp.cbase; g.ea = mp.ea; g.eb = mp.eb;
  g.blist = blist; g.lbase = lbase; g.c_data = C->data; g.c_nrm = c_nrm; g.err = d_err;
  g.rc_exp = d_rc_exp; g.rc_row = d_rc_row; g.cc_exp = d_cc_exp; g.cc_ab = d_cc_ab;
  LAMB_CUDA(ctx, cudaFuncSetAttribute(k_tc_tiles, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmemBytes));
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx->device);
  const int grid = (int)std::min<int64_t>(n_tiles, sms);
  k_tc_tiles<<<grid, kTileThreads, kSmemBytes, ctx->stream>>>(g);
  LAMB_LAUNCHED(ctx);
  int h_err = 0;
  LAMB_CUDA(ctx, cudaMemcpyAsync(&h_err, d_err, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  LAMB_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  if (h_err)
    return fail(ctx, LAMB_LEVEL_FAILURE, LAMB_TYPE_INTERNAL_ERROR,
                "mixed: tensor-core tile kernel stopped (code " + std::to_string(h_err) + ")");
  *ran = true;
  return LAMB_GPU_OK;
}

}  // namespace lamb

// ---- throughput probe of the tile kernel's instruction -------------------------------------
namespace lamb {
namespace tc {

// One CTA per SM: lane 0 of warp 0 issues `iters` rounds of tcgen05.mma
// kind::i8 (M = 128, K = 32, operands from one zeroed shared-memory stage),
// then waits for their completion (bounded).  N = 64 or 256: S(S+1)/2 MMAs
// of that width a round.  N = 0: the tile kernel's stage, the same nine
// MMAs (one per A digit plane and run of up to four B digit planes, N = 64
// to 256) with the same descriptors.
template <int N>
__global__ void __launch_bounds__(128, 1) k_tc_probe(int iters, int* err) {
  extern __shared__ unsigned char smem_raw[];
  // 1024-byte aligned base by pointer arithmetic on the shared array, so that
  // the compiler keeps the shared state space (shared loads and stores, not
  // generic ones)
  unsigned char* base = smem_raw + ((1024u - (smem_u32(smem_raw) & 1023u)) & 1023u);
  __shared__ unsigned long long bar;
  __shared__ uint32_t tmem_base;
  __shared__ int abort_flag;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int i = threadIdx.x; i < (N == 0 ? kStageBytes : kStageA + N * kK * kS) / 16; i += blockDim.x)
    reinterpret_cast<int4*>(base)[i] = make_int4(0, 0, 0, 0);
  if (threadIdx.x == 0) {
    bar_init(&bar, 1);
    abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_base)),
                 "r"(kTmemCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  fence_async_smem();
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = tmem_base;
  if (warp == 0) {
    if (lane == 0) {
      constexpr uint32_t idesc = (2u << 4) | (1u << 7) | (1u << 10) | (1u << 15) | (1u << 16) |
                                 ((uint32_t)(N >> 3) << 17) | ((uint32_t)(kM >> 4) << 24);
      const uint32_t sa = smem_u32(base), sb = sa + kStageA;
      // B rows of N bytes: 64-byte swizzle for N = 64, 128-byte for N >= 128 (one atom of 128 per 128 columns)
      const uint32_t bsw = N == 64 ? 4u : 2u, bsbo = N == 64 ? 512u : 1024u, blbo = N == 64 ? 64u : 4096u;
      const int levels = N <= 64 ? kS : 2;  // 512 tensor-memory columns hold 512 / N accumulators
      if (N == 0) {
        for (int it = 0; it < iters; ++it)
#pragma unroll
          for (int p = 0; p < kS; ++p) {
            const uint64_t da = smem_desc(sa + p * kPlaneA, 128, 1024, 2);
#pragma unroll
            for (int q0 = 0; q0 < kS - p; q0 += 4) {
              const int nq = (kS - p - q0) < 4 ? (kS - p - q0) : 4;
              const uint64_t db = smem_desc(sb + q0 * kPlaneB, kPlaneB, 512, 4);
              mma_i8(tmem + (uint32_t)(64 * (p + q0)), da, db, idesc_i8(64 * nq), 1u);
            }
          }
      } else
      for (int it = 0; it < iters; ++it)
        for (int L = 0; L < kS; ++L)
          for (int p = 0; p <= L; ++p) {
            const uint64_t da = smem_desc(sa + p * kPlaneA, 128, 1024, 2);
            const uint64_t db = smem_desc(sb + (L - p) * (N * kK), blbo, bsbo, bsw);
            asm volatile(
                "{\n\t.reg .pred q;\n\tsetp.ne.b32 q, %4, 0;\n\t"
                "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, q;\n\t}" ::"r"(tmem + (uint32_t)(N * (L % levels))),
                "l"(da), "l"(db), "r"(idesc), "r"(1u)
                : "memory");
          }
      mma_commit(&bar);
    }
    __syncwarp();
    const uint64_t t0 = now_ns();
    while (!bar_try(&bar, 0)) {
      if (now_ns() - t0 > 4000000000ull) {
        atomicOr(err, 1);
        break;
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols) : "memory");
}

template <int N>
static int32_t probe_n(int device, int reps, double* tops) {
  *tops = 0.0;
  if (cudaSetDevice(device) != cudaSuccess) return make_status(LAMB_LEVEL_FAILURE, LAMB_TYPE_EXTERNAL_ERROR);
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  const size_t smem = (N == 0 ? (size_t)kStageBytes : (size_t)kStageA + (size_t)N * kK * kS) + 1024;
  if (cudaFuncSetAttribute(k_tc_probe<N>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
    return make_status(LAMB_LEVEL_FAILURE, LAMB_TYPE_EXTERNAL_ERROR);
  int* err = nullptr;
  if (cudaMalloc(&err, sizeof(int)) != cudaSuccess) return make_status(LAMB_LEVEL_MEMORY, LAMB_TYPE_EXTERNAL_ERROR);
  cudaMemset(err, 0, sizeof(int));
  const int iters = 2000;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  k_tc_probe<N><<<sms, 128, smem>>>(10, err);  // warm-up
  float best = 1e30f;
  for (int r = 0; r < std::max(reps, 1); ++r) {
    cudaEventRecord(e0);
    k_tc_probe<N><<<sms, 128, smem>>>(iters, err);
    cudaEventRecord(e1);
    cudaEventSynchronize(e1);
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    best = std::min(best, ms);
  }
  int h_err = 0;
  const cudaError_t ce = cudaMemcpy(&h_err, err, sizeof(int), cudaMemcpyDeviceToHost);
  cudaFree(err);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (ce != cudaSuccess || h_err) return make_status(LAMB_LEVEL_FAILURE, LAMB_TYPE_EXTERNAL_ERROR);
  const double ops = 2.0 * kM * (N == 0 ? kN : N) * kK * (kS * (kS + 1) / 2) * (double)iters * sms;
  *tops = ops / (best * 1e-3) / 1e12;
  return LAMB_GPU_OK;
}

}  // namespace tc
}  // namespace lamb

// int8 tensor-core throughput of tcgen05.mma kind::i8, M = 128, K = 32, for
// N = 64, N = 256 (the widest instruction), or n = 0: the tile kernel's
// stage of nine MMAs of N = 64 to 256.
extern "C" int32_t lamb_probe_int8_tcgen05_tops(int32_t device, int32_t n, int32_t reps, double* tops) {
  if (!tops) return lamb::make_status(LAMB_LEVEL_FAILURE, LAMB_TYPE_WRONG_ARGS);
  if (n == 0) return lamb::tc::probe_n<0>(device, reps, tops);
  if (n == 64) return lamb::tc::probe_n<64>(device, reps, tops);
  if (n == 256) return lamb::tc::probe_n<256>(device, reps, tops);
  return lamb::make_status(LAMB_LEVEL_FAILURE, LAMB_TYPE_WRONG_ARGS);
}
