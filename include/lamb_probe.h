/*
 * lamb_probe.h -- measurement helper of liblamb_b200.so (not part of the
 * drop-in ABI): the FP64, int8 and bf16 tensor-pipe peaks of the current GPU;
 * the first two are the roofline denominators of the FP64 and the int8-slice
 * multiplies.  No reference counterpart.
 */
#ifndef LAMB_PROBE_H
#define LAMB_PROBE_H
#include <stdint.h>
#include "lamb_gpu.h"
#ifdef __cplusplus
extern "C" {
#endif
/* Best of `reps` launches of a DMMA (mma.m8n8k4.f64) throughput loop on
 * `device`; writes TFLOP/s.  Allocates 8 bytes per thread of the grid. */
LAMB_API int32_t lamb_probe_fp64_tflops(int32_t device, int32_t reps, double* tflops);
/* Same for the integer tensor pipe as the int8-slice kernel drives it
 * (mma.m16n8k32.s8.s8.s32 through mma.sync); writes TOP/s (1 op = 1 multiply
 * or 1 add).  Allocates 4 bytes per thread of the grid. */
LAMB_API int32_t lamb_probe_int8_tops(int32_t device, int32_t reps, double* tops);
/* Same for bf16 operands with FP32 accumulation (mma.m16n8k16.f32.bf16.bf16.f32
 * through mma.sync), the alternative slice format; writes TFLOP/s.  Allocates
 * 4 bytes per thread of the grid. */
LAMB_API int32_t lamb_probe_bf16_tflops(int32_t device, int32_t reps, double* tflops);
/* int8 throughput of the 5th-generation tensor cores as the mixed multiply's
 * tile kernel drives them: one CTA per SM issues tcgen05.mma kind::i8
 * (M = 128, K = 32, N = n: 64 or 256, the widest; n = 0 issues the tile
 * kernel's own stage, nine MMAs of N = 64 to 256 covering the 21 digit
 * pairs) from shared memory into tensor-memory accumulators; best of
 * `reps` launches, TOP/s (1 op = 1 multiply or 1 add).  Allocates 4 bytes. */
LAMB_API int32_t lamb_probe_int8_tcgen05_tops(int32_t device, int32_t n, int32_t reps, double* tops);
#ifdef __cplusplus
}
#endif
#endif
