/*
 * lamb_probe.h -- measurement helper of liblamb_b200.so (not part of the
 * drop-in ABI): the FP64 tensor-pipe peak of the current GPU, used as the
 * roofline denominator of the FP64 multiply.  No reference counterpart.
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
#ifdef __cplusplus
}
#endif
#endif
