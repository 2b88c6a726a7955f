/*
 * langevin_b200_diag.h — measurement helpers of the B200 Langevin engine (not part
 * of the simulation interface; the benchmark uses them to measure the roofline
 * denominator on the same GPU and in the same process as the timed kernels).
 * These have no counterpart in the reference.
 */
#ifndef LANGEVIN_B200_DIAG_H
#define LANGEVIN_B200_DIAG_H

#include "langevin_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Issue rate of independent FP32 FMA chains over the whole GPU: thread-level
 * FMA instructions per second (the SM instruction-issue ceiling for FP32 work),
 * measured with CUDA events on the context stream; ms is the probe duration. */
int lim_probe_fma_rate(lim_ctx* ctx, double* thread_fma_per_s, double* ms);

/* Issue rate of independent hardware-exponential (ex2.approx) chains over the whole
 * GPU: thread-level multi-function-unit instructions per second, the ceiling of the
 * transcendental / conversion (XU) pipe; measured like lim_probe_fma_rate. */
int lim_probe_mufu_rate(lim_ctx* ctx, double* thread_mufu_per_s, double* ms);

#ifdef __cplusplus
}
#endif
#endif /* LANGEVIN_B200_DIAG_H */
