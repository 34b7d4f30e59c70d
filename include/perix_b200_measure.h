/* perix_b200 — measurement entry points (benchmarks and profiling only; nothing on the computing path needs them).
 *
 * Each times single kernel launches with CUDA events on the context stream, with the L2 flushed before every
 * launch by writing (then reading back) flush_bytes of a scratch buffer (0 = no flush), so that a benchmark times
 * exactly one kernel from a cold L2 without host work inside the measured interval.  Same conventions and status
 * codes as include/perix_b200.h.  No counterpart in the reference.
 */
#ifndef PERIX_B200_MEASURE_H
#define PERIX_B200_MEASURE_H

#include <stddef.h>

#include "perix_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

/* nsteps explicit steps launched one at a time; every restore_every steps (0 = never) the snapshot
 * (pxb_epf_snapshot) is restored; ms[s] = CUDA-event duration of step s's kernel alone.  The blow-up guard is not
 * evaluated. */
int pxb_epf_time_steps(pxb_ctx *ctx, int nsteps, size_t flush_bytes, int restore_every, float *ms);
/* reps g-builds into the existing operator cache (same order/precision as the last pxb_gbuild); ms[r] = CUDA-event
 * duration of build r. */
int pxb_gbuild_time(pxb_ctx *ctx, int order, int precision, int reps, size_t flush_bytes, float *ms);
/* The fixed cost inside each timed step: reps launches of an empty kernel with the launch shape (grid, block,
 * dynamic shared memory, returned) of the last TMA-staged step launch, timed exactly like a step; ms[r] per launch. */
int pxb_epf_launch_floor(pxb_ctx *ctx, size_t flush_bytes, int reps, float *ms, int *grid, int *block,
                         size_t *smem);
/* reps launches of the current batched schedule, g-build (what 0) or apply (what 1, device buffers u_d -> out_d);
 * ms[r] per launch group. */
int pxb_batch_time(pxb_ctx *ctx, int what, int reps, size_t flush_bytes, const double *u_d, double *out_d, float *ms);

/* Fault-path test hook: the number of mbarrier try_wait calls the staged step kernels' consumer warps may make
 * before they give up on a tile (tries < 0 restores the default of 2^19).  With 0 every consumer wait runs out at
 * once: the block leaves its tile loop, waits (with the default budget) for its bulk copies in flight, and counts
 * the failure, which the step / rate call reports as PXB_ERR_CUDA ("a staged-copy wait ran out"); the context
 * stays usable.  Drops the captured step graphs. */
int pxb_epf_set_wait_budget(pxb_ctx *ctx, int tries);

#ifdef __cplusplus
}
#endif
#endif
