// Measurement entry points (include/perix_b200_measure.h): CUDA-event timing of single kernel launches on the
// context stream with the L2 flushed before each, so a benchmark can time exactly one kernel without host work
// inside the measured interval, and the launch-floor probe.  None of this is on the computing path.
#include <string>
#include <vector>

#include "../../include/perix_b200_measure.h"
#include "k_kernels.h"
#include "pxb_context.h"
#include "tune_internal.h"

using namespace pxb;

// Runs nsteps explicit steps one launch at a time; before each launch the L2 is flushed by writing
// flush_bytes (0 = no flush) and, every restore_every steps (0 = never), the snapshot is restored.  ms[s]
// receives the CUDA-event duration of step s's kernel alone.  The blow-up guard is not evaluated here.
extern "C" int pxb_epf_time_steps(pxb_ctx *c, int nsteps, size_t flush_bytes, int restore_every, float *ms) {
    if (!c || !c->epf.ready || !c->epf.started) return fail(PXB_ERR_STATE, "pxb_epf_time_steps: call pxb_epf_start first");
    if (nsteps <= 0 || !ms) return fail(PXB_ERR_INVALID, "pxb_epf_time_steps: bad arguments");
    return epf_timed_steps(c, nsteps, flush_bytes, restore_every, true, ms);
}

// The fixed cost inside a timed step: an empty kernel with the launch shape of the last staged step launch
// (grid, block, dynamic shared memory), timed exactly like a step (L2 flushed, CUDA events around the launch).
extern "C" int pxb_epf_launch_floor(pxb_ctx *c, size_t flush_bytes, int reps, float *ms, int *grid, int *block,
                                    size_t *smem) {
    if (!c || reps <= 0 || !ms) return fail(PXB_ERR_INVALID, "pxb_epf_launch_floor: bad arguments");
    const LaunchShape sh = epf_tma_last_shape();
    if (sh.grid <= 0) return fail(PXB_ERR_STATE, "pxb_epf_launch_floor: no staged step launched yet");
    Events ev;
    PXB_TRY(ev.make(2 * (size_t)reps));
    for (int r = 0; r < reps; ++r) {
        PXB_TRY(l2_flush(c, flush_bytes));
        PXB_CUDA_TRY(cudaEventRecord(ev.ev[2 * (size_t)r], c->stream));
        PXB_CUDA_TRY(launch_empty(sh.grid, sh.block, sh.smem, c->stream));
        PXB_CUDA_TRY(cudaEventRecord(ev.ev[2 * (size_t)r + 1], c->stream));
    }
    PXB_TRY(sync(c));
    for (int r = 0; r < reps; ++r) PXB_CUDA_TRY(cudaEventElapsedTime(&ms[r], ev.ev[2 * (size_t)r], ev.ev[2 * (size_t)r + 1]));
    if (grid) *grid = sh.grid;
    if (block) *block = sh.block;
    if (smem) *smem = sh.smem;
    return PXB_OK;
}

// Times `reps` g-builds (order, precision) of the current geometry, L2 flushed before each; ms[r] per build.
extern "C" int pxb_gbuild_time(pxb_ctx *c, int order, int precision, int reps, size_t flush_bytes, float *ms) {
    if (!c || !c->g.ready) return fail(PXB_ERR_STATE, "pxb_gbuild_time: geometry not set");
    if (reps <= 0 || !ms) return fail(PXB_ERR_INVALID, "pxb_gbuild_time: bad arguments");
    Events ev;
    PXB_TRY(ev.make(2 * (size_t)reps));
    for (int r = 0; r < reps; ++r) {
        PXB_TRY(l2_flush(c, flush_bytes));
        PXB_CUDA_TRY(cudaEventRecord(ev.ev[2 * (size_t)r], c->stream));
        PXB_TRY(gbuild_launch_only(c, order, precision));
        PXB_CUDA_TRY(cudaEventRecord(ev.ev[2 * (size_t)r + 1], c->stream));
    }
    PXB_TRY(sync(c));
    for (int r = 0; r < reps; ++r) PXB_CUDA_TRY(cudaEventElapsedTime(&ms[r], ev.ev[2 * (size_t)r], ev.ev[2 * (size_t)r + 1]));
    return PXB_OK;
}

// Times `reps` launches of the current schedule of the batched g-build (what 0) or apply (what 1, on the field
// u_d into out_d, device pointers), the L2 flushed before each; ms[r] per launch group.
extern "C" int pxb_batch_time(pxb_ctx *c, int what, int reps, size_t flush_bytes, const double *u_d, double *out_d,
                              float *ms) {
    return batch_time(c, what, reps, flush_bytes, u_d, out_d, ms);
}
