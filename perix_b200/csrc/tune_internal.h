// Internal pieces shared by the autotuners (tune.cpp) and the measurement entry points (measure.cpp): CUDA-event
// sets, the timed loop of single explicit steps and the timing of one batch launch group.
#pragma once

#include <cuda_runtime.h>

#include <vector>

#include "pxb_context.h"

namespace pxb {

struct Events {
    std::vector<cudaEvent_t> ev;
    Events() = default;
    Events(const Events &) = delete;
    Events &operator=(const Events &) = delete;
    ~Events() {
        for (auto e : ev)
            if (e) cudaEventDestroy(e);
    }
    int make(size_t n) {
        ev.resize(n, nullptr);
        for (auto &e : ev) PXB_CUDA_TRY(cudaEventCreate(&e));
        return PXB_OK;
    }
};

// nsteps explicit steps of the current schedule launched one at a time, the L2 flushed (flush_bytes, 0 = none)
// before each and, with from_snapshot, the context's snapshot (pxb_epf_snapshot) restored every restore_every
// steps; ms[s] = CUDA-event duration of step s's kernel alone
int epf_timed_steps(pxb_ctx *c, int nsteps, size_t flush_bytes, int restore_every, bool from_snapshot, float *ms);
// relaunch the g-build into the existing operator cache (same order/precision), no host synchronisation
int gbuild_launch_only(pxb_ctx *c, int order, int precision);
// reps launches of the current batch g-build (what 0) or apply (what 1) schedule, ms[r] per launch group
int batch_time(pxb_ctx *c, int what, int reps, size_t flush_bytes, const double *u_d, double *out_d, float *ms);

}  // namespace pxb
