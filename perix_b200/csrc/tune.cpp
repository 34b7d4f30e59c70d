// Schedule autotuners of the explicit kernel (the time step of the device loop and the per-step rate call of the
// reference boundary) and the device-side explicit-state snapshot they run from.  Each candidate schedule is timed
// with CUDA events around its kernel launches on the context stream; the choice is cached per problem signature.
#include <algorithm>
#include <map>
#include <string>
#include <vector>

#include "k_kernels.h"
#include "pxb_context.h"
#include "tune_internal.h"

namespace pxb {
int step_args(pxb_ctx *c, int par, EpfArgs *out);
int rate_args(pxb_ctx *c, EpfArgs *out);
}  // namespace pxb

using namespace pxb;

namespace {

struct Snapshot {
    DevBuf u0, u1, health;
    int cur = 0;
    double t = 0.0;
    long long step = 0;
    bool valid = false;
};

// one snapshot per context, kept outside pxb_ctx so the hot-path state stays lean
std::vector<std::pair<pxb_ctx *, Snapshot>> g_snaps;

Snapshot &snap_of(pxb_ctx *c) {
    for (auto &kv : g_snaps)
        if (kv.first == c) return kv.second;
    g_snaps.emplace_back(c, Snapshot{});
    return g_snaps.back().second;
}

int d2d(pxb_ctx *c, void *dst, const void *src, size_t bytes) {
    PXB_CUDA_TRY(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToDevice, c->stream));
    return PXB_OK;
}

int flush_l2(pxb_ctx *c, size_t bytes, DevBuf &buf) {
    if (bytes == 0) return PXB_OK;
    if (buf.bytes < bytes) PXB_TRY(dev_alloc(c, buf, bytes));
    launch_l2_flush(buf.p, bytes, c->stream);
    return check_launch(c, "l2 flush");
}

DevBuf g_flush;

}  // namespace

int pxb::l2_flush(pxb_ctx *c, size_t bytes) { return flush_l2(c, bytes, g_flush); }

namespace {

int save_state(pxb_ctx *c, Snapshot &s) {
    EpfState &e = c->epf;
    PXB_TRY(dev_alloc(c, s.u0, e.u[0].bytes));
    PXB_TRY(dev_alloc(c, s.u1, e.u[1].bytes));
    PXB_TRY(dev_alloc(c, s.health, e.health.bytes));
    PXB_TRY(d2d(c, s.u0.p, e.u[0].p, e.u[0].bytes));
    PXB_TRY(d2d(c, s.u1.p, e.u[1].p, e.u[1].bytes));
    PXB_TRY(d2d(c, s.health.p, e.health.p, e.health.bytes));
    s.cur = e.cur;
    s.t = e.t;
    s.step = e.step;
    s.valid = true;
    return sync(c);
}

int load_state(pxb_ctx *c, const Snapshot &s) {
    EpfState &e = c->epf;
    PXB_TRY(d2d(c, e.u[0].p, s.u0.p, s.u0.bytes));
    PXB_TRY(d2d(c, e.u[1].p, s.u1.p, s.u1.bytes));
    PXB_TRY(d2d(c, e.health.p, s.health.p, s.health.bytes));
    e.cur = s.cur;
    e.t = s.t;
    e.step = s.step;
    e.umax_hist.resize((size_t)std::min<long long>(s.step, (long long)e.umax_hist.size()));
    return PXB_OK;
}

// nsteps single-kernel steps of the current schedule variant, each timed alone (see pxb_epf_time_steps)
int timed_steps(pxb_ctx *c, int nsteps, size_t flush_bytes, int restore_every, const Snapshot *snap, float *ms) {
    EpfState &e = c->epf;
    if (e.graph_chunk < 1) {
        PXB_TRY(dev_alloc(c, e.umax, sizeof(unsigned long long)));
        PXB_TRY(dev_alloc(c, e.tsched, sizeof(double)));
        PXB_TRY(ensure_pinned(e.tsched_h, 64));
        e.graph_chunk = 1;
    }
    Events ev;
    PXB_TRY(ev.make(2 * (size_t)nsteps));
    double *th = static_cast<double *>(e.tsched_h.p);
    for (int s = 0; s < nsteps; ++s) {
        if (snap && restore_every > 0 && s > 0 && s % restore_every == 0) PXB_TRY(load_state(c, *snap));
        // t_{n+1} for this step (host-accumulated exactly like the reference loop)
        PXB_CUDA_TRY(cudaStreamSynchronize(c->stream));
        th[0] = e.t + e.dt;
        PXB_TRY(h2d(c, e.tsched.p, th, sizeof(double)));
        PXB_TRY(flush_l2(c, flush_bytes, g_flush));
        EpfArgs a;
        PXB_TRY(step_args(c, e.cur, &a));
        PXB_CUDA_TRY(cudaEventRecord(ev.ev[2 * (size_t)s], c->stream));
        const cudaError_t err = launch_epf(a, c->g.dim, e.precision == PXB_MIXED, EPF_STEP, e.variant, c->stream);
        if (err != cudaSuccess) return cuda_fail(err, "epf step launch");
        c->launches++;
        PXB_CUDA_TRY(cudaEventRecord(ev.ev[2 * (size_t)s + 1], c->stream));
        e.cur ^= 1;
        e.t = th[0];
        e.step++;
    }
    PXB_TRY(sync(c));
    unsigned int werr = 0;
    PXB_CUDA_TRY(cudaMemcpy(&werr, e.counters.as<unsigned long long>() + 2, sizeof(unsigned int), cudaMemcpyDeviceToHost));
    if (werr) return wait_failure(c, werr, "explicit step");
    for (int s = 0; s < nsteps; ++s) PXB_CUDA_TRY(cudaEventElapsedTime(&ms[s], ev.ev[2 * (size_t)s], ev.ev[2 * (size_t)s + 1]));
    return PXB_OK;
}

// process-wide cache of autotuned schedule choices, keyed by problem signature
std::map<std::string, int> g_tuned;

std::string signature(const pxb_ctx *c) {
    return std::to_string(c->g.dim) + ":" + std::to_string(c->epf.precision) + ":" + std::to_string(c->g.n) + ":" +
           std::to_string(c->g.nb) + ":" + std::to_string(c->g.max_family);
}

}  // namespace

namespace pxb {
int epf_timed_steps(pxb_ctx *c, int nsteps, size_t flush_bytes, int restore_every, bool from_snapshot, float *ms) {
    Snapshot &s = snap_of(c);
    return timed_steps(c, nsteps, flush_bytes, restore_every, from_snapshot && s.valid ? &s : nullptr, ms);
}

// called when a context is destroyed: release its snapshot
void drop_snapshot(pxb_ctx *c) {
    for (auto it = g_snaps.begin(); it != g_snaps.end(); ++it)
        if (it->first == c) {
            g_snaps.erase(it);
            return;
        }
}
}  // namespace pxb

extern "C" int pxb_epf_snapshot(pxb_ctx *c) {
    if (!c || !c->epf.ready || !c->epf.started) return fail(PXB_ERR_STATE, "pxb_epf_snapshot: no running explicit state");
    return save_state(c, snap_of(c));
}

extern "C" int pxb_epf_restore(pxb_ctx *c) {
    if (!c || !c->epf.ready) return fail(PXB_ERR_STATE, "pxb_epf_restore: no explicit state");
    Snapshot &s = snap_of(c);
    if (!s.valid) return fail(PXB_ERR_STATE, "pxb_epf_restore: no snapshot taken");
    return load_state(c, s);
}

extern "C" int pxb_epf_set_variant(pxb_ctx *c, int variant) {
    if (!c || !c->epf.ready) return fail(PXB_ERR_STATE, "pxb_epf_set_variant: call pxb_epf_setup first");
    if (variant < 0 || variant >= kEpfVariants) return fail(PXB_ERR_INVALID, "pxb_epf_set_variant: no such variant");
    if (!epf_variant_fits(c->g.dim, variant, c->g.max_family))
        return fail(PXB_ERR_UNSUPPORTED, "pxb_epf_set_variant: families too large for this tile size");
    c->epf.variant = variant;
    return PXB_OK;
}

extern "C" int pxb_epf_variant_count(void) { return kEpfVariants; }

extern "C" int pxb_epf_get_variant(pxb_ctx *c, int *variant, int *lanes_per_node) {
    if (!c || !c->epf.ready || !variant) return fail(PXB_ERR_STATE, "pxb_epf_get_variant: call pxb_epf_setup first");
    *variant = c->epf.variant;
    if (lanes_per_node) *lanes_per_node = epf_lanes_per_node(c->g.dim, c->epf.variant);
    return PXB_OK;
}

// Times every schedule variant for `steps` steps (L2 flushed before each) from a private copy of the current
// state, restores the state, selects the fastest and caches the choice for this problem signature.
extern "C" int pxb_epf_autotune(pxb_ctx *c, int steps, size_t flush_bytes, int use_cache, int *best,
                                float *ms_per_variant) {
    if (!c || !c->epf.ready || !c->epf.started) return fail(PXB_ERR_STATE, "pxb_epf_autotune: call pxb_epf_start first");
    if (steps <= 0) return fail(PXB_ERR_INVALID, "pxb_epf_autotune: steps must be > 0");
    const std::string key = signature(c);
    auto hit = g_tuned.find(key);
    if (use_cache && hit != g_tuned.end()) {
        c->epf.variant = hit->second;
        if (best) *best = hit->second;
        return PXB_OK;
    }
    Snapshot keep;
    PXB_TRY(save_state(c, keep));
    std::vector<float> ms((size_t)std::max(steps, 2));
    float best_ms = 1e30f;
    int best_v = c->epf.variant;
    for (int v = 0; v < kEpfVariants; ++v) {
        if (!epf_variant_fits(c->g.dim, v, c->g.max_family)) {
            if (ms_per_variant) ms_per_variant[v] = -1.f;
            continue;
        }
        c->epf.variant = v;
        // two untimed steps first: a kernel's first launch in a process also loads its module
        PXB_TRY(load_state(c, keep));
        PXB_TRY(timed_steps(c, 2, 0, 0, nullptr, ms.data()));
        PXB_TRY(load_state(c, keep));
        PXB_TRY(timed_steps(c, steps, flush_bytes, 0, nullptr, ms.data()));
        float mean = 0.f;
        for (int k = 0; k < steps; ++k) mean += ms[(size_t)k];
        mean /= (float)steps;
        if (ms_per_variant) ms_per_variant[v] = mean;
        if (mean < best_ms) { best_ms = mean; best_v = v; }
    }
    PXB_TRY(load_state(c, keep));
    PXB_TRY(sync(c));
    c->epf.variant = best_v;
    g_tuned[key] = best_v;
    if (best) *best = best_v;
    return PXB_OK;
}




// Times the per-step rate call's kernel (RATE epilogue: damage, force, acceleration out) of every schedule variant
// that fits, at the caller's displacement u (host, n*dim), reps launches each after one untimed launch; the bond
// health and the counters are restored before every launch and at the end, so the state is as before the call.
// Selects the fastest and caches it per problem signature (separately from the time-step choice).
extern "C" int pxb_epf_autotune_rate(pxb_ctx *c, const double *u, int reps, int use_cache, int *best,
                                     float *ms_per_variant) {
    if (!c || !c->g.ready || !c->epf.ready) return fail(PXB_ERR_STATE, "pxb_epf_autotune_rate: call pxb_epf_setup first");
    if (!u || reps <= 0) return fail(PXB_ERR_INVALID, "pxb_epf_autotune_rate: need u and reps > 0");
    EpfState &e = c->epf;
    const std::string key = signature(c) + ":rate";
    auto hit = g_tuned.find(key);
    if (use_cache && hit != g_tuned.end()) {
        e.variant = hit->second;
        if (best) *best = hit->second;
        return PXB_OK;
    }
    DevBuf health, counters;
    PXB_TRY(dev_alloc(c, health, e.health.bytes));
    PXB_TRY(dev_alloc(c, counters, e.counters.bytes));
    PXB_TRY(d2d(c, health.p, e.health.p, e.health.bytes));
    PXB_TRY(d2d(c, counters.p, e.counters.p, e.counters.bytes));
    PXB_TRY(h2d(c, e.u[e.cur].p, u, sizeof(double) * (size_t)c->g.n * c->g.dim));
    auto restore = [&]() -> int {
        PXB_TRY(d2d(c, e.health.p, health.p, health.bytes));
        return d2d(c, e.counters.p, counters.p, counters.bytes);
    };
    Events ev;
    PXB_TRY(ev.make(2 * (size_t)reps));
    const int keep = e.variant;
    float best_ms = 1e30f;
    int best_v = keep;
    for (int v = 0; v < kEpfVariants; ++v) {
        if (!epf_variant_fits(c->g.dim, v, c->g.max_family)) {
            if (ms_per_variant) ms_per_variant[v] = -1.f;
            continue;
        }
        e.variant = v;
        EpfArgs a;
        PXB_TRY(rate_args(c, &a));
        // one untimed launch first: a kernel's first launch in a process also loads its module
        for (int r = -1; r < reps; ++r) {
            PXB_TRY(restore());
            if (r >= 0) PXB_CUDA_TRY(cudaEventRecord(ev.ev[2 * (size_t)r], c->stream));
            const cudaError_t err = launch_epf(a, c->g.dim, e.precision == PXB_MIXED, EPF_RATE, v, c->stream);
            if (err != cudaSuccess) return cuda_fail(err, "rate autotune launch");
            c->launches++;
            if (r >= 0) PXB_CUDA_TRY(cudaEventRecord(ev.ev[2 * (size_t)r + 1], c->stream));
        }
        PXB_TRY(sync(c));
        unsigned int werr = 0;
        PXB_CUDA_TRY(cudaMemcpy(&werr, e.counters.as<unsigned long long>() + 2, sizeof(unsigned int),
                                cudaMemcpyDeviceToHost));
        if (werr) {
            e.variant = keep;
            PXB_TRY(restore());
            PXB_TRY(sync(c));
            return fail(PXB_ERR_CUDA, "pxb_epf_autotune_rate: a staged-copy wait ran out");
        }
        float mean = 0.f;
        for (int r = 0; r < reps; ++r) {
            float ms = 0.f;
            PXB_CUDA_TRY(cudaEventElapsedTime(&ms, ev.ev[2 * (size_t)r], ev.ev[2 * (size_t)r + 1]));
            mean += ms;
        }
        mean /= (float)reps;
        if (ms_per_variant) ms_per_variant[v] = mean;
        if (mean < best_ms) { best_ms = mean; best_v = v; }
    }
    PXB_TRY(restore());
    PXB_TRY(sync(c));
    e.variant = best_v;
    g_tuned[key] = best_v;
    if (best) *best = best_v;
    return PXB_OK;
}
