// C-ABI for batched clouds: many independent node clouds (2D and 3D mixed, families of uneven size) share one
// concatenated geometry and are built / applied by single persistent launches over a task table.
//
// The per-cloud semantics are those of the single-geometry entry points (pxb_gbuild / pxb_apply at order 2):
// the reference builds one PDMeshData per cloud (tests/ExplicitPDDOFracElementTests.cpp:35-64) and runs
// PDOperators::calcAMatrixCompute / calcOperatorsCompute (src/PDOperators/CalcPDOperators.cpp:108-354) on it.
#include <algorithm>
#include <climits>
#include <limits>
#include <string>
#include <vector>

#include "k_kernels.h"
#include "pxb_context.h"
#include "tune_internal.h"
#include "fam_builder.h"

using namespace pxb;

namespace {

constexpr int kTaskNodes2 = 32;  // nodes per task: ~25 bonds each in 2D (small tasks keep small batches parallel)
constexpr int kTaskNodes3 = 16;  // ~100 bonds each in 3D

int nop_of_dim(int dim) { return dim == 3 ? 9 : 5; }

int need_batch(pxb_ctx *c, const char *who, bool built) {
    if (!c) return fail(PXB_ERR_INVALID, std::string(who) + ": NULL context");
    if (!c->batch.ready) return fail(PXB_ERR_STATE, std::string(who) + ": no batch (call pxb_batch_set)");
    if (built && !c->batch.built) return fail(PXB_ERR_STATE, std::string(who) + ": call pxb_batch_gbuild first");
    PXB_CUDA_TRY(cudaSetDevice(c->device));
    return PXB_OK;
}

BatchArgs batch_args(pxb_ctx *c) {
    BatchState &b = c->batch;
    BatchArgs a;
    a.tasks = b.tasks.as<BatchTask>();
    a.clouds = b.clouds.as<BatchCloud>();
    a.off = b.off.as<int>();
    a.nbr = b.nbr.as<int>();
    a.pos = b.pos.as<unsigned char>();
    a.vol = b.vol.as<double>();
    a.ops = b.ops.p;
    a.degenerate = b.degenerate.as<uint8_t>();
    unsigned *cnt = b.counters.as<unsigned>();
    a.n_degenerate = cnt + 2;
    a.first_degenerate = reinterpret_cast<int *>(cnt + 3);
    a.defect = (b.precision == PXB_MIXED && b.defect.p) ? b.defect.as<float>() : nullptr;
    return a;
}

// enqueue the launches of one schedule: split schedules run the 3D tasks, then the 2D tasks, each with its
// own instantiation; the others run every task in one launch
template <typename Launch>
int run_tasks(pxb_ctx *c, bool split, Launch launch, const char *what) {
    BatchState &b = c->batch;
    unsigned *cnt = b.counters.as<unsigned>();
    PXB_CUDA_TRY(cudaMemsetAsync(cnt, 0, 2 * sizeof(unsigned), c->stream));
    BatchArgs a = batch_args(c);
    if (!split) {
        a.task0 = 0;
        a.ntasks = b.ntasks;
        a.counter = cnt;
        PXB_CUDA_TRY(launch(a, 3));
        c->launches++;
        return check_launch(c, what);
    }
    if (b.ntasks3 > 0) {
        a.task0 = 0;
        a.ntasks = b.ntasks3;
        a.counter = cnt;
        PXB_CUDA_TRY(launch(a, 2));
        c->launches++;
    }
    if (b.ntasks > b.ntasks3) {
        a.task0 = b.ntasks3;
        a.ntasks = b.ntasks - b.ntasks3;
        a.counter = cnt + 1;
        PXB_CUDA_TRY(launch(a, 1));
        c->launches++;
    }
    return check_launch(c, what);
}

int gbuild_enqueue(pxb_ctx *c) {
    BatchState &b = c->batch;
    const bool mixed = b.precision == PXB_MIXED;
    const int v = b.gvariant;
    return run_tasks(c, batch_gbuild_schedule(v).split,
                     [&](const BatchArgs &a, int dims) { return launch_gbuild_batch(a, mixed, v, dims, c->stream); },
                     "batch gbuild");
}

int apply_enqueue(pxb_ctx *c, const double *u_d, double *out_d) {
    BatchState &b = c->batch;
    const bool mixed = b.precision == PXB_MIXED;
    const int v = b.avariant;
    return run_tasks(c, batch_apply_schedule(v).split,
                     [&](const BatchArgs &a0, int dims) {
                         BatchArgs a = a0;
                         a.u = u_d;
                         a.out = out_d;
                         return launch_apply_batch(a, mixed, v, dims, c->stream);
                     },
                     "batch apply");
}

}  // namespace

namespace {

// The batch tables from concatenated clouds.  neigh_id (1-based within each cloud) may be NULL: the neighbour
// array is then left zeroed for the device family build to fill.
int batch_setup(pxb_ctx *c, int nclouds, const int *dims, const int *node_off, const double *coords3, const double *vols,
                const int *neigh_off, const int *neigh_id, const double *delta, const double *dx_char, const char *who) {
    const int n = node_off[nclouds];
    for (int i = 0; i < n; ++i)
        if (neigh_off[i + 1] < neigh_off[i]) return fail(PXB_ERR_INVALID, std::string(who) + ": neigh_off not non-decreasing");
    const long long nb = neigh_off[n];
    PXB_CUDA_TRY(cudaSetDevice(c->device));
    PXB_CUDA_TRY(cudaStreamSynchronize(c->stream));
    BatchState &b = c->batch;
    b = BatchState{};
    b.nclouds = nclouds;
    b.n = n;
    b.nb = nb;
    b.h_clouds.resize((size_t)nclouds);
    // cloud table, global 0-based neighbour ids, packed positions
    std::vector<int> nbr(neigh_id ? (size_t)std::max(1LL, nb) : 0);
    long long ops_off = 0, out_off = 0, pos_off = 0, def_off = 0;
    for (int k = 0; k < nclouds; ++k) {
        BatchCloud &cd = b.h_clouds[(size_t)k];
        cd.dim = dims[k];
        cd.node0 = node_off[k];
        cd.n = node_off[k + 1] - node_off[k];
        cd.bond0 = neigh_off[cd.node0];
        cd.nb = neigh_off[cd.node0 + cd.n] - cd.bond0;
        cd.delta = delta[k];
        cd.dx_char = dx_char[k];
        cd.ops_off = ops_off;
        cd.out_off = out_off;
        cd.pos_off = pos_off;
        cd.def_off = def_off;
        const int nop = nop_of_dim(cd.dim);
        def_off += (long long)cd.n * (nop - cd.dim) * cd.dim;
        ops_off += cd.nb * nop;
        out_off += (long long)cd.n * nop;
        pos_off += ((long long)cd.n * (cd.dim == 3 ? 32 : 16) + 31) / 32 * 32;
        if (!neigh_id) continue;
        for (long long t = cd.bond0; t < cd.bond0 + cd.nb; ++t) {
            const int id = neigh_id[t];
            if (id < 1 || id > cd.n)
                return fail(PXB_ERR_INVALID, std::string(who) + ": cloud " + std::to_string(k) +
                                                 ": neighbour id out of range (ids are 1-based within the cloud)");
            nbr[(size_t)t] = cd.node0 + id - 1;
        }
    }
    b.ops_len = ops_off;
    b.out_len = out_off;
    b.def_len = def_off;
    std::vector<double> pos((size_t)(pos_off / 8), 0.0);
    for (const BatchCloud &cd : b.h_clouds) {
        double *p = pos.data() + cd.pos_off / 8;
        const int w = cd.dim == 3 ? 4 : 2;
        for (int i = 0; i < cd.n; ++i)
            for (int a = 0; a < cd.dim; ++a) p[(size_t)i * w + a] = coords3[(size_t)(cd.node0 + i) * 3 + a];
    }
    // tasks: 3D clouds first (the costlier nodes start early), then 2D
    std::vector<BatchTask> tasks;
    for (int pass = 0; pass < 2; ++pass) {
        for (int k = 0; k < nclouds; ++k) {
            const BatchCloud &cd = b.h_clouds[(size_t)k];
            if ((pass == 0) != (cd.dim == 3)) continue;
            const int step = cd.dim == 3 ? kTaskNodes3 : kTaskNodes2;
            for (int f = 0; f < cd.n; f += step) tasks.push_back({k, cd.node0 + f, std::min(step, cd.n - f), cd.dim});
        }
        if (pass == 0) b.ntasks3 = (int)tasks.size();
    }
    b.ntasks = (int)tasks.size();
    PXB_TRY(dev_upload(c, b.clouds, b.h_clouds.data(), sizeof(BatchCloud) * b.h_clouds.size()));
    PXB_TRY(dev_upload(c, b.tasks, tasks.data(), sizeof(BatchTask) * tasks.size()));
    PXB_TRY(dev_upload(c, b.off, neigh_off, sizeof(int) * ((size_t)n + 1)));
    if (neigh_id) {
        PXB_TRY(dev_upload(c, b.nbr, nbr.data(), sizeof(int) * nbr.size()));
    } else {
        PXB_TRY(dev_alloc(c, b.nbr, sizeof(int) * (size_t)std::max(1LL, nb)));
        PXB_CUDA_TRY(cudaMemsetAsync(b.nbr.p, 0, b.nbr.bytes, c->stream));
    }
    PXB_TRY(dev_upload(c, b.pos, pos.data(), sizeof(double) * std::max<size_t>(1, pos.size())));
    PXB_TRY(dev_upload(c, b.vol, vols, sizeof(double) * (size_t)n));
    PXB_TRY(dev_alloc(c, b.counters, 4 * sizeof(unsigned)));
    PXB_TRY(sync(c));
    return PXB_OK;
}

int check_clouds(int nclouds, const int *dims, const int *node_off, const double *delta, const char *who) {
    if (node_off[0] != 0) return fail(PXB_ERR_INVALID, std::string(who) + ": node offsets must start at 0");
    for (int k = 0; k < nclouds; ++k) {
        if (dims[k] != 2 && dims[k] != 3) return fail(PXB_ERR_INVALID, std::string(who) + ": dims must be 2 or 3");
        if (node_off[k + 1] <= node_off[k]) return fail(PXB_ERR_INVALID, std::string(who) + ": empty or unordered cloud");
        if (!(delta[k] > 0.0)) return fail(PXB_ERR_INVALID, std::string(who) + ": delta must be > 0");
    }
    return PXB_OK;
}

}  // namespace

extern "C" int pxb_batch_set(pxb_ctx *c, int nclouds, const int *dims, const int *node_off, const double *coords3,
                             const double *vols, const int *neigh_off, const int *neigh_id, const double *delta,
                             const double *dx_char) {
    if (!c) return fail(PXB_ERR_INVALID, "pxb_batch_set: NULL context");
    if (nclouds <= 0 || !dims || !node_off || !coords3 || !vols || !neigh_off || !neigh_id || !delta || !dx_char)
        return fail(PXB_ERR_INVALID, "pxb_batch_set: bad arguments");
    if (neigh_off[0] != 0) return fail(PXB_ERR_INVALID, "pxb_batch_set: offsets must start at 0");
    PXB_TRY(check_clouds(nclouds, dims, node_off, delta, "pxb_batch_set"));
    PXB_TRY(batch_setup(c, nclouds, dims, node_off, coords3, vols, neigh_off, neigh_id, delta, dx_char, "pxb_batch_set"));
    c->batch.ready = true;
    return PXB_OK;
}

// Families of every cloud built on the device (radius[k] = family radius of cloud k), then the batch as
// pxb_batch_set sets it.
extern "C" int pxb_batch_set_points(pxb_ctx *c, int nclouds, const int *dims, const int *node_off,
                                    const double *coords3, const double *vols, const double *radius,
                                    const double *delta, const double *dx_char) {
    if (!c) return fail(PXB_ERR_INVALID, "pxb_batch_set_points: NULL context");
    if (nclouds <= 0 || !dims || !node_off || !coords3 || !vols || !radius || !delta || !dx_char)
        return fail(PXB_ERR_INVALID, "pxb_batch_set_points: bad arguments");
    PXB_TRY(check_clouds(nclouds, dims, node_off, delta, "pxb_batch_set_points"));
    for (int k = 0; k < nclouds; ++k)
        if (!(radius[k] > 0.0)) return fail(PXB_ERR_INVALID, "pxb_batch_set_points: radius must be > 0");
    PXB_CUDA_TRY(cudaSetDevice(c->device));
    const int n = node_off[nclouds];
    std::vector<int> off((size_t)n + 1, 0);
    long long acc = 0;
    for (int k = 0; k < nclouds; ++k) {  // counts (the builders are rebuilt for the fill below)
        FamBuilder fb;
        std::vector<int> h;
        int maxf = 0;
        long long tot = 0;
        const int n0 = node_off[k], nk = node_off[k + 1] - n0;
        PXB_TRY(fb.count(c, nk, dims[k] == 3, coords3 + 3 * (size_t)n0, radius[k], h, maxf, tot));
        for (int i = 0; i < nk; ++i) off[(size_t)n0 + i + 1] = (int)(acc + h[(size_t)i + 1]);
        acc += tot;
        if (acc > std::numeric_limits<int>::max()) return fail(PXB_ERR_INVALID, "pxb_batch_set_points: more than 2^31-1 bonds");
    }
    PXB_TRY(batch_setup(c, nclouds, dims, node_off, coords3, vols, off.data(), nullptr, delta, dx_char,
                        "pxb_batch_set_points"));
    BatchState &b = c->batch;
    for (int k = 0; k < nclouds; ++k) {
        FamBuilder fb;
        std::vector<int> h;
        int maxf = 0;
        long long tot = 0;
        const int n0 = node_off[k], nk = node_off[k + 1] - n0;
        PXB_TRY(fb.count(c, nk, dims[k] == 3, coords3 + 3 * (size_t)n0, radius[k], h, maxf, tot));
        PXB_TRY(fb.fill(c, b.off.as<int>() + n0, b.nbr.as<int>(), n0));
    }
    PXB_TRY(sync(c));
    b.ready = true;
    return PXB_OK;
}

// One cloud's families (1-based ids within the cloud): neigh_off n_k + 1 entries, neigh_id neigh_off[n_k].
extern "C" int pxb_batch_get_families(pxb_ctx *c, int cloud, int *neigh_off, int *neigh_id) {
    PXB_TRY(need_batch(c, "pxb_batch_get_families", false));
    const BatchState &b = c->batch;
    if (cloud < 0 || cloud >= b.nclouds) return fail(PXB_ERR_INVALID, "pxb_batch_get_families: no such cloud");
    const BatchCloud &cd = b.h_clouds[(size_t)cloud];
    std::vector<int> off((size_t)cd.n + 1);
    PXB_TRY(d2h(c, off.data(), b.off.as<int>() + cd.node0, sizeof(int) * off.size()));
    if (neigh_id) PXB_TRY(d2h(c, neigh_id, b.nbr.as<int>() + cd.bond0, sizeof(int) * (size_t)cd.nb));
    PXB_TRY(sync(c));
    if (neigh_off)
        for (size_t i = 0; i < off.size(); ++i) neigh_off[i] = off[i] - off[0];
    if (neigh_id)
        for (long long t = 0; t < cd.nb; ++t) neigh_id[t] = neigh_id[t] - cd.node0 + 1;
    return PXB_OK;
}

extern "C" int pxb_batch_info(pxb_ctx *c, long long *nodes, long long *bonds, long long *out_len, long long *ops_len) {
    PXB_TRY(need_batch(c, "pxb_batch_info", false));
    const BatchState &b = c->batch;
    if (nodes) *nodes = b.n;
    if (bonds) *bonds = b.nb;
    if (out_len) *out_len = b.out_len;
    if (ops_len) *ops_len = b.ops_len;
    return PXB_OK;
}

extern "C" int pxb_batch_gbuild(pxb_ctx *c, int precision, int *n_degenerate, int *first_degenerate) {
    PXB_TRY(need_batch(c, "pxb_batch_gbuild", false));
    if (precision != PXB_FP64 && precision != PXB_MIXED) return fail(PXB_ERR_INVALID, "pxb_batch_gbuild: bad precision");
    BatchState &b = c->batch;
    b.built = false;
    b.precision = precision;
    const size_t es = precision == PXB_MIXED ? 4 : 8;
    PXB_TRY(dev_alloc(c, b.ops, es * (size_t)std::max(1LL, b.ops_len)));
    PXB_TRY(dev_alloc(c, b.degenerate, (size_t)b.n));
    b.defect = DevBuf{};
    if (precision == PXB_MIXED) {
        PXB_TRY(dev_alloc(c, b.defect, sizeof(float) * (size_t)std::max(1LL, b.def_len)));
        PXB_CUDA_TRY(cudaMemsetAsync(b.defect.p, 0, b.defect.bytes, c->stream));
    }
    unsigned *cnt = b.counters.as<unsigned>();
    const unsigned init[2] = {0u, (unsigned)INT_MAX};
    PXB_TRY(h2d(c, cnt + 2, init, sizeof(init)));
    PXB_TRY(gbuild_enqueue(c));
    unsigned out[2] = {0, 0};
    PXB_TRY(d2h(c, out, cnt + 2, sizeof(out)));
    PXB_TRY(sync(c));
    if (n_degenerate) *n_degenerate = (int)out[0];
    if (first_degenerate) *first_degenerate = out[0] ? (int)out[1] + 1 : 0;
    if (out[0]) {
        const int g = (int)out[1];
        int k = 0;
        while (k + 1 < b.nclouds && b.h_clouds[(size_t)k + 1].node0 <= g) ++k;
        return fail(PXB_ERR_DEGENERATE, "pxb_batch_gbuild: degenerate moment matrix in cloud " + std::to_string(k) +
                                            " at node " + std::to_string(g - b.h_clouds[(size_t)k].node0 + 1) + " (" +
                                            std::to_string(out[0]) + " node(s) in the batch)");
    }
    b.built = true;
    return PXB_OK;
}

extern "C" int pxb_batch_apply_d(pxb_ctx *c, const double *u_d, double *out_d) {
    PXB_TRY(need_batch(c, "pxb_batch_apply", true));
    if (!u_d || !out_d) return fail(PXB_ERR_INVALID, "pxb_batch_apply: NULL buffer");
    return apply_enqueue(c, u_d, out_d);
}

extern "C" int pxb_batch_apply(pxb_ctx *c, const double *u, double *out) {
    PXB_TRY(need_batch(c, "pxb_batch_apply", true));
    if (!u || !out) return fail(PXB_ERR_INVALID, "pxb_batch_apply: NULL buffer");
    const BatchState &b = c->batch;
    DevBuf du, dout;
    PXB_TRY(dev_alloc(c, du, sizeof(double) * (size_t)b.n));
    PXB_TRY(dev_alloc(c, dout, sizeof(double) * (size_t)b.out_len));
    PXB_TRY(h2d(c, du.p, u, sizeof(double) * (size_t)b.n));
    PXB_TRY(apply_enqueue(c, du.as<double>(), dout.as<double>()));
    PXB_TRY(d2h(c, out, dout.p, sizeof(double) * (size_t)b.out_len));
    return sync(c);
}

extern "C" int pxb_batch_get_ops(pxb_ctx *c, int cloud, double *ops) {
    PXB_TRY(need_batch(c, "pxb_batch_get_ops", true));
    const BatchState &b = c->batch;
    if (cloud < 0 || cloud >= b.nclouds || !ops) return fail(PXB_ERR_INVALID, "pxb_batch_get_ops: bad arguments");
    const BatchCloud &cd = b.h_clouds[(size_t)cloud];
    const size_t cnt = (size_t)cd.nb * nop_of_dim(cd.dim);
    if (b.precision == PXB_MIXED) {
        std::vector<float> tmp(std::max<size_t>(1, cnt));
        PXB_TRY(d2h(c, tmp.data(), b.ops.as<float>() + cd.ops_off, sizeof(float) * cnt));
        PXB_TRY(sync(c));
        for (size_t k = 0; k < cnt; ++k) ops[k] = tmp[k];
        return PXB_OK;
    }
    PXB_TRY(d2h(c, ops, b.ops.as<double>() + cd.ops_off, sizeof(double) * cnt));
    return sync(c);
}

extern "C" int pxb_batch_set_variant(pxb_ctx *c, int which, int variant) {
    PXB_TRY(need_batch(c, "pxb_batch_set_variant", false));
    if ((which != 0 && which != 1) || variant < 0 || variant >= kBatchVariants)
        return fail(PXB_ERR_INVALID, "pxb_batch_set_variant: which is 0 (g-build) or 1 (apply), variant 0.." +
                                         std::to_string(kBatchVariants - 1));
    (which == 0 ? c->batch.gvariant : c->batch.avariant) = variant;
    return PXB_OK;
}

extern "C" int pxb_batch_get_variant(pxb_ctx *c, int which, int *variant) {
    PXB_TRY(need_batch(c, "pxb_batch_get_variant", false));
    if (!variant) return fail(PXB_ERR_INVALID, "pxb_batch_get_variant: NULL");
    *variant = which == 0 ? c->batch.gvariant : c->batch.avariant;
    return PXB_OK;
}

// Times `reps` launches of the current schedule of the g-build (what 0) or the apply (what 1, on the field
// u_d into out_d, device pointers), the L2 flushed before each; ms[r] per launch group.
int pxb::batch_time(pxb_ctx *c, int what, int reps, size_t flush_bytes, const double *u_d, double *out_d, float *ms) {
    PXB_TRY(need_batch(c, "pxb_batch_time", what == 1));
    if (reps <= 0 || !ms || (what == 1 && (!u_d || !out_d)) || (what != 0 && what != 1))
        return fail(PXB_ERR_INVALID, "pxb_batch_time: bad arguments");
    if (what == 0 && !c->batch.ops.p) return fail(PXB_ERR_STATE, "pxb_batch_time: call pxb_batch_gbuild first");
    std::vector<cudaEvent_t> ev(2 * (size_t)reps, nullptr);
    int st = PXB_OK;
    for (auto &e : ev)
        if (cudaEventCreate(&e) != cudaSuccess) st = fail(PXB_ERR_CUDA, "pxb_batch_time: event create");
    for (int r = 0; r < reps && st == PXB_OK; ++r) {
        st = l2_flush(c, flush_bytes);
        if (st == PXB_OK && cudaEventRecord(ev[2 * (size_t)r], c->stream) != cudaSuccess) st = fail(PXB_ERR_CUDA, "event record");
        if (st == PXB_OK) st = what == 0 ? gbuild_enqueue(c) : apply_enqueue(c, u_d, out_d);
        if (st == PXB_OK && cudaEventRecord(ev[2 * (size_t)r + 1], c->stream) != cudaSuccess) st = fail(PXB_ERR_CUDA, "event record");
    }
    if (st == PXB_OK) st = sync(c);
    for (int r = 0; r < reps && st == PXB_OK; ++r)
        if (cudaEventElapsedTime(&ms[r], ev[2 * (size_t)r], ev[2 * (size_t)r + 1]) != cudaSuccess)
            st = fail(PXB_ERR_CUDA, "event elapsed");
    for (auto e : ev)
        if (e) cudaEventDestroy(e);
    return st;
}

// Times every schedule of the g-build (what 0) or the apply (what 1) for `reps` launches, keeps the fastest;
// ms_per_variant (kBatchVariants entries, may be NULL) receives the mean times.
extern "C" int pxb_batch_autotune(pxb_ctx *c, int what, int reps, size_t flush_bytes, const double *u_d, double *out_d,
                                  int *best, float *ms_per_variant) {
    PXB_TRY(need_batch(c, "pxb_batch_autotune", what == 1));
    if (reps <= 0) return fail(PXB_ERR_INVALID, "pxb_batch_autotune: reps must be > 0");
    int &slot = what == 0 ? c->batch.gvariant : c->batch.avariant;
    std::vector<float> ms((size_t)reps);
    float best_ms = 1e30f;
    int best_v = slot;
    for (int v = 0; v < kBatchVariants; ++v) {
        slot = v;
        // one untimed launch first: a kernel's first launch in a process also loads its module
        PXB_TRY(batch_time(c, what, 1, 0, u_d, out_d, ms.data()));
        PXB_TRY(batch_time(c, what, reps, flush_bytes, u_d, out_d, ms.data()));
        float mean = 0.f;
        for (float x : ms) mean += x;
        mean /= (float)reps;
        if (ms_per_variant) ms_per_variant[v] = mean;
        if (mean < best_ms) { best_ms = mean; best_v = v; }
    }
    slot = best_v;
    if (best) *best = best_v;
    return PXB_OK;
}

extern "C" int pxb_batch_variant_count(void) { return kBatchVariants; }
