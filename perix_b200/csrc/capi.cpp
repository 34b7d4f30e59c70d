// The extern "C" layer of perix_b200 (C++20 host code).  Every entry point validates its arguments, drives
// the kernels on the context stream and reports failures as pxb_status codes; there is no CPU fallback.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <limits>
#include <string>
#include <vector>

#include "k_kernels.h"
#include "pxb_context.h"
#include "tune_internal.h"
#include "fam_builder.h"

namespace pxb {

static thread_local std::string t_error;

void set_error(const std::string &msg) { t_error = msg; }

int fail(int status, const std::string &msg) {
    t_error = msg;
    return status;
}

int cuda_fail(cudaError_t e, const char *what) {
    t_error = std::string("CUDA error in ") + what + ": " + cudaGetErrorString(e);
    return (e == cudaErrorMemoryAllocation) ? PXB_ERR_OOM : PXB_ERR_CUDA;
}

void DevBuf::release() {
    if (p) cudaFree(p);
    p = nullptr;
    bytes = 0;
}

PinnedBuf::~PinnedBuf() {
    if (p) cudaFreeHost(p);
}

PinnedBuf &PinnedBuf::operator=(PinnedBuf &&o) noexcept {
    if (this != &o) {
        if (p) cudaFreeHost(p);
        p = o.p;
        bytes = o.bytes;
        o.p = nullptr;
        o.bytes = 0;
    }
    return *this;
}

int ensure_pinned(PinnedBuf &b, size_t bytes) {
    if (b.bytes >= bytes) return PXB_OK;
    if (b.p) cudaFreeHost(b.p);
    b.p = nullptr;
    b.bytes = 0;
    PXB_CUDA_TRY(cudaMallocHost(&b.p, bytes));
    b.bytes = bytes;
    return PXB_OK;
}

// a failed cudaMalloc is PXB_ERR_OOM (its sticky-free error is cleared so the context stays usable)
static int malloc_dev(void **p, size_t bytes) {
    const cudaError_t e = cudaMalloc(p, bytes);
    if (e == cudaSuccess) return PXB_OK;
    *p = nullptr;
    cudaGetLastError();
    if (e == cudaErrorMemoryAllocation)
        return fail(PXB_ERR_OOM, "device allocation of " + std::to_string(bytes) + " bytes failed (out of memory)");
    return cuda_fail(e, "cudaMalloc");
}

int dev_alloc(pxb_ctx *c, DevBuf &b, size_t bytes) {
    if (b.p && b.bytes == bytes) return PXB_OK;
    if (c && c->mem_limit && bytes > b.bytes && ctx_bytes(c) - b.bytes + bytes > c->mem_limit)
        return fail(PXB_ERR_OOM, "device allocation of " + std::to_string(bytes) + " bytes would exceed the context's " +
                                     std::to_string(c->mem_limit) + "-byte limit (pxb_ctx_set_memory_limit)");
    b.release();
    if (bytes == 0) return PXB_OK;
    PXB_TRY(malloc_dev(&b.p, bytes));
    b.bytes = bytes;
    return PXB_OK;
}

int h2d(pxb_ctx *c, void *dst, const void *src, size_t bytes) {
    if (bytes == 0) return PXB_OK;
    PXB_CUDA_TRY(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, c->stream));
    return PXB_OK;
}

int d2h(pxb_ctx *c, void *dst, const void *src, size_t bytes) {
    if (bytes == 0) return PXB_OK;
    PXB_CUDA_TRY(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, c->stream));
    return PXB_OK;
}

int dev_upload(pxb_ctx *c, DevBuf &b, const void *host, size_t bytes) {
    PXB_TRY(dev_alloc(c, b, bytes));
    return h2d(c, b.p, host, bytes);
}

int sync(pxb_ctx *c) {
    PXB_CUDA_TRY(cudaStreamSynchronize(c->stream));
    return PXB_OK;
}

int check_launch(pxb_ctx *c, const char *what) {
    c->launches++;
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(e, what);
    return PXB_OK;
}

// A staged kernel's consumer wait ran out in `werr` blocks: clear the context's error word (so the next call starts
// clean) and report the failure.
int wait_failure(pxb_ctx *c, unsigned int werr, const char *what) {
    cudaMemsetAsync(c->epf.counters.as<unsigned long long>() + 2, 0, sizeof(unsigned int), c->stream);
    cudaStreamSynchronize(c->stream);
    return fail(PXB_ERR_CUDA, std::string(what) + ": a staged-copy wait ran out (" + std::to_string(werr) + " blocks)");
}

static size_t bufsz(const DevBuf &b) { return b.bytes; }

size_t ctx_bytes(const pxb_ctx *c) {
    size_t s = 0;
    const Geometry &g = c->g;
    s += bufsz(g.off) + bufsz(g.nbr) + bufsz(g.pos) + bufsz(g.vol) + bufsz(g.mirror) + bufsz(g.layer) + bufsz(g.rev);
    s += bufsz(c->ops.ops) + bufsz(c->ops.degenerate) + bufsz(c->ops.defect) + bufsz(c->ops.yeff);
    const EpfState &e = c->epf;
    s += bufsz(e.G) + bufsz(e.P) + bufsz(e.xib) + bufsz(e.health) + bufsz(e.u[0]) + bufsz(e.u[1]) + bufsz(e.accel) + bufsz(e.counters) +
         bufsz(e.umax) + bufsz(e.tsched) + bufsz(e.sc_bond);
    s += bufsz(e.adj_ckpt) + bufsz(e.adj_seg) + bufsz(e.adj_p[0]) + bufsz(e.adj_p[1]) + bufsz(e.adj_A) + bufsz(e.adj_R) +
         bufsz(e.adj_W) + bufsz(e.adj_t) + bufsz(e.adj_dC) + bufsz(e.adj_umax) + bufsz(e.adj_GR) + bufsz(e.adj_HR) + bufsz(e.adj_u0) + bufsz(e.adj_SG) + bufsz(e.adj_UW);
    s += bufsz(e.bc.own) + bufsz(e.bc.src_off) + bufsz(e.bc.tgt) + bufsz(e.bc.comp) + bufsz(e.bc.form) +
         bufsz(e.bc.vals);
    const BatchState &bt = c->batch;
    s += bufsz(bt.clouds) + bufsz(bt.tasks) + bufsz(bt.off) + bufsz(bt.nbr) + bufsz(bt.pos) + bufsz(bt.vol) +
         bufsz(bt.ops) + bufsz(bt.degenerate) + bufsz(bt.counters) + bufsz(bt.defect);
    const CsrState &k = c->csr;
    s += bufsz(k.rowptr) + bufsz(k.cols) + bufsz(k.slot) + bufsz(k.diag) + bufsz(k.kvals) + bufsz(k.rhs) +
         bufsz(k.u) + bufsz(k.uold) + bufsz(k.fnode) + bufsz(k.mnode);
    s += bufsz(c->ch.rev) + bufsz(c->ch.lap) + bufsz(c->ch.ghost) + bufsz(c->ch.lrv) + bufsz(c->ch.bfl) +
         bufsz(c->scratch);
    return s;
}

// scratch device memory for staging (grown on demand, never shrunk)
static int scratch(pxb_ctx *c, size_t bytes, void **p) {
    if (c->scratch.bytes < bytes) PXB_TRY(dev_alloc(c, c->scratch, bytes));
    *p = c->scratch.p;
    return PXB_OK;
}

static int grid_nodes(int n, int threads) {
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int wpb = threads / 32;
    const long long need = ((long long)n + wpb - 1) / wpb;
    const long long cap = (long long)sms * 16;
    const long long g = std::min(need, cap);
    return (int)std::max(1LL, g);
}

static void destroy_graphs(EpfState &e) {
    for (auto &kv : e.graphs) cudaGraphExecDestroy(kv.second);
    e.graphs.clear();
    if (e.rate_graph) cudaGraphExecDestroy(e.rate_graph);
    e.rate_graph = nullptr;
    e.rate_u = e.rate_last_u = nullptr;
    e.rate_a = e.rate_last_a = nullptr;
    e.rate_last_variant = -1;
    if (e.rate_done) cudaEventDestroy(e.rate_done);
    e.rate_done = nullptr;
    for (cudaEvent_t ev : e.rate_ev) cudaEventDestroy(ev);
    e.rate_ev.clear();
    if (e.rate_up) cudaStreamDestroy(e.rate_up);
    if (e.rate_down) cudaStreamDestroy(e.rate_down);
    e.rate_up = e.rate_down = nullptr;
}

// Waits for the work queued so far by polling an event from the calling thread: the per-step call's wait is short
// (~0.1 ms) and a blocking or yielding synchronisation adds a wake-up latency of the same order on a loaded host.
// After kSpinPolls polls it falls back to a blocking synchronisation.
static int sync_polled(pxb_ctx *c, cudaEvent_t &ev) {
    constexpr long kSpinPolls = 1L << 22;
    if (!ev) PXB_CUDA_TRY(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
    PXB_CUDA_TRY(cudaEventRecord(ev, c->stream));
    for (long k = 0; k < kSpinPolls; ++k) {
        const cudaError_t q = cudaEventQuery(ev);
        if (q == cudaSuccess) return PXB_OK;
        if (q != cudaErrorNotReady) return cuda_fail(q, "event poll");
    }
    return sync(c);
}

}  // namespace pxb

using namespace pxb;

// =============================================================================================== library / ctx
extern "C" int pxb_version(void) { return PXB_VERSION; }

extern "C" const char *pxb_last_error(void) { return t_error.c_str(); }

extern "C" int pxb_ctx_create(int device, pxb_ctx **out) {
    if (!out) return fail(PXB_ERR_INVALID, "pxb_ctx_create: out is NULL");
    *out = nullptr;
    int ndev = 0;
    cudaError_t e = cudaGetDeviceCount(&ndev);
    if (e != cudaSuccess || ndev <= 0)
        return fail(PXB_ERR_CUDA, std::string("pxb_ctx_create: no CUDA device (") + cudaGetErrorString(e) + ")");
    if (device < 0 || device >= ndev) return fail(PXB_ERR_INVALID, "pxb_ctx_create: device index out of range");
    PXB_CUDA_TRY(cudaSetDevice(device));
    auto *c = new pxb_ctx();
    c->device = device;
    e = cudaStreamCreateWithFlags(&c->own, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
        delete c;
        return cuda_fail(e, "cudaStreamCreateWithFlags");
    }
    c->stream = c->own;
    *out = c;
    return PXB_OK;
}

namespace pxb {
void drop_snapshot(pxb_ctx *c);
}

extern "C" int pxb_ctx_destroy(pxb_ctx *c) {
    if (!c) return PXB_OK;
    cudaSetDevice(c->device);
    cudaStreamSynchronize(c->stream);
    drop_snapshot(c);
    destroy_graphs(c->epf);
    if (c->own) cudaStreamDestroy(c->own);
    delete c;
    return PXB_OK;
}

extern "C" int pxb_ctx_set_stream(pxb_ctx *c, void *stream) {
    if (!c) return fail(PXB_ERR_INVALID, "pxb_ctx_set_stream: NULL context");
    cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : c->own;
    if (s != c->stream) destroy_graphs(c->epf);
    c->stream = s;
    return PXB_OK;
}

extern "C" int pxb_ctx_synchronize(pxb_ctx *c) {
    if (!c) return fail(PXB_ERR_INVALID, "pxb_ctx_synchronize: NULL context");
    return sync(c);
}

extern "C" int pxb_ctx_device_bytes(pxb_ctx *c, size_t *bytes) {
    if (!c || !bytes) return fail(PXB_ERR_INVALID, "pxb_ctx_device_bytes: NULL argument");
    *bytes = ctx_bytes(c);
    return PXB_OK;
}

extern "C" int pxb_ctx_launch_count(pxb_ctx *c, long long *count) {
    if (!c || !count) return fail(PXB_ERR_INVALID, "pxb_ctx_launch_count: NULL argument");
    *count = c->launches;
    return PXB_OK;
}

// ==================================================================================================== geometry
// drop every state that depends on the geometry, then store the CSR offsets (host copy + device) and allocate
// the zeroed neighbour array (ldb = nb rounded up to 16, plus 16)
static int geometry_reset(pxb_ctx *c, int n, int dim, const int *neigh_off, int maxf, double delta, double dx_char,
                          const int *mirror) {
    PXB_CUDA_TRY(cudaSetDevice(c->device));
    PXB_CUDA_TRY(cudaStreamSynchronize(c->stream));
    destroy_graphs(c->epf);
    c->ops = OpsCache{};
    c->epf = EpfState{};
    c->csr = CsrState{};
    c->ch = ChState{};
    Geometry &g = c->g;
    g = Geometry{};
    const long long nb = neigh_off[n];
    g.n = n;
    g.dim = dim;
    g.nb = nb;
    g.delta = delta;
    g.dx_char = dx_char;
    g.max_family = maxf;
    g.h_off.assign(neigh_off, neigh_off + n + 1);
    if (mirror) g.h_mirror.assign(mirror, mirror + n);
    g.ldb = ((nb + 16 + 15) / 16) * 16;
    PXB_TRY(dev_alloc(c, g.off, sizeof(int) * (size_t)(n + 1 + 16)));
    PXB_CUDA_TRY(cudaMemsetAsync(g.off.p, 0, g.off.bytes, c->stream));
    PXB_TRY(h2d(c, g.off.p, neigh_off, sizeof(int) * (size_t)(n + 1)));
    PXB_TRY(dev_alloc(c, g.nbr, sizeof(int) * (size_t)g.ldb));
    PXB_CUDA_TRY(cudaMemsetAsync(g.nbr.p, 0, g.nbr.bytes, c->stream));
    return PXB_OK;
}

// positions (packed double2 / double4), volumes, mirror and layer maps; marks the geometry ready
static int geometry_finish(pxb_ctx *c, const double *coords3_d, const double *vols, const int *mirror,
                           const int *layer_index) {
    Geometry &g = c->g;
    PXB_TRY(dev_alloc(c, g.pos, (g.dim == 2 ? 16 : 32) * (size_t)g.n));
    launch_pos_pack(g.n, g.dim, coords3_d, g.pos.p, c->stream);
    PXB_TRY(check_launch(c, "pos_pack"));
    PXB_TRY(dev_upload(c, g.vol, vols, sizeof(double) * (size_t)g.n));
    if (mirror) PXB_TRY(dev_upload(c, g.mirror, mirror, sizeof(int) * (size_t)g.n));
    if (layer_index) PXB_TRY(dev_upload(c, g.layer, layer_index, sizeof(int) * (size_t)g.n));
    PXB_TRY(sync(c));
    g.ready = true;
    return PXB_OK;
}

extern "C" int pxb_set_geometry(pxb_ctx *c, int n, int dim, const double *coords3, const double *vols,
                                const int *neigh_off, const int *neigh_id, double delta, double dx_char,
                                const int *mirror, const int *layer_index) {
    if (!c) return fail(PXB_ERR_INVALID, "pxb_set_geometry: NULL context");
    if (n <= 0 || (dim != 2 && dim != 3) || !coords3 || !vols || !neigh_off || !neigh_id || !(delta > 0.0))
        return fail(PXB_ERR_INVALID, "pxb_set_geometry: bad arguments (need n>0, dim 2|3, delta>0, non-NULL arrays)");
    if (neigh_off[0] != 0) return fail(PXB_ERR_INVALID, "pxb_set_geometry: neigh_off[0] must be 0");
    int maxf = 0;
    for (int i = 0; i < n; ++i) {
        const int f = neigh_off[i + 1] - neigh_off[i];
        if (f < 0) return fail(PXB_ERR_INVALID, "pxb_set_geometry: neigh_off is not non-decreasing");
        maxf = std::max(maxf, f);
    }
    const long long nb = neigh_off[n];
    for (long long t = 0; t < nb; ++t)
        if (neigh_id[t] < 1 || neigh_id[t] > n)
            return fail(PXB_ERR_INVALID, "pxb_set_geometry: neighbour id out of range (ids are 1-based)");
    PXB_TRY(geometry_reset(c, n, dim, neigh_off, maxf, delta, dx_char, mirror));
    Geometry &g = c->g;
    void *tmp = nullptr;
    PXB_TRY(scratch(c, std::max(sizeof(int) * (size_t)std::max(1LL, nb), sizeof(double) * 3 * (size_t)n), &tmp));
    PXB_TRY(h2d(c, tmp, neigh_id, sizeof(int) * (size_t)nb));
    if (nb > 0) {
        launch_ids_to0(nb, static_cast<const int *>(tmp), g.nbr.as<int>(), c->stream);
        PXB_TRY(check_launch(c, "ids_to0"));
    }
    PXB_CUDA_TRY(cudaStreamSynchronize(c->stream));
    PXB_TRY(h2d(c, tmp, coords3, sizeof(double) * 3 * (size_t)n));
    return geometry_finish(c, static_cast<const double *>(tmp), vols, mirror, layer_index);
}

// Families built on the device (k_families.cu, fam_builder.h), then the geometry as pxb_set_geometry sets it.
extern "C" int pxb_set_geometry_points(pxb_ctx *c, int n, int dim, const double *coords3, const double *vols,
                                       double radius, double delta, double dx_char, const int *mirror,
                                       const int *layer_index, long long *nbtot) {
    if (!c) return fail(PXB_ERR_INVALID, "pxb_set_geometry_points: NULL context");
    if (n <= 0 || (dim != 2 && dim != 3) || !coords3 || !vols || !(radius > 0.0) || !(delta > 0.0))
        return fail(PXB_ERR_INVALID, "pxb_set_geometry_points: bad arguments (need n>0, dim 2|3, radius>0, delta>0)");
    PXB_CUDA_TRY(cudaSetDevice(c->device));
    PXB_CUDA_TRY(cudaStreamSynchronize(c->stream));
    FamBuilder fb;
    std::vector<int> hoff;
    int maxf = 0;
    long long tot = 0;
    PXB_TRY(fb.count(c, n, dim == 3, coords3, radius, hoff, maxf, tot));
    PXB_TRY(geometry_reset(c, n, dim, hoff.data(), maxf, delta, dx_char, mirror));
    PXB_TRY(fb.fill(c, c->g.off.as<int>(), c->g.nbr.as<int>(), 0));
    if (nbtot) *nbtot = tot;
    return geometry_finish(c, fb.coords_d(), vols, mirror, layer_index);
}

static int need_geometry(pxb_ctx *c, const char *who);

// Per-node horizon and spacing for the g-build (the reference's VariableHorizon; NULL delta clears them).  Drops the
// operator caches built with the previous horizons.
extern "C" int pxb_set_node_horizons(pxb_ctx *c, const double *node_delta, const double *node_spacing) {
    PXB_TRY(need_geometry(c, "pxb_set_node_horizons"));
    Geometry &g = c->g;
    c->ops = OpsCache{};
    destroy_graphs(c->epf);
    c->epf = EpfState{};
    g.node_delta = DevBuf{};
    g.node_dxc = DevBuf{};
    g.h_node_delta.clear();
    if (!node_delta) return PXB_OK;
    for (int i = 0; i < g.n; ++i)
        if (!(node_delta[i] > 0.0)) return fail(PXB_ERR_INVALID, "pxb_set_node_horizons: delta must be > 0");
    std::vector<double> sp((size_t)g.n, 0.0);
    if (node_spacing) sp.assign(node_spacing, node_spacing + g.n);
    PXB_TRY(dev_upload(c, g.node_delta, node_delta, sizeof(double) * (size_t)g.n));
    PXB_TRY(dev_upload(c, g.node_dxc, sp.data(), sizeof(double) * (size_t)g.n));
    g.h_node_delta.assign(node_delta, node_delta + g.n);
    return sync(c);
}

// The families of the current geometry, 1-based ids (neigh_off: n+1 entries, neigh_id: neigh_off[n]).
extern "C" int pxb_get_families(pxb_ctx *c, int *neigh_off, int *neigh_id) {
    if (!c || !c->g.ready) return fail(PXB_ERR_STATE, "pxb_get_families: geometry not set");
    const Geometry &g = c->g;
    if (neigh_off) std::copy(g.h_off.begin(), g.h_off.end(), neigh_off);
    if (neigh_id) {
        PXB_TRY(d2h(c, neigh_id, g.nbr.p, sizeof(int) * (size_t)g.nb));
        PXB_TRY(sync(c));
        for (long long t = 0; t < g.nb; ++t) ++neigh_id[t];
    }
    return PXB_OK;
}

static int need_geometry(pxb_ctx *c, const char *who) {
    if (!c) return fail(PXB_ERR_INVALID, std::string(who) + ": NULL context");
    if (!c->g.ready) return fail(PXB_ERR_STATE, std::string(who) + ": geometry not set (call pxb_set_geometry)");
    PXB_CUDA_TRY(cudaSetDevice(c->device));
    return PXB_OK;
}

static int ensure_rev(pxb_ctx *c) {
    Geometry &g = c->g;
    if (g.rev.p) return PXB_OK;
    PXB_TRY(dev_alloc(c, g.rev, sizeof(int) * (size_t)std::max(1LL, g.nb)));
    launch_build_rev(g.n, g.off.as<int>(), g.nbr.as<int>(), g.rev.as<int>(), grid_nodes(g.n, kApplyThreads), c->stream);
    return check_launch(c, "build_rev");
}

// ===================================================================================================== g-build
static GBuildArgs gbuild_args(pxb_ctx *c, void *ops_out, void *G_out, uint8_t *deg_out, unsigned int *nd,
                              int *first, float *defect = nullptr) {
    Geometry &g = c->g;
    GBuildArgs a;
    a.n = g.n;
    a.off = g.off.as<int>();
    a.nbr = g.nbr.as<int>();
    a.pos = g.pos.p;
    a.vol = g.vol.as<double>();
    a.layer = g.layer.p ? g.layer.as<int>() : nullptr;
    a.delta = g.delta;
    a.dx_char = g.dx_char;
    a.nb = g.ldb;  // SoA stride of the Navier operator streams
    a.ops = ops_out;
    a.G = G_out;
    a.degenerate = deg_out;
    a.n_degenerate = nd;
    a.first_degenerate = first;
    a.defect = defect;
    if (g.node_delta.p) {
        a.node_delta = g.node_delta.as<double>();
        a.node_dxc = g.node_dxc.as<double>();
    }
    return a;
}

// the g-build schedule for this problem: one warp per node (k_gbuild_warp.cu) for 3D and for 2D above order 2,
// lane groups (k_gbuild.cu) for 2D orders 1-2, unless pxb_gbuild_set_schedule chose one
static bool gbuild_use_warp(const pxb_ctx *c, int order) {
    if (!gbuild_warp_supported(c->g.dim, order)) return false;
    if (c->g.node_delta.p) return true;  // per-node horizons: the warp-per-node kernel reads them
    if (!gbuild_supported(c->g.dim, order)) return true;
    if (c->gbuild_schedule >= 0) return c->gbuild_schedule >= 1;
    return c->g.dim == 3 || order > 2;
}

static cudaError_t gbuild_launch(pxb_ctx *c, const GBuildArgs &a, int order, bool mixed) {
    if (gbuild_use_warp(c, order)) {
        // the tensor-core products up to nine monomials unless schedule 1 (scalar warp per node) was chosen
        const bool small = c->g.dim == 3 ? order <= 2 : order <= 3;
        const bool tc = c->gbuild_schedule == 2 || (c->gbuild_schedule < 0 && small);
        return launch_gbuild_warp(a, c->g.dim, order, mixed, tc, c->stream);
    }
    return launch_gbuild(a, c->g.dim, order, mixed, grid_nodes(c->g.n, kGbuildThreads), c->stream);
}

static int run_gbuild(pxb_ctx *c, int order, bool mixed, void *ops_out, void *G_out, uint8_t *deg_out,
                      int *n_degenerate, int *first_degenerate, float *defect = nullptr) {
    Geometry &g = c->g;
    if (!gbuild_supported(g.dim, order) && !gbuild_warp_supported(g.dim, order))
        return fail(PXB_ERR_UNSUPPORTED, "pxb_gbuild: order " + std::to_string(order) + " not built for dim " +
                                             std::to_string(g.dim) + " (2D: 1..4, 3D: 1..3)");
    void *tmp = nullptr;
    PXB_TRY(scratch(c, 16, &tmp));
    unsigned int *nd = static_cast<unsigned int *>(tmp);
    int *first = reinterpret_cast<int *>(static_cast<char *>(tmp) + 8);
    PXB_CUDA_TRY(cudaMemsetAsync(nd, 0, 4, c->stream));
    const int big = std::numeric_limits<int>::max();
    PXB_TRY(h2d(c, first, &big, sizeof(int)));
    const GBuildArgs a = gbuild_args(c, ops_out, G_out, deg_out, nd, first, defect);
    cudaError_t e = gbuild_launch(c, a, order, mixed);
    c->launches++;
    if (e != cudaSuccess) return cuda_fail(e, "gbuild launch");
    unsigned int hnd = 0;
    int hfirst = big;
    PXB_TRY(d2h(c, &hnd, nd, 4));
    PXB_TRY(d2h(c, &hfirst, first, 4));
    PXB_TRY(sync(c));
    if (n_degenerate) *n_degenerate = (int)hnd;
    if (first_degenerate) *first_degenerate = hnd ? hfirst + 1 : 0;
    if (hnd)
        return fail(PXB_ERR_DEGENERATE, "degenerate moment matrix at node " + std::to_string(hfirst + 1) + " (" +
                                            std::to_string(hnd) + " non-ghost node(s)): the family cannot support "
                                            "this PDDO order");
    return PXB_OK;
}

extern "C" int pxb_gbuild(pxb_ctx *c, int order, int precision, int *n_degenerate, int *first_degenerate) {
    PXB_TRY(need_geometry(c, "pxb_gbuild"));
    if (precision != PXB_FP64 && precision != PXB_MIXED) return fail(PXB_ERR_INVALID, "pxb_gbuild: bad precision");
    OpsCache &o = c->ops;
    o.ready = false;
    int nop = 0;
    for (int k = 1; k <= order; ++k) nop += (c->g.dim == 3) ? (k + 1) * (k + 2) / 2 : (k + 1);
    const size_t es = precision == PXB_MIXED ? 4 : 8;
    PXB_TRY(dev_alloc(c, o.ops, es * (size_t)nop * (size_t)std::max(1LL, c->g.nb)));
    PXB_TRY(dev_alloc(c, o.degenerate, (size_t)c->g.n));
    o.order = order;
    o.nop = nop;
    o.precision = precision;
    o.pqr.clear();
    for (int k = 1; k <= order; ++k)
        for (int p = k; p >= 0; --p) {
            if (c->g.dim == 3)
                for (int q = k - p; q >= 0; --q) o.pqr.insert(o.pqr.end(), {p, q, k - p - q});
            else
                o.pqr.insert(o.pqr.end(), {p, k - p, 0});
        }
    float *defect = nullptr;
    o.defect = DevBuf{};
    if (precision == PXB_MIXED && order == 2) {
        PXB_TRY(dev_alloc(c, o.defect, sizeof(float) * (size_t)c->g.n * (size_t)((nop - c->g.dim) * c->g.dim)));
        PXB_CUDA_TRY(cudaMemsetAsync(o.defect.p, 0, o.defect.bytes, c->stream));
        defect = o.defect.as<float>();
    }
    const int st = run_gbuild(c, order, precision == PXB_MIXED, o.ops.p, nullptr, o.degenerate.as<uint8_t>(),
                              n_degenerate, first_degenerate, defect);
    if (st == PXB_OK || st == PXB_ERR_DEGENERATE) o.ready = true;  // degenerate rows carry zero operators
    return st;
}

namespace pxb {
int gbuild_launch_only(pxb_ctx *c, int order, int precision) {
    if (!c->ops.ready || c->ops.order != order || c->ops.precision != precision)
        return fail(PXB_ERR_STATE, "g-build timing needs a prior pxb_gbuild with the same order and precision");
    void *tmp = nullptr;
    PXB_TRY(scratch(c, 16, &tmp));
    const GBuildArgs a = gbuild_args(c, c->ops.ops.p, nullptr, c->ops.degenerate.as<uint8_t>(),
                                     static_cast<unsigned int *>(tmp),
                                     reinterpret_cast<int *>(static_cast<char *>(tmp) + 8),
                                     c->ops.defect.p ? c->ops.defect.as<float>() : nullptr);
    cudaError_t e = gbuild_launch(c, a, order, precision == PXB_MIXED);
    c->launches++;
    if (e != cudaSuccess) return cuda_fail(e, "gbuild launch");
    return PXB_OK;
}
}  // namespace pxb

extern "C" int pxb_gbuild_set_schedule(pxb_ctx *c, int schedule) {
    if (!c) return fail(PXB_ERR_INVALID, "pxb_gbuild_set_schedule: NULL context");
    if (schedule < -1 || schedule > 2) return fail(PXB_ERR_INVALID, "pxb_gbuild_set_schedule: -1, 0, 1 or 2");
    c->gbuild_schedule = schedule;
    return PXB_OK;
}

// the recorded sweep's adjoint schedule in effect (-1: the staged reverse-only kernel, schedule 4)
static int adj_sched(const pxb_ctx *c) { return c->adj_schedule < 0 ? 4 : c->adj_schedule; }

extern "C" int pxb_epf_set_rate_chunks(pxb_ctx *c, int chunks) {
    if (!c) return fail(PXB_ERR_INVALID, "pxb_epf_set_rate_chunks: NULL context");
    if (chunks < -1 || chunks == 0 || chunks > 8) return fail(PXB_ERR_INVALID, "pxb_epf_set_rate_chunks: -1 or 1..8");
    c->rate_chunks = chunks;
    c->epf.rate_plan_done = false;
    destroy_graphs(c->epf);
    return PXB_OK;
}

extern "C" int pxb_epf_set_adjoint_schedule(pxb_ctx *c, int schedule) {
    if (!c) return fail(PXB_ERR_INVALID, "pxb_epf_set_adjoint_schedule: NULL context");
    if (schedule < -1 || schedule > 4) return fail(PXB_ERR_INVALID, "pxb_epf_set_adjoint_schedule: -1 .. 4");
    c->adj_schedule = schedule;
    return PXB_OK;
}

extern "C" int pxb_gbuild_info(pxb_ctx *c, int *nop, int *pqr) {
    if (!c) return fail(PXB_ERR_INVALID, "pxb_gbuild_info: NULL context");
    if (!c->ops.ready) return fail(PXB_ERR_STATE, "pxb_gbuild_info: no operator cache (call pxb_gbuild)");
    if (nop) *nop = c->ops.nop;
    if (pqr) std::copy(c->ops.pqr.begin(), c->ops.pqr.end(), pqr);
    return PXB_OK;
}

extern "C" int pxb_get_ops(pxb_ctx *c, double *ops) {
    PXB_TRY(need_geometry(c, "pxb_get_ops"));
    if (!c->ops.ready || !ops) return fail(PXB_ERR_STATE, "pxb_get_ops: no operator cache");
    const size_t cnt = (size_t)c->ops.nop * (size_t)c->g.nb;
    if (c->ops.precision == PXB_FP64) {
        PXB_TRY(d2h(c, ops, c->ops.ops.p, cnt * 8));
        return sync(c);
    }
    std::vector<float> tmp(cnt);
    PXB_TRY(d2h(c, tmp.data(), c->ops.ops.p, cnt * 4));
    PXB_TRY(sync(c));
    for (size_t k = 0; k < cnt; ++k) ops[k] = tmp[k];
    return PXB_OK;
}

// ======================================================================================================= apply
static int apply_args(pxb_ctx *c, int nk, const int *slots, ApplyArgs &a, const char *who) {
    PXB_TRY(need_geometry(c, who));
    if (!c->ops.ready) return fail(PXB_ERR_STATE, std::string(who) + ": no operator cache (call pxb_gbuild)");
    if (nk < 1 || nk > 20 || !slots) return fail(PXB_ERR_INVALID, std::string(who) + ": nk must be 1..20");
    for (int s = 0; s < nk; ++s)
        if (slots[s] < 0 || slots[s] >= c->ops.nop) return fail(PXB_ERR_INVALID, std::string(who) + ": slot out of range");
    a.n = c->g.n;
    a.nop = c->ops.nop;
    a.nk = nk;
    for (int s = 0; s < nk; ++s) a.slots[s] = slots[s];
    a.off = c->g.off.as<int>();
    a.nbr = c->g.nbr.as<int>();
    a.ops = c->ops.ops.p;
    a.dim = c->g.dim;
    a.defect = c->ops.defect.p ? c->ops.defect.as<float>() : nullptr;
    return PXB_OK;
}

extern "C" int pxb_apply_d(pxb_ctx *c, const double *u_d, int nk, const int *slots, double *out_d) {
    ApplyArgs a;
    PXB_TRY(apply_args(c, nk, slots, a, "pxb_apply"));
    if (!u_d || !out_d) return fail(PXB_ERR_INVALID, "pxb_apply: NULL buffer");
    a.u = u_d;
    a.out = out_d;
    launch_apply(a, c->ops.precision == PXB_MIXED, grid_nodes(a.n, kApplyThreads), c->stream);
    return check_launch(c, "apply");
}

extern "C" int pxb_apply(pxb_ctx *c, const double *u, int nk, const int *slots, double *out) {
    ApplyArgs a;
    PXB_TRY(apply_args(c, nk, slots, a, "pxb_apply"));
    if (!u || !out) return fail(PXB_ERR_INVALID, "pxb_apply: NULL buffer");
    const size_t n = (size_t)c->g.n;
    void *tmp = nullptr;
    PXB_TRY(scratch(c, sizeof(double) * n * (1 + nk), &tmp));
    double *du = static_cast<double *>(tmp), *dout = du + n;
    PXB_TRY(h2d(c, du, u, sizeof(double) * n));
    PXB_TRY(pxb_apply_d(c, du, nk, slots, dout));
    PXB_TRY(d2h(c, out, dout, sizeof(double) * n * nk));
    return sync(c);
}

extern "C" int pxb_apply_adjoint_d(pxb_ctx *c, const double *ybar_d, int nk, const int *slots, double *ubar_d) {
    ApplyArgs a;
    PXB_TRY(apply_args(c, nk, slots, a, "pxb_apply_adjoint"));
    if (!ybar_d || !ubar_d) return fail(PXB_ERR_INVALID, "pxb_apply_adjoint: NULL buffer");
    PXB_TRY(ensure_rev(c));
    a.rev = c->g.rev.as<int>();
    a.u = ybar_d;
    a.out = ubar_d;
    bool second = false;
    for (int s = 0; s < nk; ++s) second |= slots[s] >= c->g.dim;
    if (a.defect && second) {
        // transpose of the defect correction: first-derivative slots join the scatter with corrected ybar
        AdjPrepArgs p;
        p.n = a.n;
        p.dim = c->g.dim;
        p.nop = a.nop;
        p.nk = nk;
        p.next = nk;
        for (int s = 0; s < nk; ++s) p.slots[s] = p.ext[s] = slots[s];
        for (int m = 0; m < c->g.dim; ++m) {
            bool have = false;
            for (int s = 0; s < nk; ++s) have |= slots[s] == m;
            if (!have) p.ext[p.next++] = m;
        }
        if (p.next > 20) return fail(PXB_ERR_INVALID, "pxb_apply_adjoint: too many slots with the defect correction");
        const size_t need = sizeof(double) * (size_t)a.n * (size_t)p.next;
        if (c->ops.yeff.bytes < need) PXB_TRY(dev_alloc(c, c->ops.yeff, need));
        p.defect = a.defect;
        p.ybar = ybar_d;
        p.yeff = c->ops.yeff.as<double>();
        PXB_CUDA_TRY(launch_apply_adjoint_prep(p, c->stream));
        PXB_TRY(check_launch(c, "apply_adjoint (defect transpose)"));
        a.nk = p.next;
        for (int s = 0; s < p.next; ++s) a.slots[s] = p.ext[s];
        a.u = p.yeff;
    }
    launch_apply_adjoint(a, c->ops.precision == PXB_MIXED, grid_nodes(a.n, kApplyThreads), c->stream);
    return check_launch(c, "apply_adjoint");
}

extern "C" int pxb_apply_adjoint(pxb_ctx *c, const double *ybar, int nk, const int *slots, double *ubar) {
    ApplyArgs a;
    PXB_TRY(apply_args(c, nk, slots, a, "pxb_apply_adjoint"));
    if (!ybar || !ubar) return fail(PXB_ERR_INVALID, "pxb_apply_adjoint: NULL buffer");
    const size_t n = (size_t)c->g.n;
    void *tmp = nullptr;
    PXB_TRY(scratch(c, sizeof(double) * n * (1 + nk), &tmp));
    double *dy = static_cast<double *>(tmp), *dout = dy + n * nk;
    PXB_TRY(h2d(c, dy, ybar, sizeof(double) * n * nk));
    PXB_TRY(pxb_apply_adjoint_d(c, dy, nk, slots, dout));
    PXB_TRY(d2h(c, ubar, dout, sizeof(double) * n));
    return sync(c);
}

// =========================================================================================== explicit fracture
static int need_epf(pxb_ctx *c, const char *who) {
    PXB_TRY(need_geometry(c, who));
    if (!c->epf.ready) return fail(PXB_ERR_STATE, std::string(who) + ": call pxb_epf_setup first");
    return PXB_OK;
}

static EpfArgs epf_args(pxb_ctx *c) {
    const Geometry &g = c->g;
    const EpfState &e = c->epf;
    EpfArgs a;
    a.n = g.n;
    a.nb = g.ldb;  // SoA stride of the operator streams
    a.off = g.off.as<int>();
    a.nbr = g.nbr.as<int>();
    a.pos = g.pos.p;
    a.G = e.G.p;
    a.health = e.health.as<uint8_t>();
    a.C11 = e.C11;
    a.C12 = e.C12;
    a.C66 = e.C66;
    a.rho = e.rho;
    for (int d = 0; d < 3; ++d) a.b[d] = e.b[d];
    a.sc = e.sc;
    a.sc_hi2 = (1.0 + e.sc) * (1.0 + e.sc);
    a.sc_lo2 = (e.sc < 1.0) ? (1.0 - e.sc) * (1.0 - e.sc) : 0.0;
    a.damage = e.sc > 0.0 ? 1 : 0;
    a.tension_only = e.tension_only;
    a.n_broken = e.counters.as<unsigned long long>();
    a.err = reinterpret_cast<unsigned int *>(e.counters.as<unsigned long long>() + 2);
    a.P = e.P.p;
    a.xib = e.xib.p ? e.xib.as<float>() : nullptr;
    if (epf_is_tma(e.variant)) a.maxb = epf_tma_maxb(g.dim, e.variant, g.max_family);
    a.evict_first = e.evict_first ? 1 : 0;
    if (e.wait_tries >= 0) a.wait_tries = e.wait_tries;
    if (e.sc_bond.p) {
        a.sc_bond = e.sc_bond.as<double>();
        a.damage = 1;
    }
    {  // displacement-first clear-hold bound (uniform critical stretch only)
        const double s = e.sc * (1.0 - 1.0e-6) - 1.0e-12;
        a.e2_hold = (e.sc > 0.0 && s > 0.0 && e.r2min > 0.0 && std::isfinite(e.r2min)) ? s * s * e.r2min : 0.0;
    }
    return a;
}

extern "C" int pxb_epf_setup(pxb_ctx *c, int precision, double C11, double C12, double C66, double rho,
                             const double *b, double sc, int tension_only, const uint8_t *health0) {
    PXB_TRY(need_geometry(c, "pxb_epf_setup"));
    if (precision != PXB_FP64 && precision != PXB_MIXED) return fail(PXB_ERR_INVALID, "pxb_epf_setup: bad precision");
    if (!(rho > 0.0)) return fail(PXB_ERR_INVALID, "pxb_epf_setup: rho must be > 0");
    Geometry &g = c->g;
    EpfState &e = c->epf;
    destroy_graphs(e);
    e = EpfState{};
    e.precision = precision;
    e.C11 = C11;
    e.C12 = C12;
    e.C66 = C66;
    e.rho = rho;
    for (int d = 0; d < g.dim; ++d) e.b[d] = b ? b[d] : 0.0;
    e.sc = sc;
    e.tension_only = tension_only ? 1 : 0;
    const int nc = g.dim == 3 ? 6 : 3;
    const size_t es = precision == PXB_MIXED ? 4 : 8;
    const size_t ldb = (size_t)g.ldb;
    PXB_TRY(dev_alloc(c, e.G, es * nc * ldb));
    PXB_CUDA_TRY(cudaMemsetAsync(e.G.p, 0, e.G.bytes, c->stream));
    PXB_TRY(dev_alloc(c, e.health, ldb));
    PXB_CUDA_TRY(cudaMemsetAsync(e.health.p, 0, e.health.bytes, c->stream));
    PXB_TRY(dev_alloc(c, e.u[0], sizeof(double) * ((size_t)g.n * g.dim + 8)));
    PXB_TRY(dev_alloc(c, e.u[1], sizeof(double) * ((size_t)g.n * g.dim + 8)));
    PXB_TRY(dev_alloc(c, e.accel, sizeof(double) * (size_t)g.n * g.dim));
    PXB_TRY(dev_alloc(c, e.counters, sizeof(unsigned long long) * 6));
    PXB_CUDA_TRY(cudaMemsetAsync(e.counters.p, 0, sizeof(unsigned long long) * 6, c->stream));
    PXB_CUDA_TRY(cudaMemsetAsync(e.u[0].p, 0, e.u[0].bytes, c->stream));
    PXB_CUDA_TRY(cudaMemsetAsync(e.u[1].p, 0, e.u[1].bytes, c->stream));
    if (health0) PXB_TRY(h2d(c, e.health.p, health0, (size_t)g.nb));
    else PXB_CUDA_TRY(cudaMemsetAsync(e.health.p, 1, (size_t)g.nb, c->stream));
    int nd = 0, first = 0;
    const int st = run_gbuild(c, 2, precision == PXB_MIXED, nullptr, e.G.p, nullptr, &nd, &first);
    if (st != PXB_OK) return st;
    PXB_TRY(dev_alloc(c, e.P, e.G.bytes));
    PXB_CUDA_TRY(launch_navier_pack(e.G.p, e.P.p, (long long)ldb, g.dim, precision == PXB_MIXED, C11, C12, C66,
                                    c->stream));
    PXB_TRY(check_launch(c, "navier pack"));
    {  // the staged kernels' FP32 bond vectors (the stretch pre-test of the configurations that stage them) and the
       // smallest bond length (the displacement-first test), its key computed in the spare counter slot 5
        PXB_TRY(dev_alloc(c, e.xib, sizeof(float) * (size_t)g.dim * ldb));
        PXB_CUDA_TRY(cudaMemsetAsync(e.xib.p, 0, e.xib.bytes, c->stream));
        unsigned long long *key = e.counters.as<unsigned long long>() + 5;
        const unsigned long long inf_key = 0x7ff0000000000000ULL;
        PXB_TRY(h2d(c, key, &inf_key, sizeof(inf_key)));
        PXB_CUDA_TRY(launch_bond_vectors(g.n, g.dim, g.off.as<int>(), g.nbr.as<int>(), g.pos.p, (long long)ldb,
                                         e.xib.as<float>(), key, c->stream));
        PXB_TRY(check_launch(c, "bond vectors"));
        unsigned long long k2 = inf_key;
        PXB_TRY(d2h(c, &k2, key, sizeof(k2)));
        PXB_CUDA_TRY(cudaStreamSynchronize(c->stream));
        std::memcpy(&e.r2min, &k2, sizeof(double));
        PXB_CUDA_TRY(cudaMemsetAsync(key, 0, sizeof(unsigned long long), c->stream));
    }
    // Bond streams larger than the L2 are staged as evict-first, so that the node rows the neighbour gathers reuse
    // stay resident; streams that fit are left to stay in L2 from one step to the next.
    int l2 = 0;
    PXB_CUDA_TRY(cudaDeviceGetAttribute(&l2, cudaDevAttrL2CacheSize, c->device));
    const size_t stream_bytes = ldb * (es * nc + 5 + 4 * (size_t)g.dim);
    e.evict_first = stream_bytes > (size_t)l2;
    e.ready = true;
    return PXB_OK;
}

// The work of one per-step rate call, queued on stream s: upload u into the state slot u[cur], snapshot the
// broken-bond count on the device, the kernel's RATE epilogue, download the acceleration and the counters.
// The pipelined rate call's chunk plan, made once per set-up: chunks of about 96 Ki nodes (at most 4; starts on
// 64-node boundaries, as the staged kernels' node ranges need), each with the chunk whose upload holds its highest
// neighbour (the upload its kernel waits for).
static int rate_plan(pxb_ctx *c) {
    EpfState &e = c->epf;
    if (e.rate_plan_done) return PXB_OK;
    e.rate_plan_done = true;
    e.rate_K = 1;
    const int n = c->g.n;
    int K = c->rate_chunks > 0 ? c->rate_chunks : std::min(4, n / 98304);
    K = std::min(K, n / 64);  // chunks of at least 64 nodes
    if (K < 2) return PXB_OK;
    std::vector<int> b((size_t)K + 1);
    for (int k = 0; k <= K; ++k) b[(size_t)k] = k == K ? n : (int)(((long long)n * k / K) & ~63LL);
    void *tmp = nullptr;
    PXB_TRY(scratch(c, sizeof(int) * (2 * (size_t)K + 1), &tmp));
    int *bd = static_cast<int *>(tmp), *reach = bd + K + 1;
    PXB_TRY(h2d(c, bd, b.data(), sizeof(int) * b.size()));
    PXB_CUDA_TRY(cudaMemsetAsync(reach, 0, sizeof(int) * K, c->stream));
    PXB_CUDA_TRY(launch_chunk_reach(c->g.off.as<int>(), c->g.nbr.as<int>(), bd, K, reach, c->stream));
    PXB_TRY(check_launch(c, "chunk reach"));
    std::vector<int> r((size_t)K);
    PXB_TRY(d2h(c, r.data(), reach, sizeof(int) * K));
    PXB_TRY(sync(c));
    e.rate_need.assign((size_t)K, K - 1);
    for (int k = 0; k < K; ++k) {
        int p = k;  // the chunk holding the chunk's highest neighbour (never below the chunk itself)
        while (p + 1 < K && b[(size_t)p + 1] <= r[(size_t)k]) ++p;
        e.rate_need[(size_t)k] = p;
    }
    e.rate_bounds = b;
    e.rate_K = K;
    return PXB_OK;
}

// pinned: both host buffers page-locked (copies from pageable memory are staged synchronously, so chunking them
// only adds per-chunk overhead)
static cudaError_t rate_ops(pxb_ctx *c, const double *u, double *accel, cudaStream_t s, bool pinned) {
    EpfState &e = c->epf;
    const size_t nd = (size_t)c->g.n * c->g.dim;
    unsigned long long *cnt = e.counters.as<unsigned long long>();
    // (a per-bond critical stretch runs the lane-group kernel, which computes every node: no chunking then)
    if (pinned && e.rate_K > 1 && epf_is_tma(e.variant) && !e.sc_bond.p) {
        // pieces of u go up on one stream, each chunk's kernel starts once its neighbours' piece is there, and each
        // chunk's acceleration goes down on another stream while the next chunk computes
        const int K = e.rate_K, dim = c->g.dim;
        cudaError_t err = cudaSuccess;
        if (!e.rate_up) err = cudaStreamCreateWithFlags(&e.rate_up, cudaStreamNonBlocking);
        if (err == cudaSuccess && !e.rate_down) err = cudaStreamCreateWithFlags(&e.rate_down, cudaStreamNonBlocking);
        while (err == cudaSuccess && e.rate_ev.size() < 2 + 2 * (size_t)K) {
            cudaEvent_t ev = nullptr;
            err = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
            if (err == cudaSuccess) e.rate_ev.push_back(ev);
        }
        if (err != cudaSuccess) return err;
        cudaEvent_t *ev = e.rate_ev.data();
        const int *b = e.rate_bounds.data();
        double *ud = e.u[e.cur].as<double>();
        auto span = [&](int k) { return (size_t)(b[k + 1] - b[k]) * dim * sizeof(double); };
        err = cudaEventRecord(ev[0], s);
        if (err == cudaSuccess) err = cudaStreamWaitEvent(e.rate_up, ev[0], 0);
        if (err == cudaSuccess) err = cudaStreamWaitEvent(e.rate_down, ev[0], 0);
        for (int p = 0; p < K && err == cudaSuccess; ++p) {
            err = cudaMemcpyAsync(ud + (size_t)b[p] * dim, u + (size_t)b[p] * dim, span(p), cudaMemcpyHostToDevice,
                                  e.rate_up);
            if (err == cudaSuccess) err = cudaEventRecord(ev[2 + p], e.rate_up);
        }
        if (err == cudaSuccess)
            err = cudaMemcpyAsync(cnt + 4, cnt, sizeof(unsigned long long), cudaMemcpyDeviceToDevice, s);
        EpfArgs a = epf_args(c);
        a.u = ud;
        a.accel = e.accel.as<double>();
        for (int k = 0; k < K && err == cudaSuccess; ++k) {
            err = cudaStreamWaitEvent(s, ev[2 + e.rate_need[(size_t)k]], 0);
            a.node0 = b[k];
            a.n = b[k + 1];
            if (err == cudaSuccess) err = launch_epf(a, dim, e.precision == PXB_MIXED, EPF_RATE, e.variant, s);
            if (err == cudaSuccess) err = cudaEventRecord(ev[2 + K + k], s);
            if (err == cudaSuccess) err = cudaStreamWaitEvent(e.rate_down, ev[2 + K + k], 0);
            if (err == cudaSuccess)
                err = cudaMemcpyAsync(accel + (size_t)b[k] * dim, e.accel.as<double>() + (size_t)b[k] * dim, span(k),
                                      cudaMemcpyDeviceToHost, e.rate_down);
        }
        if (err == cudaSuccess)
            err = cudaMemcpyAsync(e.rate_h.p, cnt, sizeof(unsigned long long) * 5, cudaMemcpyDeviceToHost,
                                  e.rate_down);
        if (err == cudaSuccess) err = cudaEventRecord(ev[1], e.rate_down);
        if (err == cudaSuccess) err = cudaStreamWaitEvent(s, ev[1], 0);
        return err;
    }
    cudaError_t err = cudaMemcpyAsync(e.u[e.cur].p, u, sizeof(double) * nd, cudaMemcpyHostToDevice, s);
    // the broken-bond count before the kernel, snapshot on the device: one host synchronisation per call
    if (err == cudaSuccess)
        err = cudaMemcpyAsync(cnt + 4, cnt, sizeof(unsigned long long), cudaMemcpyDeviceToDevice, s);
    if (err != cudaSuccess) return err;
    EpfArgs a = epf_args(c);
    a.u = e.u[e.cur].as<double>();
    a.accel = e.accel.as<double>();
    err = launch_epf(a, c->g.dim, e.precision == PXB_MIXED, EPF_RATE, e.variant, s);
    if (err == cudaSuccess)
        err = cudaMemcpyAsync(accel, e.accel.p, sizeof(double) * nd, cudaMemcpyDeviceToHost, s);
    if (err == cudaSuccess)
        err = cudaMemcpyAsync(e.rate_h.p, cnt, sizeof(unsigned long long) * 5, cudaMemcpyDeviceToHost, s);
    return err;
}

static bool pinned_host(const void *p) {
    cudaPointerAttributes at{};
    if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return at.type == cudaMemoryTypeHost;
}

// Captures rate_ops for the current buffers on the context's own stream (never the legacy default stream); the
// graph is replayed on c->stream.  One graph launch replaces five submissions per call.
static int capture_rate(pxb_ctx *c, const double *u, double *accel) {
    EpfState &e = c->epf;
    if (e.rate_graph) cudaGraphExecDestroy(e.rate_graph);
    e.rate_graph = nullptr;
    cudaGraph_t graph = nullptr;
    PXB_CUDA_TRY(cudaStreamBeginCapture(c->own, cudaStreamCaptureModeThreadLocal));
    const cudaError_t oe = rate_ops(c, u, accel, c->own, true);
    const cudaError_t ce = cudaStreamEndCapture(c->own, &graph);
    if (oe != cudaSuccess || ce != cudaSuccess) {
        if (graph) cudaGraphDestroy(graph);
        return cuda_fail(oe != cudaSuccess ? oe : ce, "per-step rate capture");
    }
    const cudaError_t ie = cudaGraphInstantiate(&e.rate_graph, graph, 0);
    cudaGraphDestroy(graph);
    if (ie != cudaSuccess) {
        e.rate_graph = nullptr;
        return cuda_fail(ie, "cudaGraphInstantiate (per-step rate)");
    }
    e.rate_u = u;
    e.rate_a = accel;
    e.rate_cur = e.cur;
    e.rate_variant = e.variant;
    return PXB_OK;
}

extern "C" int pxb_epf_rate(pxb_ctx *c, const double *u, double *accel, long long *n_broken) {
    PXB_TRY(need_epf(c, "pxb_epf_rate"));
    if (!u || !accel) return fail(PXB_ERR_INVALID, "pxb_epf_rate: NULL buffer");
    EpfState &e = c->epf;
    PXB_TRY(ensure_pinned(e.rate_h, sizeof(unsigned long long) * 5));
    PXB_TRY(rate_plan(c));
    // pinned buffers that the previous call used too, with the same schedule: replay (or capture) the call as one
    // graph; otherwise (first call with these buffers or this schedule, or pageable memory) queue the operations
    // one by one, which also gives a kernel its first, uncaptured launch
    const bool again = u == e.rate_last_u && accel == e.rate_last_a && e.variant == e.rate_last_variant;
    e.rate_last_u = u;
    e.rate_last_a = accel;
    e.rate_last_variant = e.variant;
    if (again && pinned_host(u) && pinned_host(accel)) {
        if (!e.rate_graph || e.rate_u != u || e.rate_a != accel || e.rate_cur != e.cur || e.rate_variant != e.variant)
            PXB_TRY(capture_rate(c, u, accel));
        PXB_CUDA_TRY(cudaGraphLaunch(e.rate_graph, c->stream));
        c->launches++;
    } else {
        const cudaError_t err = rate_ops(c, u, accel, c->stream, pinned_host(u) && pinned_host(accel));
        if (err != cudaSuccess) return cuda_fail(err, "epf rate");
        PXB_TRY(check_launch(c, "epf rate"));
    }
    unsigned long long *h = static_cast<unsigned long long *>(e.rate_h.p);
    PXB_TRY(sync_polled(c, e.rate_done));
    const unsigned int werr = static_cast<unsigned int>(h[2] & 0xffffffffULL);
    if (werr) return wait_failure(c, werr, "explicit rate");
    if (n_broken) *n_broken = (long long)(h[0] - h[4]);
    return PXB_OK;
}

// Output projections (ExplicitPDDOFracElement::computeNodalProjection, ExplicitPDDOFracElement.cpp:324-405) of u_d
// (NULL: the current state u^n) with the current bond health.  The first-derivative operators come from the
// context's FP64 order-2 operator cache, built here when absent (the step itself keeps only the Navier streams).
// the FP64 order-2 operator cache the projections read (built once; it uses the context scratch buffer, so it
// runs before anything is staged there)
static int ensure_fp64_ops(pxb_ctx *c) {
    const OpsCache &o = c->ops;
    if (o.ready && o.order == 2 && o.precision == PXB_FP64) return PXB_OK;
    int nd = 0, first = 0;
    const int st = pxb_gbuild(c, 2, PXB_FP64, &nd, &first);
    return st == PXB_ERR_DEGENERATE ? PXB_OK : st;  // degenerate rows carry zero operators
}

extern "C" int pxb_epf_project_d(pxb_ctx *c, const double *u_d, int plane_strain, double *damage_d,
                                 double *von_mises_d, double *stress_d, double *strain_d) {
    PXB_TRY(need_epf(c, "pxb_epf_project"));
    PXB_TRY(ensure_fp64_ops(c));
    const OpsCache &o = c->ops;
    const EpfState &e = c->epf;
    auto slot = [&](int pp, int q, int r) {
        for (int s = 0; s < o.nop; ++s)
            if (o.pqr[3 * s] == pp && o.pqr[3 * s + 1] == q && o.pqr[3 * s + 2] == r) return s;
        return -1;
    };
    ProjectArgs a;
    a.n = c->g.n;
    a.dim = c->g.dim;
    a.nop = o.nop;
    a.plane_strain = plane_strain ? 1 : 0;
    a.sl[0] = slot(1, 0, 0);
    a.sl[1] = slot(0, 1, 0);
    a.sl[2] = c->g.dim == 3 ? slot(0, 0, 1) : -1;
    a.C12 = e.C12;
    a.C66 = e.C66;
    a.off = c->g.off.as<int>();
    a.nbr = c->g.nbr.as<int>();
    a.ops = o.ops.as<double>();
    a.health = e.health.as<uint8_t>();
    a.u = u_d ? u_d : e.u[e.cur].as<double>();
    a.damage = damage_d;
    a.von_mises = von_mises_d;
    a.stress = stress_d;
    a.strain = strain_d;
    PXB_CUDA_TRY(launch_epf_project(a, c->stream));
    return check_launch(c, "epf project");
}

extern "C" int pxb_epf_project(pxb_ctx *c, const double *u, int plane_strain, double *damage, double *von_mises,
                               double *stress, double *strain) {
    PXB_TRY(need_epf(c, "pxb_epf_project"));
    PXB_TRY(ensure_fp64_ops(c));
    const size_t n = (size_t)c->g.n, nd = n * c->g.dim;
    void *tmp = nullptr;
    PXB_TRY(scratch(c, sizeof(double) * (nd + 20 * n), &tmp));
    double *du = static_cast<double *>(tmp), *dd = du + nd, *dv = dd + n, *ds = dv + n, *de = ds + 9 * n;
    if (u) PXB_TRY(h2d(c, du, u, sizeof(double) * nd));
    PXB_TRY(pxb_epf_project_d(c, u ? du : nullptr, plane_strain, damage ? dd : nullptr, von_mises ? dv : nullptr,
                              stress ? ds : nullptr, strain ? de : nullptr));
    if (damage) PXB_TRY(d2h(c, damage, dd, sizeof(double) * n));
    if (von_mises) PXB_TRY(d2h(c, von_mises, dv, sizeof(double) * n));
    if (stress) PXB_TRY(d2h(c, stress, ds, sizeof(double) * 9 * n));
    if (strain) PXB_TRY(d2h(c, strain, de, sizeof(double) * 9 * n));
    return sync(c);
}

// ---- BC program: the reference applies BCs one after another (BCSystem.cpp:114-129); each write either
//      copies/reflects a mirror value or pins g(t).  Symbolic replay on the host reduces every constrained
//      (node, component) to one of four closed forms in terms of pre-BC values, executed on the device by the
//      warp of the node whose integrated value it needs (or by the target's own warp for constants). ----------
namespace {
struct Sym {
    int form = -1;  // -1 untouched (= U(self)), 0 U(src), 1 G, 2 2G-U(src), 3 2G-G2
    int src = -1;
    double val = 0, vel = 0, val2 = 0, vel2 = 0;
};
}  // namespace

extern "C" int pxb_epf_set_bcs(pxb_ctx *c, int nbc, const int *kind, const int *comp_mask, const int *direct,
                               const double *value, const double *velocity, const int *has_box, const double *box,
                               const int *node_off, const int *nodes) {
    PXB_TRY(need_epf(c, "pxb_epf_set_bcs"));
    Geometry &g = c->g;
    EpfState &e = c->epf;
    destroy_graphs(e);
    e.has_bc = false;
    e.bc = BcDevice{};
    if (nbc <= 0) return PXB_OK;
    if (!kind || !comp_mask || !node_off || !nodes) return fail(PXB_ERR_INVALID, "pxb_epf_set_bcs: NULL array");
    const int dim = g.dim;
    // host coordinates are needed for the box test: fetch positions back once
    std::vector<double> pos((size_t)g.n * (dim == 2 ? 2 : 4));
    PXB_TRY(d2h(c, pos.data(), g.pos.p, pos.size() * sizeof(double)));
    PXB_TRY(sync(c));
    auto X = [&](int i, int a) { return pos[(size_t)i * (dim == 2 ? 2 : 4) + a]; };
    const std::vector<int> &mir = g.h_mirror;
    std::vector<Sym> sym((size_t)g.n * dim);
    auto cur = [&](int node, int comp) -> Sym {
        Sym s = sym[(size_t)node * dim + comp];
        if (s.form < 0) { s.form = 0; s.src = node; }
        return s;
    };
    for (int b = 0; b < nbc; ++b) {
        for (int p = node_off[b]; p < node_off[b + 1]; ++p) {
            const int id = nodes[p];
            if (id < 1 || id > g.n) return fail(PXB_ERR_INVALID, "pxb_epf_set_bcs: node id out of range");
            const int i = id - 1;
            const int mb = mir.empty() ? 0 : mir[(size_t)i];
            if (kind[b] == 0) {
                if (has_box && has_box[b]) {
                    // DirichletBC::insideBox (DirichletBC.cpp:89-98): every axis of the xyz coordinates (z = 0 in
                    // 2D), an axis whose min exceeds its max leaves that axis unconstrained
                    bool inside = true;
                    for (int a = 0; a < 3; ++a) {
                        const double lo = box[6 * b + 2 * a], hi = box[6 * b + 2 * a + 1];
                        if (lo > hi) continue;
                        const double x = a < dim ? X(i, a) : 0.0;
                        if (x < lo || x > hi) inside = false;
                    }
                    if (!inside) continue;
                }
                for (int a = 0; a < dim; ++a) {
                    if (!((comp_mask[b] >> a) & 1)) continue;
                    Sym s;
                    const double v = value ? value[b * dim + a] : 0.0, w = velocity ? velocity[b * dim + a] : 0.0;
                    if (mb >= 1 && !(direct && direct[b])) {
                        const Sym m = cur(mb - 1, a);
                        if (m.form == 0) { s.form = 2; s.src = m.src; s.val = v; s.vel = w; }
                        else if (m.form == 1) { s.form = 3; s.val = v; s.vel = w; s.val2 = m.val; s.vel2 = m.vel; }
                        else return fail(PXB_ERR_UNSUPPORTED, "pxb_epf_set_bcs: reflection off a reflected node");
                    } else {
                        s.form = 1; s.val = v; s.vel = w;
                    }
                    sym[(size_t)i * dim + a] = s;
                }
            } else {
                // NeumannBC::presetSolution (NeumannBC.cpp:88-105) copies from the mirror bulk and aborts the run
                // for a node without one (checkedMirror); here that is an error
                if (mb < 1)
                    return fail(PXB_ERR_INVALID, "pxb_epf_set_bcs: Neumann entry " + std::to_string(b) + " names node " +
                                                     std::to_string(id) + ", which has no mirror bulk node");
                for (int a = 0; a < dim; ++a)
                    if ((comp_mask[b] >> a) & 1) sym[(size_t)i * dim + a] = cur(mb - 1, a);
            }
        }
    }
    // group entries by executor node
    std::vector<uint8_t> own((size_t)g.n, 0);
    std::vector<std::vector<int>> by((size_t)g.n);
    int nent = 0;
    for (int i = 0; i < g.n; ++i)
        for (int a = 0; a < dim; ++a) {
            const Sym &s = sym[(size_t)i * dim + a];
            if (s.form < 0) continue;
            if (s.form == 0 && s.src == i) continue;  // identity
            own[(size_t)i] |= (uint8_t)(1u << a);
            const int ex = (s.form == 0 || s.form == 2) ? s.src : i;
            by[(size_t)ex].push_back(i * dim + a);
            ++nent;
        }
    std::vector<int> off((size_t)g.n + 1, 0), tgt, comp, form;
    std::vector<double> val, vel, val2, vel2;
    for (int i = 0; i < g.n; ++i) {
        for (int key : by[(size_t)i]) {
            const Sym &s = sym[(size_t)key];
            tgt.push_back(key / dim);
            comp.push_back(key % dim);
            form.push_back(s.form);
            val.push_back(s.val);
            vel.push_back(s.vel);
            val2.push_back(s.val2);
            vel2.push_back(s.vel2);
        }
        off[(size_t)i + 1] = (int)tgt.size();
    }
    BcDevice &d = e.bc;
    d.n_entries = nent;
    PXB_TRY(dev_upload(c, d.own, own.data(), own.size()));
    PXB_TRY(dev_upload(c, d.src_off, off.data(), off.size() * sizeof(int)));
    if (nent > 0) {
        PXB_TRY(dev_upload(c, d.tgt, tgt.data(), tgt.size() * sizeof(int)));
        PXB_TRY(dev_upload(c, d.comp, comp.data(), comp.size() * sizeof(int)));
        std::vector<double> packed;
        packed.reserve((size_t)nent * 4);
        packed.insert(packed.end(), val.begin(), val.end());
        packed.insert(packed.end(), vel.begin(), vel.end());
        packed.insert(packed.end(), val2.begin(), val2.end());
        packed.insert(packed.end(), vel2.begin(), vel2.end());
        PXB_TRY(dev_upload(c, d.vals, packed.data(), packed.size() * sizeof(double)));
        PXB_TRY(dev_upload(c, d.form, form.data(), form.size() * sizeof(int)));
    }
    PXB_TRY(sync(c));
    e.has_bc = true;
    return PXB_OK;
}

static void fill_bc(const pxb_ctx *c, EpfArgs &a) {
    const EpfState &e = c->epf;
    if (!e.has_bc) return;
    const BcDevice &d = e.bc;
    const int ne = d.n_entries;
    a.bc_own = d.own.as<uint8_t>();
    a.bc_off = d.src_off.as<int>();
    if (ne > 0) {
        a.bc_tgt = d.tgt.as<int>();
        a.bc_comp = d.comp.as<int>();
        a.bc_form = d.form.as<int>();
        const double *p = d.vals.as<double>();
        a.bc_val = p;
        a.bc_vel = p + ne;
        a.bc_val2 = p + 2 * (size_t)ne;
        a.bc_vel2 = p + 3 * (size_t)ne;
    }
}

extern "C" int pxb_epf_start(pxb_ctx *c, const double *u0, const double *v0, double dt) {
    PXB_TRY(need_epf(c, "pxb_epf_start"));
    if (!u0 || !(dt > 0.0)) return fail(PXB_ERR_INVALID, "pxb_epf_start: need u0 and dt > 0");
    EpfState &e = c->epf;
    const size_t nd = (size_t)c->g.n * c->g.dim;
    e.cur = 0;
    PXB_TRY(h2d(c, e.u[0].p, u0, sizeof(double) * nd));
    void *tmp = nullptr;
    const double *dv0 = nullptr;
    if (v0) {
        PXB_TRY(scratch(c, sizeof(double) * nd, &tmp));
        PXB_TRY(h2d(c, tmp, v0, sizeof(double) * nd));
        dv0 = static_cast<const double *>(tmp);
    }
    EpfArgs a = epf_args(c);
    a.u = e.u[0].as<double>();
    a.u_other = e.u[1].as<double>();
    a.v0 = dv0;
    a.dt = dt;
    a.dt2 = 0.5 * dt * dt;
    launch_epf(a, c->g.dim, e.precision == PXB_MIXED, EPF_START, e.variant, c->stream);
    PXB_TRY(check_launch(c, "epf start"));
    PXB_TRY(sync(c));
    e.dt = dt;
    e.t = 0.0;
    e.step = 0;
    e.dt_prev = dt;
    e.umax_hist.clear();
    e.started = true;
    return PXB_OK;
}

namespace pxb {
// argument block of one STEP launch at ping-pong parity par (reads u[par], writes u[par^1])
int step_args(pxb_ctx *c, int par, EpfArgs *out) {
    EpfState &e = c->epf;
    EpfArgs a = epf_args(c);
    fill_bc(c, a);
    a.u = e.u[par].as<double>();
    a.u_other = e.u[par ^ 1].as<double>();
    a.dt = e.dt;
    a.dt2 = e.dt * e.dt;
    a.t_sched = e.tsched.as<double>();
    a.step_in_chunk = 0;
    a.umax = e.umax.as<unsigned long long>();
    *out = a;
    return PXB_OK;
}

// argument block of one RATE launch of the per-step rate call: reads u[cur], writes the acceleration
int rate_args(pxb_ctx *c, EpfArgs *out) {
    EpfState &e = c->epf;
    EpfArgs a = epf_args(c);
    a.u = e.u[e.cur].as<double>();
    a.accel = e.accel.as<double>();
    *out = a;
    return PXB_OK;
}
}  // namespace pxb

// one STEP launch on stream s: reads u[par], writes u[par^1]
static int launch_step(pxb_ctx *c, int par, int q, cudaStream_t s, bool pdl = false) {
    EpfState &e = c->epf;
    EpfArgs a;
    step_args(c, par, &a);
    a.step_in_chunk = q;
    a.pdl = pdl ? 1 : 0;
    const cudaError_t err = launch_epf(a, c->g.dim, e.precision == PXB_MIXED, EPF_STEP, e.variant, s);
    if (err != cudaSuccess) return cuda_fail(err, "epf step launch");
    return PXB_OK;
}

static int get_graph(pxb_ctx *c, int steps, cudaGraphExec_t *out) {
    EpfState &e = c->epf;
    const GraphKey key{steps, e.cur, e.precision, e.variant};
    auto it = e.graphs.find(key);
    if (it != e.graphs.end()) { *out = it->second; return PXB_OK; }
    // captured on the context's own stream (never the legacy default stream), replayed on c->stream
    cudaGraph_t graph = nullptr;
    PXB_CUDA_TRY(cudaStreamBeginCapture(c->own, cudaStreamCaptureModeThreadLocal));
    int par = e.cur, st = PXB_OK;
    for (int q = 0; q < steps && st == PXB_OK; ++q) {
        st = launch_step(c, par, q, c->own, /*pdl=*/q > 0);
        par ^= 1;
    }
    cudaError_t ce = cudaStreamEndCapture(c->own, &graph);
    if (st != PXB_OK) { if (graph) cudaGraphDestroy(graph); return st; }
    if (ce != cudaSuccess) return cuda_fail(ce, "cudaStreamEndCapture");
    cudaGraphExec_t exec = nullptr;
    ce = cudaGraphInstantiate(&exec, graph, 0);
    cudaGraphDestroy(graph);
    if (ce != cudaSuccess) return cuda_fail(ce, "cudaGraphInstantiate");
    e.graphs[key] = exec;
    *out = exec;
    return PXB_OK;
}

// reference blow-up guard (TimeStepping.cpp:550-573): 50-step window, x1e3 growth, non-finite
static int check_blowup(EpfState &e, const unsigned long long *keys, int steps, int *bad_step) {
    for (int q = 0; q < steps; ++q) {
        double umax;
        std::memcpy(&umax, &keys[q], sizeof(double));
        const long long step = e.step + q + 1;
        const bool finite = umax <= std::numeric_limits<double>::max();
        double cap = std::numeric_limits<double>::infinity();
        if (step > 50) cap = 1.0e3 * std::max(1.0, e.umax_hist[(size_t)(step - 1 - 50)]);
        if (!finite || umax > cap) {
            if (bad_step) *bad_step = (int)step;
            return fail(PXB_ERR_BLOWUP, "explicit loop blew up at step " + std::to_string(step) +
                                            (finite ? " (max|U| grew more than 1e3x in 50 steps)" : " (non-finite U)") +
                                            ": reduce dt below the CFL limit");
        }
        e.umax_hist.push_back(umax);
    }
    return PXB_OK;
}

extern "C" int pxb_epf_advance(pxb_ctx *c, int nsteps, int chunk, int *bad_step) {
    PXB_TRY(need_epf(c, "pxb_epf_advance"));
    EpfState &e = c->epf;
    if (!e.started) return fail(PXB_ERR_STATE, "pxb_epf_advance: call pxb_epf_start first");
    if (nsteps < 0) return fail(PXB_ERR_INVALID, "pxb_epf_advance: nsteps < 0");
    if (bad_step) *bad_step = 0;
    if (chunk <= 0) chunk = 200;
    chunk = std::min(chunk, std::max(1, nsteps));
    if (e.graph_chunk < chunk) {
        PXB_TRY(dev_alloc(c, e.umax, sizeof(unsigned long long) * (size_t)chunk));
        PXB_TRY(dev_alloc(c, e.tsched, sizeof(double) * (size_t)chunk));
        PXB_TRY(ensure_pinned(e.tsched_h, sizeof(double) * (size_t)chunk * 2 + 16));
        destroy_graphs(e);
        e.graph_chunk = chunk;
    }
    int done = 0;
    std::vector<unsigned long long> keys((size_t)chunk);
    while (done < nsteps) {
        const int s = std::min(chunk, nsteps - done);
        double *th = static_cast<double *>(e.tsched_h.p);
        double t = e.t;
        for (int q = 0; q < s; ++q) { t = t + e.dt; th[q] = t; }
        PXB_TRY(h2d(c, e.tsched.p, th, sizeof(double) * (size_t)s));
        PXB_CUDA_TRY(cudaMemsetAsync(e.umax.p, 0, sizeof(unsigned long long) * (size_t)s, c->stream));
        cudaGraphExec_t exec = nullptr;
        PXB_TRY(get_graph(c, s, &exec));
        PXB_CUDA_TRY(cudaGraphLaunch(exec, c->stream));
        c->launches += s;
        PXB_TRY(d2h(c, keys.data(), e.umax.p, sizeof(unsigned long long) * (size_t)s));
        unsigned int werr = 0;
        PXB_TRY(d2h(c, &werr, e.counters.as<unsigned long long>() + 2, sizeof(unsigned int)));
        PXB_TRY(sync(c));
        if (werr) return wait_failure(c, werr, "explicit step");
        const int st = check_blowup(e, keys.data(), s, bad_step);
        e.cur ^= (s & 1);
        e.t = t;
        e.step += s;
        e.dt_prev = e.dt;
        done += s;
        if (st != PXB_OK) return st;
    }
    return PXB_OK;
}

// One step of length dtA launched alone, with the BC pass at t + dtA and the blow-up guard: the uniform form with
// dt^2 = dtA^2 when dtA equals the previous step's dt, else the variable-step central difference
// (TimeStepping.cpp:529-545).
static int single_step(pxb_ctx *c, double dtA, int *bad_step) {
    EpfState &e = c->epf;
    if (e.graph_chunk < 1) {
        PXB_TRY(dev_alloc(c, e.umax, sizeof(unsigned long long)));
        PXB_TRY(dev_alloc(c, e.tsched, sizeof(double)));
        PXB_TRY(ensure_pinned(e.tsched_h, 64));
        e.graph_chunk = 1;
    }
    const double t_new = e.t + dtA;
    double *th = static_cast<double *>(e.tsched_h.p);
    PXB_TRY(sync(c));
    th[0] = t_new;
    PXB_TRY(h2d(c, e.tsched.p, th, sizeof(double)));
    PXB_CUDA_TRY(cudaMemsetAsync(e.umax.p, 0, sizeof(unsigned long long), c->stream));
    EpfArgs a;
    PXB_TRY(step_args(c, e.cur, &a));
    a.step_in_chunk = 0;
    a.dt2 = dtA * dtA;
    a.var_step = dtA == e.dt_prev ? 0 : 1;
    a.cv_rho = dtA / e.dt_prev;
    a.cv_w = 0.5 * dtA * (dtA + e.dt_prev);
    const cudaError_t err = launch_epf(a, c->g.dim, e.precision == PXB_MIXED, EPF_STEP, e.variant, c->stream);
    if (err != cudaSuccess) return cuda_fail(err, "epf variable step launch");
    c->launches++;
    unsigned long long key = 0;
    unsigned int werr = 0;
    PXB_TRY(d2h(c, &key, e.umax.p, sizeof(key)));
    PXB_TRY(d2h(c, &werr, e.counters.as<unsigned long long>() + 2, sizeof(unsigned int)));
    PXB_TRY(sync(c));
    if (werr) return wait_failure(c, werr, "explicit step");
    const int st = check_blowup(e, &key, 1, bad_step);
    e.cur ^= 1;
    e.t = t_new;
    e.step += 1;
    e.dt_prev = dtA;
    return st;
}

extern "C" int pxb_epf_advance_to(pxb_ctx *c, double t_end, int chunk, int *bad_step, long long *steps_taken) {
    PXB_TRY(need_epf(c, "pxb_epf_advance_to"));
    EpfState &e = c->epf;
    if (!e.started) return fail(PXB_ERR_STATE, "pxb_epf_advance_to: call pxb_epf_start first");
    if (!(t_end > 0.0)) return fail(PXB_ERR_INVALID, "pxb_epf_advance_to: t_end must be > 0");
    if (bad_step) *bad_step = 0;
    const long long step0 = e.step;
    // the reference's loop (TimeStepping.cpp:495-599): while t < T - 1e-12 T, dt_attempt = min(dt, T - t); a step
    // whose dt_attempt equals the previous step's dt is uniform, any other takes the variable-step form
    const double t_eps = 1.0e-12 * t_end;
    int st = PXB_OK;
    while (st == PXB_OK && e.t < t_end - t_eps) {
        const double dtA = std::min(e.dt, t_end - e.t);
        if (dtA == e.dt && e.dt_prev == e.dt) {
            // the run of uniform steps up to the clamp, t accumulated exactly like the reference loop
            long long k = 0;
            double t = e.t;
            while (t < t_end - t_eps && std::min(e.dt, t_end - t) == e.dt) {
                t = t + e.dt;
                ++k;
            }
            while (st == PXB_OK && k > 0) {
                const int s = (int)std::min<long long>(k, 1 << 30);
                st = pxb_epf_advance(c, s, chunk, bad_step);
                k -= s;
            }
        } else {
            st = single_step(c, dtA, bad_step);
        }
    }
    if (steps_taken) *steps_taken = e.step - step0;
    return st;
}

extern "C" int pxb_ctx_set_memory_limit(pxb_ctx *c, size_t bytes) {
    if (!c) return fail(PXB_ERR_INVALID, "pxb_ctx_set_memory_limit: NULL context");
    c->mem_limit = bytes;
    return PXB_OK;
}

extern "C" int pxb_epf_set_wait_budget(pxb_ctx *c, int tries) {
    PXB_TRY(need_epf(c, "pxb_epf_set_wait_budget"));
    EpfState &e = c->epf;
    e.wait_tries = tries < 0 ? -1 : tries;
    destroy_graphs(e);  // captured steps carry the old budget
    if (e.rate_graph) cudaGraphExecDestroy(e.rate_graph);
    e.rate_graph = nullptr;
    return PXB_OK;
}

extern "C" int pxb_epf_get_state(pxb_ctx *c, double *u, double *u_prev, uint8_t *health, double *t) {
    PXB_TRY(need_epf(c, "pxb_epf_get_state"));
    EpfState &e = c->epf;
    const size_t nd = (size_t)c->g.n * c->g.dim;
    if (u) PXB_TRY(d2h(c, u, e.u[e.cur].p, sizeof(double) * nd));
    if (u_prev) PXB_TRY(d2h(c, u_prev, e.u[e.cur ^ 1].p, sizeof(double) * nd));
    if (health) PXB_TRY(d2h(c, health, e.health.p, (size_t)c->g.nb));
    if (t) *t = e.t;
    return sync(c);
}

extern "C" int pxb_epf_set_state(pxb_ctx *c, const double *u, const double *u_prev, const uint8_t *health, double t) {
    PXB_TRY(need_epf(c, "pxb_epf_set_state"));
    EpfState &e = c->epf;
    const size_t nd = (size_t)c->g.n * c->g.dim;
    if (u) PXB_TRY(h2d(c, e.u[e.cur].p, u, sizeof(double) * nd));
    if (u_prev) PXB_TRY(h2d(c, e.u[e.cur ^ 1].p, u_prev, sizeof(double) * nd));
    if (health) PXB_TRY(h2d(c, e.health.p, health, (size_t)c->g.nb));
    e.t = t;
    if (u && u_prev) e.started = true;
    return sync(c);
}

extern "C" int pxb_epf_broken_count(pxb_ctx *c, long long *n_broken) {
    PXB_TRY(need_epf(c, "pxb_epf_broken_count"));
    if (!n_broken) return fail(PXB_ERR_INVALID, "pxb_epf_broken_count: NULL");
    void *tmp = nullptr;
    PXB_TRY(scratch(c, 8, &tmp));
    PXB_CUDA_TRY(cudaMemsetAsync(tmp, 0, 8, c->stream));
    launch_count_zero(c->g.nb, c->epf.health.as<uint8_t>(), static_cast<unsigned long long *>(tmp), c->stream);
    PXB_TRY(check_launch(c, "count_zero"));
    unsigned long long h = 0;
    PXB_TRY(d2h(c, &h, tmp, 8));
    PXB_TRY(sync(c));
    *n_broken = (long long)h;
    return PXB_OK;
}

extern "C" int pxb_epf_force_frozen_d(pxb_ctx *c, const double *u_d, double *a_d) {
    PXB_TRY(need_epf(c, "pxb_epf_force_frozen"));
    if (!u_d || !a_d) return fail(PXB_ERR_INVALID, "pxb_epf_force_frozen: NULL buffer");
    EpfArgs a = epf_args(c);
    a.u = u_d;
    a.accel = a_d;
    a.damage = 0;
    launch_epf(a, c->g.dim, c->epf.precision == PXB_MIXED, EPF_FORCE_FROZEN, c->epf.variant, c->stream);
    return check_launch(c, "epf force (frozen mask)");
}

// s_c from the fracture energy (reference include/ElmtSystem/FractureCriterion.h:30-43): 3D 5 G0 / (6 E delta),
// plane stress 4 pi G0 / (9 E delta), plane strain 5 pi G0 / (12 E delta); 0 when a value is not positive
static double critical_stretch(double G0, double E, double delta, int dim, bool plane_stress) {
    if (G0 <= 0.0 || E <= 0.0 || delta <= 0.0) return 0.0;
    if (dim >= 3) return std::sqrt(5.0 * G0 / (6.0 * E * delta));
    if (plane_stress) return std::sqrt(4.0 * M_PI * G0 / (9.0 * E * delta));
    return std::sqrt(5.0 * M_PI * G0 / (12.0 * E * delta));
}

extern "C" int pxb_epf_set_variable_horizon_stretch(pxb_ctx *c, double G0, double E, int plane_stress) {
    PXB_TRY(need_epf(c, "pxb_epf_set_variable_horizon_stretch"));
    Geometry &g = c->g;
    EpfState &e = c->epf;
    if (g.h_node_delta.empty())
        return fail(PXB_ERR_STATE, "pxb_epf_set_variable_horizon_stretch: no node horizons (pxb_set_node_horizons)");
    std::vector<int> nbr((size_t)std::max(1LL, g.nb));
    PXB_TRY(d2h(c, nbr.data(), g.nbr.p, sizeof(int) * (size_t)g.nb));
    PXB_TRY(sync(c));
    std::vector<double> sc((size_t)g.ldb, 0.0);
    const bool ps = g.dim < 3 && plane_stress != 0;
    for (int i = 0; i < g.n; ++i) {
        const double di = g.h_node_delta[(size_t)i];
        for (int t = g.h_off[(size_t)i]; t < g.h_off[(size_t)i + 1]; ++t) {
            const double db = 0.5 * (di + g.h_node_delta[(size_t)nbr[(size_t)t]]);
            sc[(size_t)t] = critical_stretch(G0, E, db, g.dim, ps);
        }
    }
    destroy_graphs(e);
    if (e.rate_graph) cudaGraphExecDestroy(e.rate_graph);
    e.rate_graph = nullptr;
    PXB_TRY(dev_upload(c, e.sc_bond, sc.data(), sizeof(double) * sc.size()));
    return sync(c);
}

extern "C" int pxb_epf_set_constants(pxb_ctx *c, double C11, double C12, double C66, double rho) {
    PXB_TRY(need_epf(c, "pxb_epf_set_constants"));
    if (!(rho > 0.0)) return fail(PXB_ERR_INVALID, "pxb_epf_set_constants: rho must be > 0");
    EpfState &e = c->epf;
    destroy_graphs(e);  // captured launches carry the old constants
    e.C11 = C11;
    e.C12 = C12;
    e.C66 = C66;
    e.rho = rho;
    PXB_CUDA_TRY(launch_navier_pack(e.G.p, e.P.p, (long long)c->g.ldb, c->g.dim, e.precision == PXB_MIXED, C11, C12,
                                    C66, c->stream));
    return check_launch(c, "navier pack");
}

extern "C" int pxb_epf_force_adjoint_d(pxb_ctx *c, const double *u_d, const double *abar_d, double *ubar_d,
                                       double *dC_d) {
    PXB_TRY(need_epf(c, "pxb_epf_force_adjoint"));
    if (!u_d || !abar_d || !ubar_d) return fail(PXB_ERR_INVALID, "pxb_epf_force_adjoint: NULL buffer");
    PXB_TRY(ensure_rev(c));
    const EpfState &e = c->epf;
    EpfAdjArgs a;
    a.n = c->g.n;
    a.nb = c->g.ldb;  // SoA stride of the operator streams
    a.off = c->g.off.as<int>();
    a.nbr = c->g.nbr.as<int>();
    a.rev = c->g.rev.as<int>();
    a.G = e.G.p;
    a.health = e.health.as<uint8_t>();
    a.C11 = e.C11;
    a.C12 = e.C12;
    a.C66 = e.C66;
    a.inv_rho = 1.0 / e.rho;
    a.u = u_d;
    a.abar = abar_d;
    a.ubar = ubar_d;
    a.dC = dC_d;
    if (dC_d) PXB_CUDA_TRY(cudaMemsetAsync(dC_d, 0, 3 * sizeof(double), c->stream));
    launch_epf_adjoint(a, c->g.dim, e.precision == PXB_MIXED, epf_grid(c->g.n, c->g.dim, 0), c->stream);
    return check_launch(c, "epf adjoint");
}

// ---- adjoint of the explicit loop with a frozen damage mask ------------------------------------------------------
// Forward (the reference loop, TimeStepping.cpp:479-536, with the context's BC program after every step):
//   u^{-1} = u0 - dt v0 + dt^2/2 a(u0),  w^n = 2u^n - u^{n-1} + dt^2 a(u^n),  u^{n+1} = P w^n + g(t_{n+1}),
// a(u) = (L(C) u + b)/rho linear in u for a fixed health mask.  Reverse, with A = dJ/du^{n+1} and R = the part of
// dJ/du^n carried from step n+1 (where u^n is the previous state):
//   W = P^T A;  A <- R + 2 W + (da/du)^T (dt^2 W);  R <- -W;  dJ/dC += (da/dC(u^n))^T (dt^2 W)
// and at the start  dJ/du0 = A + R + (da/du)^T (dt^2/2 R),  dJ/dv0 = -dt R,  dJ/dC += (da/dC(u0))^T (dt^2/2 R).
// The forward states for dJ/dC come from checkpoints every `checkpoint_every` steps, recomputed segment by segment.
namespace {

// one STEP launch of the forward loop on explicit buffers: reads cur (u^n) and other (u^{n-1}), writes u^{n+1}
// into other; the BC pass at t_sched[q]; damage off (frozen mask)
int adj_step(pxb_ctx *c, double *cur, double *other, const double *tsched, int q, double dt) {
    EpfState &e = c->epf;
    EpfArgs a;
    PXB_TRY(step_args(c, 0, &a));
    a.dt = dt;
    a.dt2 = dt * dt;
    a.u = cur;
    a.u_other = other;
    a.t_sched = tsched;
    a.step_in_chunk = q;
    a.umax = e.adj_umax.as<unsigned long long>();
    a.damage = 0;
    a.sc_bond = nullptr;
    a.pdl = 0;
    const cudaError_t err = launch_epf(a, c->g.dim, e.precision == PXB_MIXED, EPF_STEP, e.variant, c->stream);
    if (err != cudaSuccess) return cuda_fail(err, "adjoint forward step");
    c->launches++;
    return PXB_OK;
}

// staged: the recorded sweep's per-step call, whose u, w and rin rows the staged reverse-only kernel (adjoint
// schedule 2) may copy in bulk (16-byte aligned, padded buffers)
int adj_kernel(pxb_ctx *c, const double *u, const double *w, double scale, double c_r, const double *rin, double c_w,
               double *ubar, double c_o, double *rout, bool staged = false, const double *uw = nullptr) {
    const EpfState &e = c->epf;
    EpfAdjArgs a;
    a.n = c->g.n;
    a.nb = c->g.ldb;
    a.off = c->g.off.as<int>();
    a.nbr = c->g.nbr.as<int>();
    a.rev = c->g.rev.as<int>();
    a.G = e.G.p;
    a.GR = e.adj_GR.p;
    a.hrev = e.adj_GR.p ? e.adj_HR.as<uint8_t>() : nullptr;
    a.health = e.health.as<uint8_t>();
    a.C11 = e.C11;
    a.C12 = e.C12;
    a.C66 = e.C66;
    a.inv_rho = 1.0 / e.rho;
    a.u = u;
    a.abar = w;
    a.ubar = ubar;
    a.dC = e.adj_dC.as<double>();
    a.step = 1;
    a.scale = scale;
    a.c_r = c_r;
    a.rin = rin;
    a.c_w = c_w;
    a.c_o = c_o;
    a.rout = rout;
    if (e.adj_sg_on) a.SG = e.adj_SG.as<double>();
    const bool aligned = ((reinterpret_cast<uintptr_t>(u) | reinterpret_cast<uintptr_t>(w) |
                           reinterpret_cast<uintptr_t>(rin)) & 15u) == 0;
    if (staged && e.adj_sg_on && adj_sched(c) >= 2 && rin && aligned) {
        a.maxb = epf_adj_tma_maxb(c->g.dim, c->g.max_family);
        a.err = reinterpret_cast<unsigned int *>(e.counters.as<unsigned long long>() + 2);
        if (e.wait_tries >= 0) a.wait_tries = e.wait_tries;
        a.evict_first = e.evict_first ? 1 : 0;
        a.UW = uw;
        const cudaError_t err = launch_epf_adjoint_tma(a, c->g.dim, e.precision == PXB_MIXED, adj_sched(c) - 2,
                                                       c->stream);
        if (err != cudaSuccess) return cuda_fail(err, "staged adjoint step");
        return check_launch(c, "staged adjoint step");
    }
    launch_epf_adjoint(a, c->g.dim, e.precision == PXB_MIXED, epf_grid(c->g.n, c->g.dim, 0), c->stream);
    return check_launch(c, "epf adjoint step");
}

}  // namespace

namespace {

// The adjoint kernel's reverse-bond operators as a bond-ordered copy (GR[c][t] = G[c][rev t]), built once per setup:
// the kernel then streams them instead of gathering six scattered values per bond.  Without room for the copy
// (a memory cap, or a full device) the kernel gathers them.
int ensure_grev(pxb_ctx *c) {
    EpfState &e = c->epf;
    if (e.adj_GR.p || e.adj_GR_none) return PXB_OK;
    PXB_TRY(ensure_rev(c));
    if (dev_alloc(c, e.adj_GR, e.G.bytes) != PXB_OK) {
        e.adj_GR_none = true;
        return PXB_OK;
    }
    PXB_CUDA_TRY(cudaMemsetAsync(e.adj_GR.p, 0, e.adj_GR.bytes, c->stream));
    PXB_CUDA_TRY(launch_reverse_gather(e.G.p, e.adj_GR.p, c->g.rev.as<int>(), c->g.nb, (long long)c->g.ldb, c->g.dim,
                                       e.precision == PXB_MIXED, c->stream));
    return check_launch(c, "reverse gather");
}

}  // namespace

extern "C" int pxb_epf_record_d(pxb_ctx *c, const double *u0_d, const double *v0_d, double dt, int nsteps,
                                int checkpoint_every, double *uN_d, double *uNm1_d) {
    PXB_TRY(need_epf(c, "pxb_epf_record_d"));
    if (!u0_d || !(dt > 0.0) || nsteps < 0)
        return fail(PXB_ERR_INVALID, "pxb_epf_record_d: need u0, dt > 0, nsteps >= 0");
    EpfState &e = c->epf;
    e.rec_steps = -1;
    const size_t nd = (size_t)c->g.n * c->g.dim, bytes = sizeof(double) * nd;
    // every state kept when checkpoint_every <= 0 or covers the run: the reverse sweep then recomputes nothing
    const bool all = checkpoint_every <= 0 || checkpoint_every >= nsteps;
    const int K = all ? std::max(nsteps, 1) : checkpoint_every;
    const int nseg = nsteps > 0 ? (nsteps + K - 1) / K : 0;
    PXB_TRY(dev_alloc(c, e.adj_ckpt, all ? 0 : 2 * bytes * (size_t)std::max(nseg, 1)));
    PXB_TRY(dev_alloc(c, e.adj_seg, bytes * (size_t)K + 64));  // + the staged adjoint's bulk-copy slack
    for (int k = 0; k < 2; ++k) PXB_TRY(dev_alloc(c, e.adj_p[k], bytes + 64));
    PXB_TRY(dev_alloc(c, e.adj_u0, bytes));
    PXB_TRY(dev_alloc(c, e.adj_t, sizeof(double) * (size_t)std::max(nsteps, 1)));
    PXB_TRY(dev_alloc(c, e.adj_umax, sizeof(unsigned long long) * (size_t)std::max(nsteps, 1)));
    // step times t_{n+1}, accumulated as the forward loop does
    std::vector<double> th((size_t)std::max(nsteps, 1));
    double t = 0.0;
    for (int s = 0; s < nsteps; ++s) { t = t + dt; th[(size_t)s] = t; }
    PXB_TRY(h2d(c, e.adj_t.p, th.data(), sizeof(double) * th.size()));
    const double *tdev = e.adj_t.as<double>();
    double *P[2] = {e.adj_p[0].as<double>(), e.adj_p[1].as<double>()};
    double *ck = e.adj_ckpt.as<double>(), *seg = e.adj_seg.as<double>();
    auto d2d = [&](void *dst, const void *src, size_t b) -> int {
        PXB_CUDA_TRY(cudaMemcpyAsync(dst, src, b, cudaMemcpyDeviceToDevice, c->stream));
        return PXB_OK;
    };
    PXB_TRY(d2d(e.adj_u0.p, u0_d, bytes));
    // start: u^{-1} = u0 - dt v0 + dt^2/2 a(u0) with the frozen mask (the START mode of the lane-group kernel)
    {
        EpfArgs a = epf_args(c);
        a.u = u0_d;
        a.u_other = P[1];
        a.v0 = v0_d;
        a.dt = dt;
        a.dt2 = 0.5 * dt * dt;
        a.damage = 0;
        a.sc_bond = nullptr;
        const cudaError_t err = launch_epf(a, c->g.dim, e.precision == PXB_MIXED, EPF_START, 1, c->stream);
        if (err != cudaSuccess) return cuda_fail(err, "recorded start");
        c->launches++;
        PXB_TRY(d2d(P[0], u0_d, bytes));
    }
    // the forward loop, keeping every state u^q (all) or the pair (u^{sK}, u^{sK-1}) at every segment start; the
    // last segment's states are kept as they pass (the reverse sweep starts there, so it is not recomputed)
    int cur = 0;
    const int qlast = (nseg - 1) * K;
    for (int q = 0; q < nsteps; ++q) {
        if (all) {
            PXB_TRY(d2d(seg + (size_t)q * nd, P[cur], bytes));
        } else {
            if (q % K == 0) {
                const size_t s = (size_t)(q / K);
                PXB_TRY(d2d(ck + (2 * s) * nd, P[cur], bytes));
                PXB_TRY(d2d(ck + (2 * s + 1) * nd, P[cur ^ 1], bytes));
            }
            if (q >= qlast) PXB_TRY(d2d(seg + (size_t)(q - qlast) * nd, P[cur], bytes));
        }
        PXB_TRY(adj_step(c, P[cur], P[cur ^ 1], tdev, q, dt));
        cur ^= 1;
    }
    if (uN_d) PXB_TRY(d2d(uN_d, P[cur], bytes));
    if (uNm1_d) PXB_TRY(d2d(uNm1_d, P[cur ^ 1], bytes));
    e.rec_dt = dt;
    e.rec_steps = nsteps;
    e.rec_K = K;
    e.rec_all = all;
    e.rec_seg = all ? -1 : nseg - 1;
    return PXB_OK;
}

extern "C" int pxb_epf_adjoint_recorded_d(pxb_ctx *c, const double *ubar_N_d, const double *ubar_Nm1_d,
                                          double *u0bar_d, double *v0bar_d, double *dC_d) {
    PXB_TRY(need_epf(c, "pxb_epf_adjoint_recorded_d"));
    EpfState &e = c->epf;
    if (e.rec_steps < 0)
        return fail(PXB_ERR_STATE, "pxb_epf_adjoint_recorded_d: no recorded forward loop (pxb_epf_record_d)");
    if (!ubar_N_d || !u0bar_d) return fail(PXB_ERR_INVALID, "pxb_epf_adjoint_recorded_d: need dJ/du^N and dJ/du0");
    PXB_TRY(ensure_grev(c));
    struct SgOff {  // the reverse-only kernel is used inside this sweep only
        EpfState &e;
        ~SgOff() { e.adj_sg_on = false; }
    } sg_off{e};
    e.adj_sg_on = false;
    if (e.adj_GR.p) {  // the frozen mask in reverse-bond order, for this sweep
        PXB_TRY(dev_alloc(c, e.adj_HR, (size_t)std::max(1LL, c->g.ldb)));  // to ldb: the staged kernel's copies
        PXB_CUDA_TRY(cudaMemsetAsync(e.adj_HR.p, 0, e.adj_HR.bytes, c->stream));
        PXB_CUDA_TRY(launch_reverse_health(e.health.as<uint8_t>(), c->g.rev.as<int>(), e.adj_HR.as<uint8_t>(), c->g.nb,
                                           c->stream));
        PXB_TRY(check_launch(c, "reverse health"));
        // the own bonds' operator sums under the frozen mask: with every bond's reverse present, the reverse-only
        // kernel then reads one operator stream per step instead of two (the missing count uses counter slot 5)
        const int nc = c->g.dim == 3 ? 6 : 3;
        if (adj_sched(c) != 0 &&
            dev_alloc(c, e.adj_SG, sizeof(double) * nc * (size_t)std::max(1, c->g.n)) == PXB_OK) {
            unsigned int *miss = reinterpret_cast<unsigned int *>(e.counters.as<unsigned long long>() + 5);
            PXB_CUDA_TRY(cudaMemsetAsync(miss, 0, sizeof(unsigned int), c->stream));
            PXB_CUDA_TRY(launch_own_sums(c->g.n, c->g.dim, e.precision == PXB_MIXED, c->g.off.as<int>(),
                                         c->g.rev.as<int>(), e.health.as<uint8_t>(), e.G.p, (long long)c->g.ldb,
                                         e.adj_SG.as<double>(), miss, c->stream));
            PXB_TRY(check_launch(c, "own sums"));
            unsigned int nmiss = 1;
            PXB_TRY(d2h(c, &nmiss, miss, sizeof(nmiss)));
            PXB_CUDA_TRY(cudaStreamSynchronize(c->stream));
            e.adj_sg_on = nmiss == 0;
            // the staged kernel's interleaved (u, w) gather rows (without room for them it gathers u and w apart)
            if (!e.adj_sg_on || adj_sched(c) < 2 ||
                dev_alloc(c, e.adj_UW, sizeof(double) * 2 * c->g.dim * (size_t)std::max(1, c->g.n)) != PXB_OK)
                e.adj_UW.release();
        }
    }
    const size_t nd = (size_t)c->g.n * c->g.dim, bytes = sizeof(double) * nd;
    const int nsteps = e.rec_steps, K = e.rec_K;
    const double dt = e.rec_dt, dt2 = dt * dt;
    const int nseg = nsteps > 0 ? (nsteps + K - 1) / K : 0;
    PXB_TRY(dev_alloc(c, e.adj_A, bytes));
    PXB_TRY(dev_alloc(c, e.adj_R, bytes + 64));  // + the staged adjoint's bulk-copy slack
    PXB_TRY(dev_alloc(c, e.adj_W, bytes + 64));
    if (adj_sched(c) >= 2)  // the staged adjoint's wait-failure word
        PXB_CUDA_TRY(cudaMemsetAsync(e.counters.as<unsigned long long>() + 2, 0, sizeof(unsigned int), c->stream));
    PXB_TRY(dev_alloc(c, e.adj_dC, 4 * sizeof(double)));
    PXB_CUDA_TRY(cudaMemsetAsync(e.adj_dC.p, 0, 4 * sizeof(double), c->stream));
    auto d2d = [&](void *dst, const void *src, size_t b) -> int {
        PXB_CUDA_TRY(cudaMemcpyAsync(dst, src, b, cudaMemcpyDeviceToDevice, c->stream));
        return PXB_OK;
    };
    const double *tdev = e.adj_t.as<double>();
    double *P[2] = {e.adj_p[0].as<double>(), e.adj_p[1].as<double>()};
    double *ck = e.adj_ckpt.as<double>(), *seg = e.adj_seg.as<double>();
    double *A = e.adj_A.as<double>(), *Rv = e.adj_R.as<double>(), *W = e.adj_W.as<double>();
    PXB_TRY(d2d(A, ubar_N_d, bytes));
    if (ubar_Nm1_d) PXB_TRY(d2d(Rv, ubar_Nm1_d, bytes));
    else PXB_CUDA_TRY(cudaMemsetAsync(Rv, 0, bytes, c->stream));
    EpfArgs bc = epf_args(c);
    fill_bc(c, bc);
    for (int s = nseg - 1; s >= 0; --s) {
        const int q0 = s * K, q1 = std::min(nsteps, (s + 1) * K);
        // recompute the segment's states u^{q0} .. u^{q1-1} from its checkpoint, unless seg still holds them (the
        // last segment, kept by the forward loop, on the first sweep over a recording)
        if (!e.rec_all && e.rec_seg != s) {
            e.rec_seg = -1;
            PXB_TRY(d2d(P[0], ck + (size_t)(2 * s) * nd, bytes));
            PXB_TRY(d2d(P[1], ck + (size_t)(2 * s + 1) * nd, bytes));
            int cur = 0;
            for (int q = q0; q < q1; ++q) {
                PXB_TRY(d2d(seg + (size_t)(q - q0) * nd, P[cur], bytes));
                if (q + 1 < q1) {
                    PXB_TRY(adj_step(c, P[cur], P[cur ^ 1], tdev, q, dt));
                    cur ^= 1;
                }
            }
            e.rec_seg = s;
        }
        for (int q = q1 - 1; q >= q0; --q) {
            const double *uq = seg + (size_t)(q - q0) * nd;
            double *uw = e.adj_UW.p ? e.adj_UW.as<double>() : nullptr;
            const cudaError_t err = launch_bc_transpose(bc, c->g.n, c->g.dim, A, W, c->stream, uq, uw);
            if (err != cudaSuccess) return cuda_fail(err, "bc transpose");
            c->launches++;
            PXB_TRY(adj_kernel(c, uq, W, dt2, 1.0, Rv, 2.0, A, -1.0, Rv, true, uw));
        }
    }
    if (adj_sched(c) >= 2) {  // a staged wait that ran out fails the sweep
        unsigned int werr = 0;
        PXB_TRY(d2h(c, &werr, e.counters.as<unsigned long long>() + 2, sizeof(unsigned int)));
        PXB_TRY(sync(c));
        if (werr) return wait_failure(c, werr, "staged adjoint sweep");
    }
    // the start: dJ/du0 = A + R + (da/du)^T (dt^2/2 R), dJ/dv0 = -dt R
    PXB_TRY(adj_kernel(c, e.adj_u0.as<double>(), Rv, 0.5 * dt2, 1.0, A, 1.0, u0bar_d, -dt, v0bar_d));
    if (dC_d) PXB_TRY(d2d(dC_d, e.adj_dC.p, 3 * sizeof(double)));
    return PXB_OK;
}

extern "C" int pxb_epf_adjoint_d(pxb_ctx *c, const double *u0_d, const double *v0_d, double dt, int nsteps,
                                 int checkpoint_every, const double *ubar_N_d, const double *ubar_Nm1_d,
                                 double *u0bar_d, double *v0bar_d, double *dC_d) {
    PXB_TRY(need_epf(c, "pxb_epf_adjoint_d"));
    if (!u0_d || !ubar_N_d || !u0bar_d || !(dt > 0.0) || nsteps < 0)
        return fail(PXB_ERR_INVALID, "pxb_epf_adjoint_d: need u0, dJ/du^N, the dJ/du0 output, dt > 0, nsteps >= 0");
    PXB_TRY(pxb_epf_record_d(c, u0_d, v0_d, dt, nsteps, checkpoint_every, nullptr, nullptr));
    return pxb_epf_adjoint_recorded_d(c, ubar_N_d, ubar_Nm1_d, u0bar_d, v0bar_d, dC_d);
}

extern "C" int pxb_epf_force_adjoint(pxb_ctx *c, const double *u, const double *abar, double *ubar, double *dC) {
    PXB_TRY(need_epf(c, "pxb_epf_force_adjoint"));
    if (!u || !abar || !ubar) return fail(PXB_ERR_INVALID, "pxb_epf_force_adjoint: NULL buffer");
    const size_t nd = (size_t)c->g.n * c->g.dim;
    void *tmp = nullptr;
    PXB_TRY(scratch(c, sizeof(double) * (3 * nd + 4), &tmp));
    double *du = static_cast<double *>(tmp), *da = du + nd, *dub = da + nd, *ddc = dub + nd;
    PXB_TRY(h2d(c, du, u, sizeof(double) * nd));
    PXB_TRY(h2d(c, da, abar, sizeof(double) * nd));
    PXB_TRY(pxb_epf_force_adjoint_d(c, du, da, dub, ddc));
    PXB_TRY(d2h(c, ubar, dub, sizeof(double) * nd));
    double hdc[3];
    PXB_TRY(d2h(c, hdc, ddc, sizeof(double) * 3));
    PXB_TRY(sync(c));
    if (dC) std::copy(hdc, hdc + 3, dC);
    return PXB_OK;
}

// ============================================================================================== CSR assembly
namespace pxb {
// the slot map, diagonal slots, exact-pattern flags and value buffers of the pattern in c->csr (rowptr, cols, ndof,
// nnz set on the device)
int csr_finish(pxb_ctx *c, const char *who) {
    CsrState &k = c->csr;
    const int ndof = k.ndof;
    const size_t rows = (size_t)c->g.n * ndof;
    PXB_TRY(dev_alloc(c, k.slot, sizeof(int) * (size_t)std::max(1LL, c->g.nb) * ndof * ndof));
    PXB_TRY(dev_alloc(c, k.diag, sizeof(int) * (size_t)c->g.n * ndof * ndof));
    PXB_TRY(dev_alloc(c, k.extra, sizeof(int) * (size_t)c->g.n * ndof * ndof));
    void *tmp = nullptr;
    PXB_TRY(scratch(c, 8, &tmp));
    PXB_CUDA_TRY(cudaMemsetAsync(tmp, 0, 8, c->stream));
    CsrMapArgs a;
    a.n = c->g.n;
    a.ndof = ndof;
    a.off = c->g.off.as<int>();
    a.nbr = c->g.nbr.as<int>();
    a.rowptr = k.rowptr.as<int>();
    a.cols = k.cols.as<int>();
    a.slot = k.slot.as<int>();
    a.diag = k.diag.as<int>();
    a.missing = static_cast<int *>(tmp);
    a.inexact = static_cast<int *>(tmp) + 1;
    a.mirror = c->g.mirror.p ? c->g.mirror.as<int>() : nullptr;
    a.extra = k.extra.as<int>();
    launch_csr_map(a, c->stream);
    PXB_TRY(check_launch(c, "csr_map"));
    int flags[2] = {0, 0};
    PXB_TRY(d2h(c, flags, tmp, 8));
    PXB_TRY(sync(c));
    const int missing = flags[0];
    k.exact = flags[1] == 0;
    if (missing) return fail(PXB_ERR_INVALID, std::string(who) + ": pattern lacks " + std::to_string(missing) +
                                                  " entries required by the families");
    PXB_TRY(dev_alloc(c, k.kvals, sizeof(double) * (size_t)k.nnz));
    PXB_TRY(dev_alloc(c, k.rhs, sizeof(double) * rows));
    PXB_TRY(dev_alloc(c, k.u, sizeof(double) * rows));
    PXB_TRY(dev_alloc(c, k.uold, sizeof(double) * rows));
    k.ready = true;
    return PXB_OK;
}
}  // namespace pxb

extern "C" int pxb_csr_set_pattern(pxb_ctx *c, int ndof, const int *rowptr, const int *cols, long long nnz) {
    PXB_TRY(need_geometry(c, "pxb_csr_set_pattern"));
    if (ndof < 1 || ndof > 5 || !rowptr || !cols || nnz <= 0) return fail(PXB_ERR_INVALID, "pxb_csr_set_pattern: bad arguments");
    if (rowptr[(size_t)c->g.n * ndof] != nnz) return fail(PXB_ERR_INVALID, "pxb_csr_set_pattern: rowptr[rows] != nnz");
    CsrState &k = c->csr;
    k = CsrState{};
    k.ndof = ndof;
    k.nnz = nnz;
    const size_t rows = (size_t)c->g.n * ndof;
    PXB_TRY(dev_upload(c, k.rowptr, rowptr, sizeof(int) * (rows + 1)));
    PXB_TRY(dev_upload(c, k.cols, cols, sizeof(int) * (size_t)nnz));
    if (ndof == 2 && block_view(c->g.n, rowptr, cols, k.h_bptr, k.h_bcol)) {
        PXB_TRY(dev_upload(c, k.bptr, k.h_bptr.data(), sizeof(int) * k.h_bptr.size()));
        PXB_TRY(dev_upload(c, k.bcol, k.h_bcol.data(), sizeof(int) * std::max<size_t>(1, k.h_bcol.size())));
        k.blocked2 = true;
    }
    return csr_finish(c, "pxb_csr_set_pattern");
}

extern "C" int pxb_csr_build_pattern(pxb_ctx *c, int ndof, long long *nnz) {
    PXB_TRY(need_geometry(c, "pxb_csr_build_pattern"));
    if (ndof < 1 || ndof > 5) return fail(PXB_ERR_INVALID, "pxb_csr_build_pattern: ndof must be 1..5");
    const int n = c->g.n;
    if (n < 1) return fail(PXB_ERR_INVALID, "pxb_csr_build_pattern: no nodes");
    CsrState &k = c->csr;
    k = CsrState{};
    k.ndof = ndof;
    DevBuf count, first, bsum, small;
    PXB_TRY(dev_alloc(c, count, sizeof(int) * (size_t)n));
    PXB_TRY(dev_alloc(c, first, sizeof(long long) * ((size_t)n + 1)));
    PXB_TRY(dev_alloc(c, bsum, sizeof(long long) * (size_t)pattern_scan_blocks(n)));
    PXB_TRY(dev_alloc(c, small, 16));
    PXB_CUDA_TRY(cudaMemsetAsync(small.p, 0, 16, c->stream));
    PatternArgs a;
    a.n = n;
    a.ndof = ndof;
    a.off = c->g.off.as<int>();
    a.nbr = c->g.nbr.as<int>();
    a.mirror = c->g.mirror.p ? c->g.mirror.as<int>() : nullptr;
    a.count = count.as<int>();
    a.first = first.as<long long>();
    a.overflow = reinterpret_cast<int *>(small.as<char>() + 8);
    PXB_CUDA_TRY(launch_pattern_count(a, bsum.as<long long>(), small.as<long long>(), c->stream));
    c->launches += 4;
    long long h[2] = {0, 0};
    PXB_TRY(d2h(c, h, small.p, 16));
    PXB_TRY(sync(c));
    const long long blocks = h[0];
    const int overflow = static_cast<int>(h[1] & 0xffffffffLL);
    if (overflow)
        return fail(PXB_ERR_UNSUPPORTED, "pxb_csr_build_pattern: " + std::to_string(overflow) +
                                             " nodes have more than 256 column nodes (use pxb_csr_pattern)");
    const long long total = blocks * ndof * ndof;
    if (total > std::numeric_limits<int>::max())
        return fail(PXB_ERR_INVALID, "pxb_csr_build_pattern: nnz exceeds 2^31-1");
    k.nnz = total;
    PXB_TRY(dev_alloc(c, k.rowptr, sizeof(int) * ((size_t)n * ndof + 1)));
    PXB_TRY(dev_alloc(c, k.cols, sizeof(int) * (size_t)std::max(1LL, total)));
    if (ndof == 2) {
        PXB_TRY(dev_alloc(c, k.bptr, sizeof(int) * ((size_t)n + 1)));
        PXB_TRY(dev_alloc(c, k.bcol, sizeof(int) * (size_t)std::max(1LL, blocks)));
        a.bptr = k.bptr.as<int>();
        a.bcol = k.bcol.as<int>();
        k.blocked2 = true;
    }
    a.rowptr = k.rowptr.as<int>();
    a.cols = k.cols.as<int>();
    PXB_CUDA_TRY(launch_pattern_fill(a, c->stream));
    c->launches++;
    PXB_TRY(csr_finish(c, "pxb_csr_build_pattern"));
    if (nnz) *nnz = total;
    return PXB_OK;
}

extern "C" int pxb_csr_get_pattern(pxb_ctx *c, int *rowptr, int *cols) {
    if (!c || !c->csr.ready) return fail(PXB_ERR_STATE, "pxb_csr_get_pattern: no pattern set");
    const CsrState &k = c->csr;
    if (rowptr) PXB_TRY(d2h(c, rowptr, k.rowptr.p, sizeof(int) * ((size_t)c->g.n * k.ndof + 1)));
    if (cols) PXB_TRY(d2h(c, cols, k.cols.p, sizeof(int) * (size_t)k.nnz));
    return sync(c);
}

extern "C" int pxb_assemble_scalar_d(pxb_ctx *c, int type, double coef, double f, const double *f_node_d, double dt,
                                     const double *u_d, const double *uold_d, double *kvals_d, double *rhs_d) {
    PXB_TRY(need_geometry(c, "pxb_assemble_scalar"));
    CsrState &k = c->csr;
    if (!k.ready || k.ndof != 1) return fail(PXB_ERR_STATE, "pxb_assemble_scalar: set a 1-dof pattern first");
    if (!c->ops.ready || c->ops.order < 2) return fail(PXB_ERR_STATE, "pxb_assemble_scalar: needs a g-build of order >= 2");
    if (type != 0 && type != 1) return fail(PXB_ERR_INVALID, "pxb_assemble_scalar: type must be 0 (Poisson) or 1 (diffusion)");
    if (type == 1 && (!(dt > 0.0) || !uold_d)) return fail(PXB_ERR_INVALID, "pxb_assemble_scalar: diffusion is transient-only (dt>0, uold)");
    if (!u_d || !kvals_d || !rhs_d) return fail(PXB_ERR_INVALID, "pxb_assemble_scalar: NULL buffer");
    const auto &q = c->ops.pqr;
    auto slot = [&](int p, int qq, int r) {
        for (size_t s = 0; s < q.size() / 3; ++s)
            if (q[3 * s] == p && q[3 * s + 1] == qq && q[3 * s + 2] == r) return (int)s;
        return -1;
    };
    ScalarAsmArgs a;
    a.n = c->g.n;
    a.dim = c->g.dim;
    a.nop = c->ops.nop;
    a.type = type;
    a.mixed = c->ops.precision == PXB_MIXED;
    a.s_xx = slot(2, 0, 0);
    a.s_yy = slot(0, 2, 0);
    a.s_zz = c->g.dim == 3 ? slot(0, 0, 2) : -1;
    a.coef = coef;
    a.f = f;
    a.dt = dt;
    a.f_node = f_node_d;
    a.off = c->g.off.as<int>();
    a.nbr = c->g.nbr.as<int>();
    a.rowptr = k.rowptr.as<int>();
    a.slot = k.slot.as<int>();
    a.diag = k.diag.as<int>();
    a.ops = c->ops.ops.p;
    a.degenerate = c->ops.degenerate.as<uint8_t>();
    a.u = u_d;
    a.uold = uold_d;
    a.kvals = kvals_d;
    a.rhs = rhs_d;
    launch_assemble_scalar(a, c->stream);
    return check_launch(c, "assemble_scalar");
}

extern "C" int pxb_assemble_scalar(pxb_ctx *c, int type, double coef, double f, const double *f_node, double dt,
                                   const double *u, const double *uold, double *kvals, double *rhs) {
    PXB_TRY(need_geometry(c, "pxb_assemble_scalar"));
    CsrState &k = c->csr;
    if (!k.ready) return fail(PXB_ERR_STATE, "pxb_assemble_scalar: set a pattern first");
    if (!u || !kvals || !rhs) return fail(PXB_ERR_INVALID, "pxb_assemble_scalar: NULL buffer");
    const size_t n = (size_t)c->g.n;
    PXB_TRY(h2d(c, k.u.p, u, sizeof(double) * n));
    if (uold) PXB_TRY(h2d(c, k.uold.p, uold, sizeof(double) * n));
    if (f_node) {
        PXB_TRY(dev_alloc(c, k.fnode, sizeof(double) * n));
        PXB_TRY(h2d(c, k.fnode.p, f_node, sizeof(double) * n));
    }
    PXB_TRY(pxb_assemble_scalar_d(c, type, coef, f, f_node ? k.fnode.as<double>() : nullptr, dt, k.u.as<double>(),
                                  uold ? k.uold.as<double>() : nullptr, k.kvals.as<double>(), k.rhs.as<double>()));
    PXB_TRY(d2h(c, kvals, k.kvals.p, sizeof(double) * (size_t)k.nnz));
    PXB_TRY(d2h(c, rhs, k.rhs.p, sizeof(double) * n));
    return sync(c);
}

// the CH assembly's bond-order streams of the fixed geometry (vol_j lap[rev t] and the ghost / reverse flags)
static int ch_bond_streams(pxb_ctx *c) {
    ChState &h = c->ch;
    const size_t nb = (size_t)std::max(1LL, c->g.nb);
    PXB_TRY(dev_alloc(c, h.lrv, sizeof(double) * nb));
    PXB_TRY(dev_alloc(c, h.bfl, nb));
    PXB_CUDA_TRY(launch_ch_bond_streams(c->g.n, c->g.off.as<int>(), c->g.nbr.as<int>(), h.rev.as<int>(),
                                        h.lap.as<double>(), c->g.vol.as<double>(),
                                        h.ghost.p ? h.ghost.as<char>() : nullptr, h.lrv.as<double>(),
                                        h.bfl.as<uint8_t>(), c->stream));
    return check_launch(c, "ch bond streams");
}

extern "C" int pxb_ch_set_geometry(pxb_ctx *c, const int *rev, const double *lapbond, const char *isghost) {
    PXB_TRY(need_geometry(c, "pxb_ch_set_geometry"));
    if (!rev || !lapbond) return fail(PXB_ERR_INVALID, "pxb_ch_set_geometry: NULL array");
    ChState &h = c->ch;
    const size_t nb = (size_t)std::max(1LL, c->g.nb);
    PXB_TRY(dev_upload(c, h.rev, rev, sizeof(int) * (size_t)c->g.nb));
    if (c->g.nb == 0) PXB_TRY(dev_alloc(c, h.rev, sizeof(int) * nb));
    PXB_TRY(dev_upload(c, h.lap, lapbond, sizeof(double) * (size_t)c->g.nb));
    if (isghost) PXB_TRY(dev_upload(c, h.ghost, isghost, (size_t)c->g.n));
    PXB_TRY(ch_bond_streams(c));
    PXB_TRY(sync(c));
    h.ready = true;
    return PXB_OK;
}

extern "C" int pxb_ch_build_geometry(pxb_ctx *c) {
    PXB_TRY(need_geometry(c, "pxb_ch_build_geometry"));
    const OpsCache &o = c->ops;
    if (!o.ready || o.order != 2) return fail(PXB_ERR_STATE, "pxb_ch_build_geometry: needs an order-2 operator cache (pxb_gbuild)");
    const int dim = c->g.dim;
    auto slot = [&](int p, int q, int r) {
        for (int k = 0; k < o.nop; ++k)
            if (o.pqr[3 * k] == p && o.pqr[3 * k + 1] == q && o.pqr[3 * k + 2] == r) return k;
        return -1;
    };
    const int sxx = slot(2, 0, 0), syy = slot(0, 2, 0), szz = dim == 3 ? slot(0, 0, 2) : 0;
    ChState &h = c->ch;
    PXB_TRY(ensure_rev(c));
    const size_t nb = (size_t)std::max(1LL, c->g.nb);
    PXB_TRY(dev_alloc(c, h.rev, sizeof(int) * nb));
    PXB_CUDA_TRY(cudaMemcpyAsync(h.rev.p, c->g.rev.p, sizeof(int) * (size_t)c->g.nb, cudaMemcpyDeviceToDevice, c->stream));
    PXB_TRY(dev_alloc(c, h.lap, sizeof(double) * nb));
    PXB_TRY(dev_alloc(c, h.ghost, (size_t)c->g.n));
    PXB_CUDA_TRY(launch_ch_geometry(c->g.n, dim, c->g.off.as<int>(), c->g.nbr.as<int>(), c->g.pos.p,
                                    c->g.mirror.p ? c->g.mirror.as<int>() : nullptr, o.ops.p, o.precision == PXB_MIXED,
                                    o.nop, sxx, syy, szz, h.lap.as<double>(), h.ghost.as<char>(), c->stream));
    PXB_TRY(check_launch(c, "ch geometry"));
    PXB_TRY(ch_bond_streams(c));
    PXB_TRY(sync(c));
    h.ready = true;
    return PXB_OK;
}

extern "C" int pxb_ch_get_geometry(pxb_ctx *c, int *rev, double *lapbond, char *isghost) {
    PXB_TRY(need_geometry(c, "pxb_ch_get_geometry"));
    if (!c->ch.ready) return fail(PXB_ERR_STATE, "pxb_ch_get_geometry: no CH geometry");
    const size_t nb = (size_t)c->g.nb;
    if (rev) PXB_TRY(d2h(c, rev, c->ch.rev.p, sizeof(int) * nb));
    if (lapbond) PXB_TRY(d2h(c, lapbond, c->ch.lap.p, sizeof(double) * nb));
    if (isghost && c->ch.ghost.p) PXB_TRY(d2h(c, isghost, c->ch.ghost.p, (size_t)c->g.n));
    return sync(c);
}

extern "C" int pxb_ch_mobility_d(pxb_ctx *c, double M0, const double *u_d, double *mnode_d) {
    PXB_TRY(need_geometry(c, "pxb_ch_mobility"));
    if (!u_d || !mnode_d) return fail(PXB_ERR_INVALID, "pxb_ch_mobility: NULL buffer");
    PXB_CUDA_TRY(launch_ch_mobility(c->g.n, M0, u_d, mnode_d, c->stream));
    return check_launch(c, "ch mobility");
}

static int ch_args(pxb_ctx *c, double kappa, double chi, double dt, const double *mnode_d, const double *u_d,
                   const double *uold_d, double *kvals_d, double *rhs_d, ChAsmArgs &a, const char *who) {
    PXB_TRY(need_geometry(c, who));
    CsrState &k = c->csr;
    if (!k.ready || k.ndof != 2) return fail(PXB_ERR_STATE, std::string(who) + ": set a 2-dof pattern first");
    if (!c->ch.ready) return fail(PXB_ERR_STATE, std::string(who) + ": call pxb_ch_set_geometry or pxb_ch_build_geometry first");
    if (!(dt > 0.0)) return fail(PXB_ERR_INVALID, std::string(who) + ": dt must be > 0 (transient-only element)");
    a.n = c->g.n;
    a.kappa = kappa;
    a.chi = chi;
    a.dt = dt;
    a.off = c->g.off.as<int>();
    a.nbr = c->g.nbr.as<int>();
    a.rev = c->ch.rev.as<int>();
    a.lap = c->ch.lap.as<double>();
    a.vol = c->g.vol.as<double>();
    a.mnode = mnode_d;
    a.ghost = c->ch.ghost.p ? c->ch.ghost.as<char>() : nullptr;
    a.rowptr = k.rowptr.as<int>();
    a.slot = k.slot.as<int>();
    a.diag = k.diag.as<int>();
    a.extra = k.exact ? k.extra.as<int>() : nullptr;
    a.u = u_d;
    a.uold = uold_d;
    a.kvals = kvals_d;
    a.rhs = rhs_d;
    if (c->ch.lrv.p && c->ch.bfl.p) {
        a.lrv = c->ch.lrv.as<double>();
        a.bfl = c->ch.bfl.as<uint8_t>();
    }
    return PXB_OK;
}

extern "C" int pxb_assemble_ch_d(pxb_ctx *c, double kappa, double chi, double dt, const double *mnode_d,
                                 const double *u_d, const double *uold_d, double *kvals_d, double *rhs_d) {
    if (!mnode_d || !u_d || !uold_d || !kvals_d || !rhs_d) return fail(PXB_ERR_INVALID, "pxb_assemble_ch: NULL buffer");
    ChAsmArgs a;
    PXB_TRY(ch_args(c, kappa, chi, dt, mnode_d, u_d, uold_d, kvals_d, rhs_d, a, "pxb_assemble_ch"));
    launch_assemble_ch(a, c->stream);
    return check_launch(c, "assemble_ch");
}

extern "C" int pxb_assemble_stress_ch_d(pxb_ctx *c, const pxb_stress_ch_params *p, const double *mnode_d,
                                        const double *health_d, const double *vel_d, const double *u_d,
                                        const double *uold_d, double *kvals_d, double *rhs_d) {
    PXB_TRY(need_geometry(c, "pxb_assemble_stress_ch"));
    const int dim = c->g.dim, nd = dim + 2;
    CsrState &k = c->csr;
    if (!k.ready || k.ndof != nd) return fail(PXB_ERR_STATE, "pxb_assemble_stress_ch: set a pattern with ndof = dim + 2 first");
    if (!c->ch.ready) return fail(PXB_ERR_STATE, "pxb_assemble_stress_ch: needs the CH geometry (pxb_ch_set_geometry)");
    const OpsCache &o = c->ops;
    if (!o.ready || o.order != 2 || o.precision != PXB_FP64)
        return fail(PXB_ERR_STATE, "pxb_assemble_stress_ch: needs an FP64 order-2 g-build (pxb_gbuild)");
    if (!p || !(p->dt > 0.0) || !mnode_d || !u_d || !kvals_d || !rhs_d)
        return fail(PXB_ERR_INVALID, "pxb_assemble_stress_ch: bad arguments");
    auto slot = [&](int pp, int q, int r) {
        for (int s = 0; s < o.nop; ++s)
            if (o.pqr[3 * s] == pp && o.pqr[3 * s + 1] == q && o.pqr[3 * s + 2] == r) return s;
        return -1;
    };
    StressChAsmArgs a;
    a.n = c->g.n;
    a.dim = dim;
    a.nop = o.nop;
    const int mi[9][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}, {2, 0, 0}, {1, 1, 0}, {0, 2, 0}, {1, 0, 1}, {0, 1, 1}, {0, 0, 2}};
    for (int q = 0; q < 9; ++q) a.sl[q] = (dim == 3 || mi[q][2] == 0) ? slot(mi[q][0], mi[q][1], mi[q][2]) : -1;
    a.C11 = p->C11;
    a.C12 = p->C12;
    a.C66 = p->C66;
    a.A = p->A;
    a.Kh = p->Kh;
    a.Ch = p->Ch;
    a.Omega = p->Omega;
    a.cref = p->cref;
    a.chi = p->chi;
    a.kappa = p->kappa;
    a.dt = p->dt;
    a.kres = p->kres;
    a.rho = p->rho;
    a.off = c->g.off.as<int>();
    a.nbr = c->g.nbr.as<int>();
    a.rev = c->ch.rev.as<int>();
    a.lap = c->ch.lap.as<double>();
    a.vol = c->g.vol.as<double>();
    a.mnode = mnode_d;
    a.ghost = c->ch.ghost.p ? c->ch.ghost.as<char>() : nullptr;
    a.ops = o.ops.as<double>();
    a.degenerate = o.degenerate.as<uint8_t>();
    a.health = health_d;
    a.vel = vel_d;
    a.rowptr = k.rowptr.as<int>();
    a.slot = k.slot.as<int>();
    a.diag = k.diag.as<int>();
    a.u = u_d;
    a.uold = uold_d;
    a.kvals = kvals_d;
    a.rhs = rhs_d;
    PXB_CUDA_TRY(launch_assemble_stress_ch(a, c->stream));
    return check_launch(c, "assemble_stress_ch");
}

extern "C" int pxb_assemble_stress_ch(pxb_ctx *c, const pxb_stress_ch_params *p, const double *mnode,
                                      const double *health, const double *vel, const double *u, const double *uold,
                                      double *kvals, double *rhs) {
    PXB_TRY(need_geometry(c, "pxb_assemble_stress_ch"));
    CsrState &k = c->csr;
    const int dim = c->g.dim, nd = dim + 2;
    if (!k.ready || k.ndof != nd) return fail(PXB_ERR_STATE, "pxb_assemble_stress_ch: set a pattern with ndof = dim + 2 first");
    if (!mnode || !u || !kvals || !rhs) return fail(PXB_ERR_INVALID, "pxb_assemble_stress_ch: NULL buffer");
    const size_t n = (size_t)c->g.n, nb = (size_t)c->g.nb;
    void *tmp = nullptr;
    PXB_TRY(scratch(c, sizeof(double) * (n + (health ? nb : 0) + (vel ? n * dim : 0) + 1), &tmp));
    double *dm = static_cast<double *>(tmp), *dh = dm + n, *dv = dh + (health ? nb : 0);
    PXB_TRY(h2d(c, dm, mnode, sizeof(double) * n));
    if (health) PXB_TRY(h2d(c, dh, health, sizeof(double) * nb));
    if (vel) PXB_TRY(h2d(c, dv, vel, sizeof(double) * n * dim));
    PXB_TRY(h2d(c, k.u.p, u, sizeof(double) * n * nd));
    if (uold) PXB_TRY(h2d(c, k.uold.p, uold, sizeof(double) * n * nd));
    PXB_TRY(pxb_assemble_stress_ch_d(c, p, dm, health ? dh : nullptr, vel ? dv : nullptr, k.u.as<double>(),
                                     uold ? k.uold.as<double>() : nullptr, k.kvals.as<double>(), k.rhs.as<double>()));
    PXB_TRY(d2h(c, kvals, k.kvals.p, sizeof(double) * (size_t)k.nnz));
    PXB_TRY(d2h(c, rhs, k.rhs.p, sizeof(double) * n * nd));
    return sync(c);
}

extern "C" int pxb_assemble_cached_d(pxb_ctx *c, const pxb_cached_params *p, const double *nodecache_d, int ncache,
                                     const double *bondcache_d, int nbcache, const double *u_d, const double *uold_d,
                                     double *kvals_d, double *rhs_d) {
    PXB_TRY(need_geometry(c, "pxb_assemble_cached"));
    const int dim = c->g.dim;
    CsrState &k = c->csr;
    if (!k.ready || k.ndof != dim) return fail(PXB_ERR_STATE, "pxb_assemble_cached: set a pattern with ndof = dim first");
    const OpsCache &o = c->ops;
    if (!o.ready || o.order != 2 || o.precision != PXB_FP64)
        return fail(PXB_ERR_STATE, "pxb_assemble_cached: needs an FP64 order-2 g-build (pxb_gbuild)");
    if (!p || !(p->dt > 0.0) || !u_d || !kvals_d || !rhs_d || (nodecache_d && ncache < dim) ||
        (bondcache_d && nbcache < 1))
        return fail(PXB_ERR_INVALID, "pxb_assemble_cached: bad arguments");
    auto slot = [&](int pp, int q, int r) {
        for (int s = 0; s < o.nop; ++s)
            if (o.pqr[3 * s] == pp && o.pqr[3 * s + 1] == q && o.pqr[3 * s + 2] == r) return s;
        return -1;
    };
    CachedAsmArgs a;
    a.n = c->g.n;
    a.dim = dim;
    a.nop = o.nop;
    a.ncache = ncache;
    a.nbcache = nbcache;
    a.sl[0] = slot(2, 0, 0);
    a.sl[1] = slot(1, 1, 0);
    a.sl[2] = slot(0, 2, 0);
    if (dim == 3) {
        a.sl[3] = slot(1, 0, 1);
        a.sl[4] = slot(0, 1, 1);
        a.sl[5] = slot(0, 0, 2);
    }
    a.C11 = p->C11;
    a.C12 = p->C12;
    a.C66 = p->C66;
    a.rho = p->rho;
    a.dt = p->dt;
    for (int d = 0; d < 3; ++d) a.b[d] = p->b[d];
    a.off = c->g.off.as<int>();
    a.nbr = c->g.nbr.as<int>();
    a.pos = c->g.pos.p;
    a.ops = o.ops.as<double>();
    a.degenerate = o.degenerate.as<uint8_t>();
    a.nodecache = nodecache_d;
    a.bondcache = bondcache_d;
    a.rowptr = k.rowptr.as<int>();
    a.slot = k.slot.as<int>();
    a.diag = k.diag.as<int>();
    a.u = u_d;
    a.uold = uold_d;
    a.kvals = kvals_d;
    a.rhs = rhs_d;
    PXB_CUDA_TRY(launch_assemble_cached(a, c->stream));
    return check_launch(c, "assemble_cached");
}

extern "C" int pxb_assemble_cached(pxb_ctx *c, const pxb_cached_params *p, const double *nodecache, int ncache,
                                   const double *bondcache, int nbcache, const double *u, const double *uold,
                                   double *kvals, double *rhs) {
    PXB_TRY(need_geometry(c, "pxb_assemble_cached"));
    CsrState &k = c->csr;
    const int dim = c->g.dim;
    if (!k.ready || k.ndof != dim) return fail(PXB_ERR_STATE, "pxb_assemble_cached: set a pattern with ndof = dim first");
    if (!u || !kvals || !rhs || (nodecache && ncache < dim) || (bondcache && nbcache < 1))
        return fail(PXB_ERR_INVALID, "pxb_assemble_cached: bad arguments");
    const size_t n = (size_t)c->g.n, nb = (size_t)c->g.nb;
    const size_t nn = nodecache ? n * (size_t)ncache : 0, nbb = bondcache ? nb * (size_t)nbcache : 0;
    void *tmp = nullptr;
    PXB_TRY(scratch(c, sizeof(double) * (nn + nbb + 1), &tmp));
    double *dn = static_cast<double *>(tmp), *db = dn + nn;
    if (nodecache) PXB_TRY(h2d(c, dn, nodecache, sizeof(double) * nn));
    if (bondcache) PXB_TRY(h2d(c, db, bondcache, sizeof(double) * nbb));
    PXB_TRY(h2d(c, k.u.p, u, sizeof(double) * n * dim));
    if (uold) PXB_TRY(h2d(c, k.uold.p, uold, sizeof(double) * n * dim));
    PXB_TRY(pxb_assemble_cached_d(c, p, nodecache ? dn : nullptr, ncache, bondcache ? db : nullptr, nbcache,
                                  k.u.as<double>(), uold ? k.uold.as<double>() : nullptr, k.kvals.as<double>(),
                                  k.rhs.as<double>()));
    PXB_TRY(d2h(c, kvals, k.kvals.p, sizeof(double) * (size_t)k.nnz));
    PXB_TRY(d2h(c, rhs, k.rhs.p, sizeof(double) * n * dim));
    return sync(c);
}

extern "C" int pxb_assemble_ch(pxb_ctx *c, double kappa, double chi, double dt, const double *mnode,
                               const double *u, const double *uold, double *kvals, double *rhs) {
    PXB_TRY(need_geometry(c, "pxb_assemble_ch"));
    CsrState &k = c->csr;
    if (!k.ready || k.ndof != 2) return fail(PXB_ERR_STATE, "pxb_assemble_ch: set a 2-dof pattern first");
    if (!c->ch.ready) return fail(PXB_ERR_STATE, "pxb_assemble_ch: call pxb_ch_set_geometry first");
    if (!(dt > 0.0) || !mnode || !u || !uold || !kvals || !rhs) return fail(PXB_ERR_INVALID, "pxb_assemble_ch: bad arguments (transient-only)");
    const size_t n = (size_t)c->g.n;
    PXB_TRY(dev_alloc(c, k.mnode, sizeof(double) * n));
    PXB_TRY(h2d(c, k.mnode.p, mnode, sizeof(double) * n));
    PXB_TRY(h2d(c, k.u.p, u, sizeof(double) * 2 * n));
    PXB_TRY(h2d(c, k.uold.p, uold, sizeof(double) * 2 * n));
    ChAsmArgs a;
    a.n = c->g.n;
    a.kappa = kappa;
    a.chi = chi;
    a.dt = dt;
    a.off = c->g.off.as<int>();
    a.nbr = c->g.nbr.as<int>();
    a.rev = c->ch.rev.as<int>();
    a.lap = c->ch.lap.as<double>();
    a.vol = c->g.vol.as<double>();
    a.mnode = k.mnode.as<double>();
    a.ghost = c->ch.ghost.p ? c->ch.ghost.as<char>() : nullptr;
    a.rowptr = k.rowptr.as<int>();
    a.slot = k.slot.as<int>();
    a.diag = k.diag.as<int>();
    a.extra = k.exact ? k.extra.as<int>() : nullptr;
    a.u = k.u.as<double>();
    a.uold = k.uold.as<double>();
    a.kvals = k.kvals.as<double>();
    a.rhs = k.rhs.as<double>();
    if (c->ch.lrv.p && c->ch.bfl.p) {
        a.lrv = c->ch.lrv.as<double>();
        a.bfl = c->ch.bfl.as<uint8_t>();
    }
    launch_assemble_ch(a, c->stream);
    PXB_TRY(check_launch(c, "assemble_ch"));
    PXB_TRY(d2h(c, kvals, k.kvals.p, sizeof(double) * (size_t)k.nnz));
    PXB_TRY(d2h(c, rhs, k.rhs.p, sizeof(double) * 2 * n));
    return sync(c);
}
