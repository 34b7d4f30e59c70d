// Host-side (C++20) state of a perix_b200 context: device-resident geometry, operator caches, explicit-loop
// state, CSR maps and captured graphs.  One context = one device, one stream, no globals.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <map>
#include <string>
#include <vector>

#include "../../include/perix_b200.h"
#include "k_kernels.h"

namespace pxb {

// ---- error plumbing ----------------------------------------------------------------------------------------
void set_error(const std::string &msg);
int fail(int status, const std::string &msg);
int cuda_fail(cudaError_t e, const char *what);

#define PXB_CUDA_TRY(expr)                                           \
    do {                                                             \
        cudaError_t _e = (expr);                                     \
        if (_e != cudaSuccess) return ::pxb::cuda_fail(_e, #expr);   \
    } while (0)

#define PXB_TRY(expr)                   \
    do {                                \
        int _s = (expr);                \
        if (_s != PXB_OK) return _s;    \
    } while (0)

// ---- device buffer ---------------------------------------------------------------------------------------------
struct DevBuf {
    void *p = nullptr;
    size_t bytes = 0;
    DevBuf() = default;
    DevBuf(const DevBuf &) = delete;
    DevBuf &operator=(const DevBuf &) = delete;
    DevBuf(DevBuf &&o) noexcept : p(o.p), bytes(o.bytes) { o.p = nullptr; o.bytes = 0; }
    DevBuf &operator=(DevBuf &&o) noexcept {
        if (this != &o) { release(); p = o.p; bytes = o.bytes; o.p = nullptr; o.bytes = 0; }
        return *this;
    }
    ~DevBuf() { release(); }
    void release();
    template <typename T>
    T *as() const { return static_cast<T *>(p); }
};

// Pinned host staging buffer (grown on demand).
struct PinnedBuf {
    void *p = nullptr;
    size_t bytes = 0;
    PinnedBuf() = default;
    PinnedBuf(const PinnedBuf &) = delete;
    PinnedBuf &operator=(const PinnedBuf &) = delete;
    PinnedBuf(PinnedBuf &&o) noexcept : p(o.p), bytes(o.bytes) { o.p = nullptr; o.bytes = 0; }
    PinnedBuf &operator=(PinnedBuf &&o) noexcept;
    ~PinnedBuf();
};

struct Geometry {
    bool ready = false;
    int n = 0, dim = 2;
    long long nb = 0;
    long long ldb = 0;  // padded per-bond stride: nb rounded up past nb+16 to a multiple of 16 elements, so
                        // 16-byte-aligned bulk copies of any bond range stay inside the allocation
    double delta = 0.0, dx_char = 0.0;
    DevBuf off;     // int32 [n+1+16] (zero tail)
    DevBuf nbr;     // int32 [ldb], 0-based (zero tail)
    DevBuf pos;     // double2 [n] (2D) or double4 [n] (3D)
    DevBuf vol;     // double [n]
    DevBuf mirror;  // int32 [n], 1-based mirror bulk, 0 none (may be empty)
    DevBuf layer;   // int32 [n] ghost layer index (may be empty)
    DevBuf rev;     // int32 [nb] reverse bond index (built lazily)
    DevBuf node_delta, node_dxc;     // double [n] per-node horizon and spacing (variable horizon; empty: global)
    std::vector<double> h_node_delta;
    int max_family = 0;
    std::vector<int> h_off, h_mirror;
};

struct OpsCache {
    bool ready = false;
    int order = 0, nop = 0, precision = PXB_FP64;
    DevBuf ops;         // AoS [nb][nop], double or float
    DevBuf degenerate;  // uint8 [n]
    DevBuf defect;      // mixed, order 2: double [n][(nop - dim) * dim] first-moment defects (GBuildArgs::defect)
    DevBuf yeff;        // adjoint with defects: transposed-correction ybar (grown on demand)
    std::vector<int> pqr;
};

struct BcDevice {
    int n_entries = 0;
    DevBuf own;      // uint8 [n]: bitmask of components whose final value comes from the BC pass
    DevBuf src_off;  // int32 [n+1]: BC target entries grouped by the node whose warp executes them
    DevBuf tgt;      // int32 [n_entries]: target node (0-based)
    DevBuf comp;     // int32 [n_entries]: component
    DevBuf form;     // int32 [n_entries]: closed form (see EpfArgs)
    DevBuf vals;     // double [4*n_entries]: val | vel | val2 | vel2 blocks
};

struct GraphKey {
    int steps, parity, prec, variant;
    bool operator<(const GraphKey &o) const {
        if (steps != o.steps) return steps < o.steps;
        if (parity != o.parity) return parity < o.parity;
        if (prec != o.prec) return prec < o.prec;
        return variant < o.variant;
    }
};

struct EpfState {
    bool ready = false, started = false;
    int precision = PXB_FP64;
    double C11 = 0, C12 = 0, C66 = 0, rho = 1, b[3] = {0, 0, 0}, sc = 0;
    double r2min = 0;  // smallest positive squared bond length (reference rounding)
    int tension_only = 1;
    DevBuf G;          // SoA Navier operators [c][ldb], double or float (c = 3 in 2D, 6 in 3D)
    DevBuf P;          // SoA packed Navier coefficients [c][ldb] (same type): the staged step kernels' stream
    DevBuf xib;        // mixed: FP32 reference bond vectors [dim][ldb] (the staged kernels' stretch pre-test)
    DevBuf sc_bond;    // variable horizon: per-bond critical stretch s_c(0.5 (delta_i + delta_j)) [ldb]
    // explicit-loop adjoint (pxb_epf_adjoint_d): checkpoints, a segment's states, the two ping-pong states, the
    // adjoint vectors A (dJ/du^n), R (dJ/du^{n-1} carried), W (BC-transposed A), step times, dC accumulator
    DevBuf adj_ckpt, adj_seg, adj_p[2], adj_A, adj_R, adj_W, adj_t, adj_dC, adj_umax;
    DevBuf adj_u0;       // the recorded loop's u0 (the reverse sweep's start term)
    DevBuf adj_GR;       // the Navier operators in reverse-bond order (the adjoint kernel's second stream)
    DevBuf adj_HR;       // the health mask in reverse-bond order (rebuilt by every reverse sweep)
    bool adj_GR_none = false;  // no room for adj_GR: the adjoint kernel gathers the reverse bonds' operators
    DevBuf adj_SG;             // per-node sums of the healthy own bonds' operators (rebuilt by every reverse sweep)
    DevBuf adj_UW;             // the staged adjoint's gather rows (u, w) interleaved, [n][2 dim] (empty: apart)
    bool adj_sg_on = false;    // inside a reverse sweep whose families all have reverse bonds: reverse-only kernel
    // the recorded forward loop (pxb_epf_record_d): rec_steps < 0 when there is none; rec_all: every state kept
    double rec_dt = 0.0;
    int rec_steps = -1, rec_K = 1;
    bool rec_all = false;
    int rec_seg = -1;  // checkpointed recording: the segment whose states adj_seg holds (-1: none)
    DevBuf health;     // uint8 [ldb] (zero tail)
    DevBuf u[2];       // double [n*dim + 8] ping-pong: u[cur] = u^n, u[cur^1] = u^{n-1}
    DevBuf accel;      // double [n*dim]
    DevBuf counters;   // unsigned long long [6]: [0] broken bonds, [2] staged-kernel wait failures (u32),
                       // [4] broken bonds before the last rate call, [5] scratch of the set-up and sweep reductions
    PinnedBuf rate_h;  // host copy of counters[0..4] for the per-step rate call
    cudaEvent_t rate_done = nullptr;  // end of a rate call's work (polled by the host)
    // the per-step rate call captured as one graph for one pair of pinned host buffers (u in, acceleration out),
    // the state slot u[cur] and the schedule variant; rate_last_* are the buffers of the previous call
    cudaGraphExec_t rate_graph = nullptr;
    // pipelined rate call (staged variants, large meshes, pinned buffers): node chunks [rate_bounds[k],
    // rate_bounds[k+1]), uploaded and computed in order; chunk k's kernel waits for the upload of chunk
    // rate_need[k] (where its highest neighbour lies), and its acceleration goes down while the next chunk
    // computes; rate_K <= 1: one upload, one kernel, one download
    bool rate_plan_done = false;
    int rate_K = 1;
    std::vector<int> rate_bounds, rate_need;
    cudaStream_t rate_up = nullptr, rate_down = nullptr;
    std::vector<cudaEvent_t> rate_ev;  // [0] start, [1] downloads done, [2..2+K) uploads, [2+K..2+2K) kernels
    const void *rate_u = nullptr, *rate_last_u = nullptr;
    void *rate_a = nullptr, *rate_last_a = nullptr;
    int rate_cur = -1, rate_variant = -1, rate_last_variant = -1;
    DevBuf umax;       // unsigned long long [chunk] per-step max |u| keys
    DevBuf tsched;     // double [chunk] t_{n+1} of each step in the chunk
    PinnedBuf tsched_h;
    int cur = 0;
    double t = 0.0, dt = 0.0;
    double dt_prev = 0.0;  // dt of the last step taken (differs from dt after a clamped final step)
    long long step = 0;
    std::vector<double> umax_hist;  // host history for the windowed blow-up guard
    BcDevice bc;
    bool has_bc = false;
    std::map<GraphKey, cudaGraphExec_t> graphs;
    int graph_chunk = 0;
    int variant = 1;   // schedule variant of the explicit kernel (set by the autotuner or pxb_epf_set_variant)
    bool evict_first = false;  // the step's bond streams exceed the L2: stage them with an evict-first policy
    int wait_tries = -1;       // staged kernels' consumer waits: try_wait calls allowed (-1: the default bound)
};

struct CsrState {
    bool ready = false;
    int ndof = 1;
    long long nnz = 0;
    DevBuf rowptr, cols;
    DevBuf slot;       // int32 [nb*ndof*ndof]: CSR slot of (row i*ndof+a, col j*ndof+b) for bond t
    DevBuf diag;       // int32 [n*ndof*ndof]: slot of the diagonal block entries
    // exact pattern (every row = own block + family blocks + mirror block): the assembly kernels then write every
    // entry once instead of zeroing the rows first; extra = slots of a mirror block outside the family (-1 none)
    bool exact = false;
    // ndof 2 and rows 2i, 2i+1 share one list of column pairs (2j, 2j+1): the block view (block_view) and, built on
    // first use by an adjoint solve, the block view of the transpose with its value permutation
    bool blocked2 = false, transposed = false;
    std::vector<int> h_bptr, h_bcol;
    DevBuf bptr, bcol, tbptr, tbcol, tperm;
    DevBuf extra;      // int32 [n*ndof*ndof]
    DevBuf kvals, rhs, u, uold, fnode, mnode;
};

struct ChState {
    bool ready = false;
    DevBuf rev, lap, ghost;
    DevBuf lrv, bfl;  // the assembly's bond-order streams: vol_j lap[rev t]; ghost j | 2 (reverse exists)
    // implicit run (ch_solver.cpp): state, Newton / BiCGStab work vectors, block-Jacobi inverse, history
    DevBuf U, Uold, dU, rhs, kv, mnode, binv, red, ones, hist;
    DevBuf w[11];
    DevBuf nodal;  // per-node scratch (energy, dkappa terms)
    DevBuf kvt;         // values of K^T (adjoint solves)
    DevBuf bicg;        // BiCGStab scalars and partial sums (k_bicg.cu)
    PinnedBuf bicg_h;   // host copy of the scalars
};

}  // namespace pxb

namespace pxb {
// Batched clouds (C-ABI pxb_batch_*): concatenated geometry, task table, operators of every cloud.
struct BatchState {
    bool ready = false, built = false;
    int nclouds = 0, n = 0;
    long long nb = 0, ops_len = 0, out_len = 0, def_len = 0;
    int ntasks = 0, ntasks3 = 0;  // tasks of 3D clouds first: [0, ntasks3), then 2D
    int precision = PXB_FP64;
    int gvariant = 3, avariant = 0;  // schedules (batch_gbuild_schedule / batch_apply_schedule)
    std::vector<BatchCloud> h_clouds;
    DevBuf clouds, tasks, off, nbr, pos, vol, ops, degenerate, counters;
    DevBuf defect;  // mixed: per-cloud first-moment defects of the second-derivative operators
};
}  // namespace pxb

struct pxb_ctx {
    int device = 0;
    size_t mem_limit = 0;  // device bytes the context may hold (0: no limit beyond the GPU's)
    int gbuild_schedule = -1;  // g-build: -1 by problem, 0 lane groups, 1 one warp per node, 2 the same with
                               // its products on the FP64 tensor cores
    int adj_schedule = -1;     // recorded reverse sweep: -1 default (4), 0 both operator streams, 1 reverse-only,
                               // 2-4 reverse-only staged (bulk-copy ring) in three launch configurations
    int rate_chunks = -1;      // pipelined rate call: -1 by mesh size, 1 off, 2..8 node chunks
    cudaStream_t own = nullptr;
    cudaStream_t stream = nullptr;
    long long launches = 0;
    pxb::Geometry g;
    pxb::OpsCache ops;
    pxb::EpfState epf;
    pxb::CsrState csr;
    pxb::ChState ch;
    pxb::BatchState batch;
    pxb::DevBuf scratch;
    pxb::PinnedBuf pinned;
};

namespace pxb {
// device allocation helpers (track bytes per context)
int dev_alloc(pxb_ctx *c, DevBuf &b, size_t bytes);
int dev_upload(pxb_ctx *c, DevBuf &b, const void *host, size_t bytes);
int h2d(pxb_ctx *c, void *dst, const void *src, size_t bytes);
int d2h(pxb_ctx *c, void *dst, const void *src, size_t bytes);
int ensure_pinned(PinnedBuf &b, size_t bytes);
int sync(pxb_ctx *c);
int check_launch(pxb_ctx *c, const char *what);
size_t ctx_bytes(const pxb_ctx *c);
int l2_flush(pxb_ctx *c, size_t bytes);  // writes `bytes` through the L2 on the context stream (0: nothing)
int wait_failure(pxb_ctx *c, unsigned int werr, const char *what);  // report (and clear) a staged wait that ran out
}  // namespace pxb
