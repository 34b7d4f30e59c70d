// Kernel argument blocks and launchers shared between the .cu kernels and the C++ host code.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <vector>

namespace pxb {

constexpr int kGbuildThreads = 128;
constexpr int kEpfThreads = 256;
constexpr int kApplyThreads = 256;

// ---------------------------------------------------------------------------------------------------- g-build
struct GBuildArgs {
    int n = 0;
    long long nb = 0;
    const int *off = nullptr;
    const int *nbr = nullptr;
    const void *pos = nullptr;  // double2 / double4
    const double *vol = nullptr;
    const int *layer = nullptr;
    double delta = 0.0, dx_char = 0.0;
    void *ops = nullptr;  // AoS [nb][nop] (double, or float when mixed); may be null
    void *G = nullptr;    // SoA Navier [c][nb] (double, or float when mixed); may be null
    uint8_t *degenerate = nullptr;
    unsigned int *n_degenerate = nullptr;
    int *first_degenerate = nullptr;
    int node_base = 0;       // positions are read at pos[j - node_base] (a batch cloud's slice)
    long long bond_base = 0; // AoS operators are written at ops[(t - bond_base) * nop]
    // MIXED, order 2: per node the first moments of the stored (FP32-rounded) second-derivative operators,
    // sum_j g~^k_j xi_j[m] for k = dim..nop-1, m < dim (exactly 0 for exact operators; FP32 is ample for a
    // correction of that size), at defect[(i - node_base) * (nop - dim) * dim + (k - dim) * dim + m]; may be null
    float *defect = nullptr;
    // per-node horizon and spacing (variable horizon), read at [i - node_base]; null: delta / dx_char for all
    const double *node_delta = nullptr;
    const double *node_dxc = nullptr;
};
cudaError_t launch_gbuild(const GBuildArgs &a, int dim, int order, bool mixed, int grid, cudaStream_t s);
bool gbuild_supported(int dim, int order);
// one warp per node (k_gbuild_warp.cu): FP64 moment sums; MIXED stores FP32 operators (and the order-2 defects)
// tc: moment sums and operator products on the FP64 tensor cores (up to nine monomials)
cudaError_t launch_gbuild_warp(const GBuildArgs &a, int dim, int order, bool mixed, bool tc, cudaStream_t s);
bool gbuild_warp_supported(int dim, int order);

// ------------------------------------------------------------------------------ families on the device (A1)
constexpr int kFamMax = 256;   // largest family the device build sorts
constexpr int kFamCell = 4096; // largest cell population (12-bit positions in the visit key)
struct FamArgs {
    int n = 0, is3d = 0;
    const double *coords = nullptr;  // xyz per node
    double lo[3] = {0, 0, 0};
    double radius = 0, r2 = 0, r2tol = 0;
    unsigned mask = 0;               // cell table size - 1 (power of two)
    unsigned long long *keys = nullptr;
    int *ccount = nullptr, *cminid = nullptr, *cstart = nullptr, *cfill = nullptr, *members = nullptr;
    int *cell_of = nullptr, *cxyz = nullptr, *pos = nullptr;
    int *fcount = nullptr;
    const int *off = nullptr;  // family offsets (a batch cloud's slice: global bond indices)
    int off_base = 0;          // off[0]: fkey / fval are indexed from it
    unsigned long long *fkey = nullptr;
    int *fval = nullptr;
    int *nbr = nullptr;  // output, 0-based, plus id_base (a batch cloud's first node)
    int id_base = 0;
    int *err = nullptr;
};
cudaError_t launch_fam_cells(const FamArgs &a, cudaStream_t s);
cudaError_t launch_fam_members(const FamArgs &a, cudaStream_t s);
cudaError_t launch_fam_sort_cells(const FamArgs &a, cudaStream_t s);
cudaError_t launch_fam_candidates(const FamArgs &a, bool write, cudaStream_t s);
cudaError_t launch_fam_sort(const FamArgs &a, cudaStream_t s);

// ------------------------------------------------------------------------------------------ batched clouds
// Many independent clouds (2D and 3D mixed) in one node/bond numbering: cloud c owns nodes [node0, node0+n) and
// bonds [bond0, bond0+nb) of the global CSR; its operators (order 2: nop 5 in 2D, 9 in 3D, AoS [nb][nop]) start
// at element ops_off, its apply output ([n][nop]) at element out_off, its positions (double2 in 2D, double4 in
// 3D) at byte pos_off.  A task is a run of consecutive nodes of one cloud; persistent warps take tasks from a
// counter (zero at launch).
struct BatchCloud {
    int dim = 2, node0 = 0, n = 0, pad = 0;
    long long bond0 = 0, nb = 0;
    long long ops_off = 0, out_off = 0, pos_off = 0;
    long long def_off = 0;  // element offset of the cloud's defects ([n][(nop - dim) * dim], mixed)
    double delta = 0.0, dx_char = 0.0;
};
struct BatchTask {
    int cloud = 0, first = 0, count = 0, dim = 2;
};
struct BatchArgs {
    int task0 = 0, ntasks = 0;  // tasks [task0, task0 + ntasks) of the table
    const BatchTask *tasks = nullptr;
    const BatchCloud *clouds = nullptr;
    const int *off = nullptr;
    const int *nbr = nullptr;  // 0-based global node ids
    const unsigned char *pos = nullptr;
    const double *vol = nullptr;
    void *ops = nullptr;  // double, or float when mixed
    uint8_t *degenerate = nullptr;
    unsigned int *n_degenerate = nullptr;
    int *first_degenerate = nullptr;
    float *defect = nullptr;  // mixed: per-cloud first-moment defects at def_off (GBuildArgs::defect)
    unsigned int *counter = nullptr;
    const double *u = nullptr;  // apply: field (N)
    double *out = nullptr;      // apply: derivatives
};
// schedules: lanes per node for 2D / 3D clouds, and whether both dimensions share one launch
struct BatchSchedule {
    int lpn2, lpn3;
    bool split;
    bool warp = false;  // g-build: one warp per node (k_gbuild_warp.cu) instead of lane groups
    bool tc = false;    // g-build, warp per node: moment sums and operator products on the FP64 tensor cores
    bool hybrid = false;  // g-build, split: lane groups of lpn2 lanes for the 2D clouds, a warp per node for 3D
};
constexpr int kBatchVariants = 10;
cudaError_t launch_gbuild_batch_warp(const BatchArgs &a, bool mixed, bool split, int dims, bool tc, cudaStream_t s);
BatchSchedule batch_gbuild_schedule(int variant);
BatchSchedule batch_apply_schedule(int variant);
// dims: 1 = 2D tasks only, 2 = 3D tasks only, 3 = both
cudaError_t launch_gbuild_batch(const BatchArgs &a, bool mixed, int variant, int dims, cudaStream_t s);
cudaError_t launch_apply_batch(const BatchArgs &a, bool mixed, int variant, int dims, cudaStream_t s);

// ---------------------------------------------------------------------------------------- explicit fracture
enum EpfMode { EPF_RATE = 0, EPF_START = 1, EPF_STEP = 2, EPF_FORCE_FROZEN = 3 };

struct EpfArgs {
    int n = 0;
    long long nb = 0;
    const int *off = nullptr;
    const int *nbr = nullptr;
    const void *pos = nullptr;
    const void *G = nullptr;  // SoA [c][nb]
    const void *P = nullptr;  // TMA variants: packed Navier coefficients SoA [c][nb] (navier_pack)
    const float *xib = nullptr;  // mixed TMA variants: reference bond vectors x_j - x_i, FP32 SoA [dim][nb]
    uint8_t *health = nullptr;
    double C11 = 0, C12 = 0, C66 = 0, rho = 1, b[3] = {0, 0, 0};
    double sc = 0;                  // critical stretch
    double sc_hi2 = 0, sc_lo2 = 0;  // (1+sc)^2 and (1-sc)^2 (0 when 1-sc <= 0)
    int damage = 0, tension_only = 1;
    const double *u = nullptr;    // u^n (N*dim)
    double *u_other = nullptr;    // STEP: u^{n-1} in, u^{n+1} out; START: u^{-1} out
    const double *v0 = nullptr;   // START
    double *accel = nullptr;      // RATE / FORCE_FROZEN
    double dt = 0, dt2 = 0;  // START: dt2 = 0.5*dt*dt; STEP: dt2 = dt*dt
    // time of the new state for the BC pass: t_sched[step_in_chunk]
    const double *t_sched = nullptr;
    int step_in_chunk = 0;
    // BC program (STEP only)
    // entry e (executed by the warp of its source node): target node, component, form
    //   0: U(src)   1: G   2: 2G - U(src)   3: 2G - G2,   G = val + vel*t, G2 = val2 + vel2*t
    const uint8_t *bc_own = nullptr;
    const int *bc_off = nullptr;
    const int *bc_tgt = nullptr;
    const int *bc_comp = nullptr;
    const int *bc_form = nullptr;
    const double *bc_val = nullptr, *bc_vel = nullptr, *bc_val2 = nullptr, *bc_vel2 = nullptr;
    unsigned long long *umax = nullptr;     // per-step max|u| keys
    unsigned long long *n_broken = nullptr; // broken-bond counter
    int maxb = 0;                           // TMA variants: staged bonds per tile (multiple of 32)
    unsigned int *err = nullptr;            // TMA variants: pipeline waits that ran out
    int rate = 0;                           // TMA variants: RATE mode (accel out; u_other and BCs unused)
    int node0 = 0;  // TMA variants: the launch computes nodes [node0, n) (node0 a multiple of 64; RATE mode only)
    // TMA variants, STEP mode: launch with programmatic stream serialisation, so that inside a captured loop of
    // steps the next step's blocks start their set-up while this step's last blocks finish (host-side only)
    int pdl = 0;
    int evict_first = 0;  // TMA variants: stage the bond streams with an L2 evict-first policy
    // STEP: a step whose dt differs from the previous one takes the variable-step form (see cd_next)
    int var_step = 0;
    double cv_rho = 0, cv_w = 0;
    int wait_tries = 1 << 19;  // TMA variants: try_wait calls a consumer wait may make before it gives up
    // variable horizon: per-bond critical stretch [nb] (null: sc for every bond); the staged kernels do not read
    // it, launch_epf runs the lane-group kernel instead
    const double *sc_bond = nullptr;
    // staged kernels with the displacement-first test: a bond whose relative displacement satisfies |e|^2 < e2_hold
    // clearly holds (its stretch is at most |e| / |xi| < sc for every bond length |xi| >= r_min), so its positions
    // are not gathered; e2_hold = (sc (1 - 1e-6) - 1e-12)^2 r_min^2 (0: every bond takes the position test)
    double e2_hold = 0;
};
// schedule variants of the explicit kernel (lanes per node x bonds per lane per pass); see k_epf.cu
constexpr int kEpfTmaConfigs = 16;                // staged (TMA) configurations per dimension
constexpr int kEpfVariants = 5 + kEpfTmaConfigs;  // 0-2 lane groups, 3-4 CSR tiles, 5.. staged
cudaError_t launch_epf(const EpfArgs &a, int dim, bool mixed, int mode, int variant, cudaStream_t s);
// P[c][t] from G[c][t] (t < ldb, SoA stride ldb): 2D p11 = C11 Gxx + C66 Gyy, p22 = C66 Gxx + C11 Gyy,
// pxy = (C12 + C66) Gxy; 3D p11/p22/p33 and (C12 + C66) times Gxy, Gxz, Gyz
// xib[d][t] = (float)(x_j - x_i)[d] for every bond t = (i -> j) (t < off[n]; the tail is left as it is); and, when
// r2min_key is given, the smallest positive squared bond length in the reference's rounding (x_j - x_i and the dot
// product rounded op by op) as an atomicMin over the bit pattern (the caller initialises it to +inf)
cudaError_t launch_bond_vectors(int n, int dim, const int *off, const int *nbr, const void *pos, long long ldb,
                                float *xib, unsigned long long *r2min_key, cudaStream_t s);
cudaError_t launch_navier_pack(const void *G, void *P, long long ldb, int dim, bool mixed, double C11, double C12,
                               double C66, cudaStream_t s);
int epf_grid(int n, int dim, int variant);
int epf_lanes_per_node(int dim, int variant);
int epf_tile_nodes(int dim, int variant);
// the CSR-stream variants map at most 4096 bonds per tile
bool epf_variant_fits(int dim, int variant, int max_family);
// TMA-staged step (k_epf_tma.cu): STEP mode only; `which` selects one of kEpfTmaConfigs configurations
bool epf_is_tma(int variant);
int epf_tma_maxb(int dim, int variant, int max_family);
int epf_tma_tile_nodes(int dim, int which);
size_t epf_tma_smem(int dim, bool mixed, int which, int maxb);
int epf_tma_lanes(int dim, int which);
cudaError_t launch_epf_tma(const EpfArgs &a, int dim, bool mixed, int which, cudaStream_t s);
// grid, block and dynamic shared memory of the last staged launch (host bookkeeping for the launch-floor probe)
struct LaunchShape {
    int grid, block;
    size_t smem;
};
LaunchShape epf_tma_last_shape();
// an empty kernel with the given launch shape (the fixed cost of a launch, timed like a step)
cudaError_t launch_empty(int grid, int block, size_t smem, cudaStream_t s);

struct EpfAdjArgs {
    int n = 0;
    long long nb = 0;
    const int *off = nullptr;
    const int *nbr = nullptr;
    const int *rev = nullptr;
    const void *G = nullptr;
    const void *GR = nullptr;  // optional: G in reverse-bond order, GR[c][t] = G[c][rev t] (0 without a reverse bond)
    const uint8_t *hrev = nullptr;  // optional with GR: health in reverse-bond order (then rev is not read)
    const uint8_t *health = nullptr;
    double C11 = 0, C12 = 0, C66 = 0, inv_rho = 1;
    const double *u = nullptr;
    const double *abar = nullptr;
    double *ubar = nullptr;
    double *dC = nullptr;  // 3 doubles, atomically accumulated (must be zeroed)
    // reverse time step (step != 0): Lbar = scale abar / rho, and per node
    //   ubar = c_r rin + c_w abar + (da/du)^T (scale abar),   rout = c_o abar   (rin / rout may alias, per node)
    int step = 0;
    double scale = 1.0, c_r = 0.0, c_w = 0.0, c_o = 0.0;
    const double *rin = nullptr;
    double *rout = nullptr;
    // reverse-only mode (with GR and hrev, the damage mask frozen for the sweep): SG[m][c] = sum over the node's
    // healthy bonds of G[c][t] (launch_own_sums), so the own-bond term is one 3x3 product per node and dJ/dC is
    // summed over the reverse bonds; the forward operator stream is not read
    const double *SG = nullptr;
    // staged reverse-only kernel (launch_epf_adjoint_tma): bonds staged per tile (epf_adj_tma_maxb), the wait-failure
    // counter and budget, the L2 policy of the bond streams
    int maxb = 0;
    unsigned int *err = nullptr;
    int wait_tries = 1 << 19;
    int evict_first = 0;
    // staged kernel, optional: the rows (u_j, abar_j) interleaved, [n][2 dim] (launch_bc_transpose's uw), so that a
    // reverse bond gathers its source node with dim 16-byte loads
    const double *UW = nullptr;
};
cudaError_t launch_epf_adjoint(const EpfAdjArgs &a, int dim, bool mixed, int grid, cudaStream_t s);
// The reverse-only adjoint step with the tile's ids, reverse health and node rows (u, abar, rin) staged through a
// shared-memory ring by bulk copies, and the reverse operators prefetched into L2 (SG, GR and hrev required; u, abar
// and rin 16-byte aligned, readable 64 bytes past n*dim; hrev readable to ldb); which = 0, 1, 2 picks the lanes per
// node / bonds per pass / occupancy configuration.
cudaError_t launch_epf_adjoint_tma(const EpfAdjArgs &a, int dim, bool mixed, int which, cudaStream_t s);
int epf_adj_tma_maxb(int dim, int max_family);
// SG[m][c] = sum_{t in fam(m), health[t]} G[c][t] (nc = 3 in 2D, 6 in 3D, FP64 sums); missing[0] += the bonds
// without a reverse bond (rev t < 0)
cudaError_t launch_own_sums(int n, int dim, bool mixed, const int *off, const int *rev, const uint8_t *health,
                            const void *G, long long ldb, double *SG, unsigned int *missing, cudaStream_t s);
// reach[k] = max(k's bonds' neighbour ids) for the node chunks [bounds[k], bounds[k+1]) (reach zeroed by the caller)
cudaError_t launch_chunk_reach(const int *off, const int *nbr, const int *bounds, int nchunks, int *reach,
                               cudaStream_t s);
// hr[t] = health[rev t] for t < nb (0 where rev t < 0)
cudaError_t launch_reverse_health(const uint8_t *health, const int *rev, uint8_t *hr, long long nb, cudaStream_t s);
// GR[c][t] = G[c][rev t] for t < nb (0 where rev t < 0), SoA stride ldb
cudaError_t launch_reverse_gather(const void *G, void *GR, const int *rev, long long nb, long long ldb, int dim,
                                  bool mixed, cudaStream_t s);
// transpose of the BC program's linear part: w[i] = (component owned by the BC pass ? 0 : a[i]) + sum over the
// entries executed by node i of +-a[target] (form 0: +, form 2: -, constants: none)
// with uw: also uw[i] = (u[i], w[i]) interleaved ([n][2 dim]: the staged adjoint's gather rows)
cudaError_t launch_bc_transpose(const EpfArgs &bc, int n, int dim, const double *a, double *w, cudaStream_t s,
                                const double *u = nullptr, double *uw = nullptr);

// ---------------------------------------------------------------------------------------------------- apply
struct ApplyArgs {
    int n = 0;
    int nop = 0;
    int nk = 0;
    int slots[32];
    const int *off = nullptr;
    const int *nbr = nullptr;
    const int *rev = nullptr;
    const void *ops = nullptr;  // AoS [nb][nop]
    const double *u = nullptr;  // forward: u (N); adjoint: ybar (N*nk)
    double *out = nullptr;      // forward: N*nk; adjoint: N
    // mixed, order 2: first-moment defects of the second-derivative operators (GBuildArgs::defect); the forward
    // subtracts sum_m defect[k][m] * D^m u from every second derivative it returns
    const float *defect = nullptr;
    int dim = 2;
};
cudaError_t launch_apply(const ApplyArgs &a, bool mixed, int grid, cudaStream_t s);
cudaError_t launch_apply_adjoint(const ApplyArgs &a, bool mixed, int grid, cudaStream_t s);
struct AdjPrepArgs {
    int n = 0, dim = 2, nop = 0, nk = 0, next = 0;
    int slots[32], ext[32];
    const float *defect = nullptr;
    const double *ybar = nullptr;
    double *yeff = nullptr;
};
cudaError_t launch_apply_adjoint_prep(const AdjPrepArgs &p, cudaStream_t s);

// ------------------------------------------------------------------------------------------------------- misc
cudaError_t launch_build_rev(int n, const int *off, const int *nbr, int *rev, int grid, cudaStream_t s);
cudaError_t launch_pos_pack(int n, int dim, const double *coords3, void *pos, cudaStream_t s);
cudaError_t launch_ids_to0(long long nb, const int *ids1, int *ids0, cudaStream_t s);
cudaError_t launch_health_from_double(long long nb, const double *h, uint8_t *out, cudaStream_t s);
cudaError_t launch_health_to_double(long long nb, const uint8_t *h, double *out, cudaStream_t s);
cudaError_t launch_count_zero(long long nb, const uint8_t *h, unsigned long long *count, cudaStream_t s);
cudaError_t launch_l2_flush(void *buf, size_t bytes, cudaStream_t s);

// ------------------------------------------------------------------------------------------------ CSR assembly
struct CsrMapArgs {
    int n = 0, ndof = 1;
    const int *off = nullptr;
    const int *nbr = nullptr;
    const int *rowptr = nullptr;
    const int *cols = nullptr;
    int *slot = nullptr;   // [nb*ndof*ndof]
    int *diag = nullptr;   // [n*ndof*ndof]
    int *missing = nullptr;
    const int *mirror = nullptr;  // 1-based mirror bulk node, 0 none (may be NULL)
    int *extra = nullptr;         // [n*ndof*ndof] slots of the mirror block when it is not a family member, else -1
    int *inexact = nullptr;       // rows holding entries beyond own block + family + mirror block
};
cudaError_t launch_csr_map(const CsrMapArgs &a, cudaStream_t s);

struct ScalarAsmArgs {
    int n = 0, dim = 2, nop = 0, type = 0, mixed = 0;
    int s_xx = -1, s_yy = -1, s_zz = -1;
    double coef = 0, f = 0, dt = 0;
    const double *f_node = nullptr;
    const int *off = nullptr;
    const int *nbr = nullptr;
    const int *rowptr = nullptr;
    const int *slot = nullptr;
    const int *diag = nullptr;
    const void *ops = nullptr;
    const uint8_t *degenerate = nullptr;
    const double *u = nullptr, *uold = nullptr;
    double *kvals = nullptr, *rhs = nullptr;
};
cudaError_t launch_assemble_scalar(const ScalarAsmArgs &a, cudaStream_t s);

struct ChAsmArgs {
    int n = 0;
    const int *extra = nullptr;  // exact pattern: mirror-block slots to clear (rows are not zeroed first)
    double kappa = 0, chi = 0, dt = 1;
    const int *off = nullptr, *nbr = nullptr, *rev = nullptr;
    const double *lap = nullptr, *vol = nullptr, *mnode = nullptr;
    const char *ghost = nullptr;
    const int *rowptr = nullptr, *slot = nullptr, *diag = nullptr;
    const double *u = nullptr, *uold = nullptr;
    double *kvals = nullptr, *rhs = nullptr;
    // optional bond-order streams of the fixed geometry (launch_ch_bond_streams): lrv[t] = vol[j] lap[rev t] (0
    // without a reverse bond) and bfl[t] = (ghost j) | 2 (reverse bond exists); with them the kernel gathers only
    // the neighbour's mobility and u
    const double *lrv = nullptr;
    const uint8_t *bfl = nullptr;
};
cudaError_t launch_assemble_ch(const ChAsmArgs &a, cudaStream_t s);
cudaError_t launch_ch_bond_streams(int n, const int *off, const int *nbr, const int *rev, const double *lap,
                                   const double *vol, const char *ghost, double *lrv, uint8_t *bfl, cudaStream_t s);
// Stress-coupled Cahn-Hilliard (rows c, mu, u_x, u_y[, u_z] per node; ndof = dim + 2): the device twin of
// the reference's stressCahnHilliardKernel (src/PDSystem/CudaAssembleKernels.cu:685-874) on the FP64 order-2
// operator cache.  sl = operator slots of d/dx d/dy d/dz d2/dx2 d2/dxdy d2/dy2 d2/dxdz d2/dydz d2/dz2 (-1 absent).
struct StressChAsmArgs {
    int n = 0, dim = 2, nop = 0;
    int sl[9] = {-1, -1, -1, -1, -1, -1, -1, -1, -1};
    double C11 = 0, C12 = 0, C66 = 0, A = 0, Kh = 0, Ch = 0, Omega = 0, cref = 0, chi = 0, kappa = 0, dt = 1;
    double kres = 1e-8, rho = 0;
    const int *off = nullptr, *nbr = nullptr, *rev = nullptr;
    const double *lap = nullptr, *vol = nullptr, *mnode = nullptr;
    const char *ghost = nullptr;
    const double *ops = nullptr;        // FP64 [nb][nop]
    const uint8_t *degenerate = nullptr;
    const double *health = nullptr;     // [nb] frozen bond health (NULL: every bond intact)
    const double *vel = nullptr;        // [n*dim] committed velocity (inertia when rho > 0)
    const int *rowptr = nullptr, *slot = nullptr, *diag = nullptr;
    const double *u = nullptr, *uold = nullptr;
    double *kvals = nullptr, *rhs = nullptr;
};
cudaError_t launch_assemble_stress_ch(const StressChAsmArgs &a, cudaStream_t s);
// Implicit PDDO dynamic fracture (rows u per node; ndof = dim): the device twin of the reference's
// cachedAssembleKernel (src/PDSystem/CudaAssembleKernels.cu:880-1024) on the FP64 order-2 operator cache.
// nodecache[i*ncache + a] = committed velocity, bondcache[t*nbcache] = frozen bond health.
struct CachedAsmArgs {
    int n = 0, dim = 2, nop = 0, ncache = 3, nbcache = 1;
    int sl[6] = {-1, -1, -1, -1, -1, -1};  // d2/dx2 d2/dxdy d2/dy2 d2/dxdz d2/dydz d2/dz2
    double C11 = 0, C12 = 0, C66 = 0, rho = 0, dt = 1, b[3] = {0, 0, 0};
    const int *off = nullptr, *nbr = nullptr;
    const void *pos = nullptr;          // double2 / double4
    const double *ops = nullptr;        // FP64 [nb][nop]
    const uint8_t *degenerate = nullptr;
    const double *nodecache = nullptr, *bondcache = nullptr;
    const int *rowptr = nullptr, *slot = nullptr, *diag = nullptr;
    const double *u = nullptr, *uold = nullptr;
    double *kvals = nullptr, *rhs = nullptr;
};
cudaError_t launch_assemble_cached(const CachedAsmArgs &a, cudaStream_t s);
// Output projections of the explicit state (k_project.cu; ExplicitPDDOFracElement.cpp:324-405).  Outputs may be
// NULL; stress and strain are 3x3 row-major per node.  sl = operator slots of d/dx, d/dy, d/dz.
struct ProjectArgs {
    int n = 0, dim = 2, nop = 0, plane_strain = 1;
    int sl[3] = {-1, -1, -1};
    double C12 = 0, C66 = 0;
    const int *off = nullptr, *nbr = nullptr;
    const double *ops = nullptr;      // FP64 [nb][nop]
    const uint8_t *health = nullptr;  // [nb]
    const double *u = nullptr;        // [n*dim]
    double *damage = nullptr, *von_mises = nullptr, *stress = nullptr, *strain = nullptr;
};
cudaError_t launch_epf_project(const ProjectArgs &a, cudaStream_t s);
// ---- device linear algebra and Cahn-Hilliard Newton / adjoint pieces (k_linalg.cu) ----
int dot_scratch_doubles();
// *out = a . b over n entries (fixed-order reduction; scratch: dot_scratch_doubles() doubles)
cudaError_t launch_dot(long long n, const double *a, const double *b, double *scratch, double *out, cudaStream_t s);
cudaError_t launch_axpby(long long n, double alpha, const double *x, double beta, double *y, cudaStream_t s);
cudaError_t launch_block_inv(int n, const int *diag, const double *val, bool transpose, double *binv, cudaStream_t s);
cudaError_t launch_ch_ghost_rows(int n, const int *mirror, const int *rowptr, const int *cols, const double *u,
                                 double *kv, double *rhs, cudaStream_t s);
struct ChAdjArgs {
    int n = 0;
    double M0 = 1.0;
    const int *off = nullptr, *nbr = nullptr, *rev = nullptr, *mirror = nullptr;
    const char *ghost = nullptr;
    const double *lap = nullptr, *vol = nullptr, *u = nullptr, *x = nullptr;
    double *y = nullptr;
};
// CSR sparsity pattern on the device (k_pattern.cu): count pass with the node-list scan, then the fill
struct PatternArgs {
    int n = 0, ndof = 1;
    const int *off = nullptr, *nbr = nullptr;  // families, nbr 0-based
    const int *mirror = nullptr;               // 1-based mirror node, 0 none (may be NULL)
    int *count = nullptr;                      // [n] unique column nodes per node
    long long *first = nullptr;                // [n+1] exclusive scan of count
    int *overflow = nullptr;                   // nodes whose list exceeds the sort capacity
    int *rowptr = nullptr, *cols = nullptr;    // fill: [n*ndof+1], [nnz]
    int *bptr = nullptr, *bcol = nullptr;      // fill, optional: block view [n+1], [sum count]
};
int pattern_scan_blocks(int n);  // long longs of the scan's block-sum scratch
cudaError_t launch_pattern_count(const PatternArgs &a, long long *bsum, long long *total, cudaStream_t s);
cudaError_t launch_pattern_fill(const PatternArgs &a, cudaStream_t s);
// device-resident BiCGStab (k_bicg.cu): one cooperative kernel per solve, the host reads the outcome
enum BicgStatus : int { kBicgRunning = 0, kBicgDone = 2, kBicgBreakdown = 3, kBicgMaxIts = 4 };
constexpr int kBicgParts = 148 * 8;  // most blocks of the solve kernel (one partial sum slot each)
struct BicgScalars {
    double relres;
    int status, its;                     // status: kBicgRunning until the solve ends (then abort tells a timeout)
    unsigned int bar_count;              // grid barrier arrivals
    int abort;                           // set by a barrier wait that gave up
};
struct BicgArgs {
    int n = 0;                                  // node blocks (rows 2i, 2i+1)
    const int *bptr = nullptr, *bcol = nullptr;  // block view of the pattern (block_view)
    const double *val = nullptr, *binv = nullptr, *b = nullptr;
    double *x = nullptr, *r = nullptr, *r0 = nullptr, *rh = nullptr, *v = nullptr, *s = nullptr, *sh = nullptr;
    double *t = nullptr, *ph[2] = {nullptr, nullptr}, *vh[2] = {nullptr, nullptr};
    BicgScalars *sc = nullptr;
    double *part = nullptr;  // 6 * kBicgParts doubles (two alternating sets of three)
};
// Block view of a 2-dof CSR pattern (host arrays): false unless rows 2i and 2i+1 share one column list of pairs
// (2j, 2j+1); then bptr[i] = rowptr[2i] / 4 and bcol lists node i's column nodes.
bool block_view(int n, const int *rowptr, const int *cols, std::vector<int> &bptr, std::vector<int> &bcol);
// Block view of the transpose and perm: transposed value q = value perm[q] of the matrix
void block_transpose(int n, const std::vector<int> &bptr, const std::vector<int> &bcol, std::vector<int> &tbptr,
                     std::vector<int> &tbcol, std::vector<int> &perm);
cudaError_t launch_gather_values(long long nnz, const int *perm, const double *v, double *vt, cudaStream_t s);
// the whole solve A x = b (x from 0) as one cooperative kernel; the outcome is in *a.sc when it ends
cudaError_t launch_bicg_solve(const BicgArgs &a, double tol, int max_its, cudaStream_t s);
// K' = K - J_M in place on the (c, c) entries of bulk rows, J_M the mobility derivative the Picard Jacobian omits
// (the adjoint operator is K'^T); slot: bond slot map, diag: diagonal slots of the 2-dof pattern
cudaError_t launch_ch_fold_mobility(const ChAdjArgs &a, const int *slot, const int *diag, double *kv, cudaStream_t s);
// per-node lambda_mu dF_mu/dkappa
cudaError_t launch_ch_dkappa(const ChAdjArgs &a, cudaStream_t s);
struct ChEnergyArgs {
    int n = 0, nop = 0, sx = 0, sy = 1;
    double kappa = 0, chi = 0;
    const int *off = nullptr, *nbr = nullptr, *rev = nullptr, *mirror = nullptr;
    const double *vol = nullptr, *ops = nullptr, *u = nullptr;
    double *e_out = nullptr, *grad_e = nullptr, *gbar = nullptr, *fprime = nullptr;
};
cudaError_t launch_ch_energy(const ChEnergyArgs &a, cudaStream_t s);
cudaError_t launch_ch_energy_grad(const ChEnergyArgs &a, double *dedu, cudaStream_t s);
cudaError_t launch_ch_prev_cot(int n, const int *mirror, const double *lam, double dt, double *g, cudaStream_t s);
// CH one-off geometry from the order-2 operator cache (CahnHilliardElement.cpp:93-152): per bond the PDDO
// Laplacian g_xx + g_yy (+ g_zz), lambda-corrected on non-ghost bonds with lambda = 2 dim / sum_j g2_ij
// (|x_j|^2 - |x_i|^2); ghost flags from the mirror map.  slots: the operator slots of d2/dx2, d2/dy2, d2/dz2.
cudaError_t launch_ch_geometry(int n, int dim, const int *off, const int *nbr, const void *pos, const int *mirror,
                               const void *ops, bool mixed, int nop, int sxx, int syy, int szz, double *lap,
                               char *ghost, cudaStream_t s);
// mnode[i] = M0 c(1 - c), c = u[2i] clamped to [1e-8, 1 - 1e-8] (CahnHilliardElement.cpp:45-50)
cudaError_t launch_ch_mobility(int n, double M0, const double *u, double *mnode, cudaStream_t s);

}  // namespace pxb
