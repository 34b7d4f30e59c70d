/* perix_b200 — B200-native (sm_100a) PDDO hot-path backend for PeriX: the C-ABI.
 *
 * Plain C types only (no CUDA or torch types), so a C++ PeriX build, ctypes, or any FFI can bind it.
 * All functions return a pxb_status (0 = success).  On failure pxb_last_error() returns a human-readable
 * message (thread-local).  There is no CPU fallback: a device failure is returned as an error.
 *
 * Conventions (identical to the reference boundary, include/PDSystem/CudaAssemble.h:59-80):
 *   - node coordinates are xyz-interleaved doubles (3*N), z = 0 in 2D;
 *   - families are a CSR: neigh_off[N+1] (0-based offsets), neigh_id[nbtot] with 1-BASED node ids;
 *   - nodal fields are interleaved, entry (i, a) at i*ndof + a;
 *   - CSR matrices are 0-based with columns sorted per row.
 *
 * Functions suffixed _d take DEVICE pointers and enqueue on the context stream without synchronising;
 * every other function takes HOST pointers and returns after its results are in the caller's buffers.
 * A context is not re-entrant: one host thread drives it at a time.
 */
#ifndef PERIX_B200_H
#define PERIX_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PXB_VERSION 1

typedef enum {
    PXB_OK = 0,
    PXB_ERR_INVALID = 1,        /* bad argument or size */
    PXB_ERR_CUDA = 2,           /* CUDA runtime error (message in pxb_last_error) */
    PXB_ERR_DEGENERATE = 3,     /* a non-ghost family cannot support the PDDO order */
    PXB_ERR_OOM = 4,            /* device allocation failed */
    PXB_ERR_BLOWUP = 5,         /* explicit loop: non-finite or runaway displacement */
    PXB_ERR_STATE = 6,          /* call order (e.g. step before geometry) */
    PXB_ERR_UNSUPPORTED = 7     /* configuration outside what this backend implements */
} pxb_status;

typedef enum { PXB_FP64 = 0, PXB_MIXED = 1 } pxb_precision;

typedef struct pxb_ctx pxb_ctx;

/* ---- library / context --------------------------------------------------------------------------------- */
int pxb_version(void);
const char *pxb_last_error(void);
/* Create a context on CUDA device `device` with its own non-blocking stream. */
int pxb_ctx_create(int device, pxb_ctx **out);
int pxb_ctx_destroy(pxb_ctx *ctx);
/* Use an external stream (cudaStream_t passed as void*), e.g. torch's current stream.  NULL restores the
 * context's own stream, which is non-blocking: work on it is NOT ordered against the legacy default stream.
 * To share the legacy default stream (torch's default stream, handle 0) pass cudaStreamLegacy ((void*)1). */
int pxb_ctx_set_stream(pxb_ctx *ctx, void *stream);
int pxb_ctx_synchronize(pxb_ctx *ctx);
/* Device bytes currently held by the context. */
int pxb_ctx_device_bytes(pxb_ctx *ctx, size_t *bytes);
/* Caps the device bytes the context may hold (0 = no cap beyond the GPU's own memory), e.g. to share a GPU with
 * other work: an allocation past the cap fails with PXB_ERR_OOM before reaching the driver, like one the driver
 * refuses (cudaErrorMemoryAllocation is also reported as PXB_ERR_OOM).  No counterpart in the reference. */
int pxb_ctx_set_memory_limit(pxb_ctx *ctx, size_t bytes);
/* Kernel launches issued by this context since creation (graph replays count each captured launch). */
int pxb_ctx_launch_count(pxb_ctx *ctx, long long *count);

/* ---- host-side mesh utilities (C++20, no device work) ------------------------------------------------------
 * Structured PD lattice with mirrored ghosts, as PDMesh::createPDMesh builds it for an axis-aligned quad4 or
 * hex8 background mesh (reference src/PDMesh/CreatePDMesh.cpp:451-800): bulk cell centres (x fastest), then
 * one ghost per boundary face in the reference group order (2D left,right,bottom,top; 3D
 * left,right,bottom,top,back,front).  Two-phase: call with coords3==NULL to get *n_nodes. */
int pxb_lattice(int dim, int nx, int ny, int nz, const double *box /* xmin,xmax,ymin,ymax[,zmin,zmax] */,
                int *n_nodes, double *coords3, double *vols, int *mirror /* 1-based bulk id, 0 for bulk */,
                int *ghost_group /* -1 bulk, else group index in the order above */, double *dxyz /* 3 */);

/* Family lists in the reference's visit order (reference src/PDMesh/CreatePDMesh.cpp:910-1082), uniform
 * horizon `radius` (already including the 1e-6 inclusion margin).  cracks: xy segments (4 doubles) and
 * bounded quads (12 doubles); with force_only=0 a crossing bond is dropped, with force_only=1 it is kept.
 * Two-phase: neigh_id==NULL fills neigh_off only.  *nbtot receives the directed bond count. */
int pxb_families(int n, const double *coords3, double radius, int is3d, int ncracks, const double *cracks,
                 int nplanes, const double *planes, const int *mirror, int force_only, int *neigh_off,
                 int *neigh_id, long long *nbtot);

/* Families with a per-node horizon (the reference's VariableHorizon, CreatePDMesh.cpp:932-938, 1043-1057): the cell
 * size is the largest horizon and a pair is kept when |x_i - x_j|^2 <= cut^2 (1 + 64 eps), cut = max(delta_i,
 * delta_j), so each family is the dual family (it may hold j with |x_j - x_i| > delta_i).  Otherwise as
 * pxb_families. */
int pxb_families_vh(int n, const double *coords3, const double *node_horizon, int is3d, int ncracks,
                    const double *cracks, int nplanes, const double *planes, const int *mirror, int force_only,
                    int *neigh_off, int *neigh_id, long long *nbtot);
/* Per-node horizon and rim spacing (reference PDMesh::computeVariableHorizon, CreatePDMesh.cpp:828-905):
 * s_i = V_i^(1/dim), s_ref = median of s_i over bulk nodes (mirror[i] == 0; mirror may be NULL: all bulk),
 * node_delta[i] = horizon s_i / s_ref, node_spacing[i] = dx_char s_i / s_ref (may be NULL). */
int pxb_variable_horizon(int n, int dim, const double *vols, const int *mirror, double horizon, double dx_char,
                         double *node_delta, double *node_spacing);

/* Crack-crossing test for every bond of the family (reference src/PDMesh/PDMesh.cpp:104-159); out[t]=1
 * where bond t is cut.  Used to seed force-only notch health. */
int pxb_crack_cut_mask(int n, const double *coords3, const int *mirror, const int *neigh_off, const int *neigh_id,
                       int ncracks, const double *cracks, int nplanes, const double *planes, uint8_t *out);

/* CSR sparsity pattern (reference src/MathUtils/SparseMatrix.cpp:73-185).  Two-phase: cols==NULL. */
int pxb_csr_pattern(int n, int ndof, const int *neigh_off, const int *neigh_id, const int *mirror, int *rowptr,
                    int *cols, long long *nnz);

/* ---- geometry ------------------------------------------------------------------------------------------------
 * Upload the reference geometry (replaces the AssembleMesh upload of reference
 * src/PDSystem/CudaAssembleKernels.cu:1121-1146).  delta = horizon radius (with margin); dx_char =
 * max(DX,DY,DZ) or 0 to disable the rim volume correction.  mirror (1-based, 0 = none) and layer_index
 * (ghost layer, 0 bulk) may be NULL. */
int pxb_set_geometry(pxb_ctx *ctx, int n, int dim, const double *coords3, const double *vols, const int *neigh_off,
                     const int *neigh_id, double delta, double dx_char, const int *mirror, const int *layer_index);
/* The same geometry with the families built on the device: the reference's createNeighborNodes
 * (src/PDMesh/CreatePDMesh.cpp:910-1082) in its exact order (bit-equal to pxb_families), for meshes without
 * bond-cutting cracks (force-only cracks keep their bonds and are fine); radius is the family radius (the
 * reference adds its 1e-6 margin), delta the horizon of the g-build.  nbtot (may be NULL) receives the bond
 * count; pxb_get_families copies the families out (1-based ids).  PXB_ERR_UNSUPPORTED when a family exceeds
 * 256 members or a cell of size radius holds 4096 nodes or more. */
int pxb_set_geometry_points(pxb_ctx *ctx, int n, int dim, const double *coords3, const double *vols, double radius,
                            double delta, double dx_char, const int *mirror, const int *layer_index, long long *nbtot);
int pxb_get_families(pxb_ctx *ctx, int *neigh_off, int *neigh_id);
/* Variable horizon for the context's geometry (the reference's NodeHorizon / NodeSpacing): node i's moment system and
 * operators use delta_i and spacing_i (its rim correction; NULL spacing = 0, no rim correction), and bonds longer
 * than delta_i get zero operators (CalcPDOperators.cpp:113-147, 307-354).  NULL node_delta clears them.  Call after
 * pxb_set_geometry and before pxb_gbuild / pxb_epf_setup (the operator and explicit state are dropped). */
int pxb_set_node_horizons(pxb_ctx *ctx, const double *node_delta, const double *node_spacing);

/* ---- g-functions (reference PDOperators::buildGeometryCache, src/PDOperators/CalcPDOperators.cpp:356-463) ----
 * Builds the per-bond operator vectors ops[bond*nop+k] for multi-index order `order` (2D 1..4, 3D 1..3) on the
 * device.  precision PXB_MIXED stores g in FP32 with the solve in FP64; its moment sums run
 * in FP32 on delta-scaled bond vectors with compensated (two-sum) accumulation on the lane-group schedule and in FP64
 * on the warp-per-node schedule (pxb_gbuild_set_schedule).
 * Returns PXB_ERR_DEGENERATE when a non-ghost family is degenerate; *n_degenerate / *first_degenerate
 * (1-based) describe them (either may be NULL).  Deep ghosts (layer > 1) get zero operators. */
int pxb_gbuild(pxb_ctx *ctx, int order, int precision, int *n_degenerate, int *first_degenerate);
/* Schedule of the g-build kernels: 0 lane groups (a group of 8-32 lanes per node; at MIXED the moment sums run in
 * FP32 with two-sum compensation), 1 one warp per node (moment sums in FP64 at both precisions; MIXED stores FP32),
 * 2 the same with its moment sums and per-bond operator products on the FP64 tensor cores (mma m8n8k4; up to nine
 * monomials, larger systems as 1), -1 (default) the one this backend picks: warp per node in 3D and above order 2
 * (with the tensor-core products up to nine monomials), lane groups for 2D orders 1-2.
 * Orders 2D 4 and 3D 3 exist only as the warp-per-node schedule. */
int pxb_gbuild_set_schedule(pxb_ctx *ctx, int schedule);
/* nop of the current operator cache and its multi-index table (pqr: 3*nop ints, may be NULL). */
int pxb_gbuild_info(pxb_ctx *ctx, int *nop, int *pqr);
/* Copy the operator cache to host (always returned as double). */
int pxb_get_ops(pxb_ctx *ctx, double *ops);

/* g-build without any device allocation.  No counterpart in the reference: it serves callers that cannot
 * call cudaMalloc (their device memory belongs to another allocator, or they cannot afford its implicit
 * synchronisation).  Inputs and outputs are device memory owned by the caller: neigh_off_d (n+1; neigh_off_d[0]
 * == 0, non-decreasing, neigh_off_d[n] == nbtot), neigh_id0_d (nbtot, 0-BASED ids in [0, n)), coords3_d (3n,
 * xyz), vols_d (n), layer_d (n ghost layer indices, 0 bulk; may be NULL: then deep ghosts are not told apart and
 * a degenerate family anywhere is an error, whereas with it nodes of layer > 1 get zero operators as in
 * pxb_gbuild), ops_d (nbtot*nop, double, or float with PXB_MIXED), defect_d (PXB_MIXED at order 2 only: n *
 * (nop - dim) * dim floats receiving the per-node first moments of the stored second-derivative operators,
 * the correction the mixed apply subtracts, laid out [node][k - dim][m]; may be NULL, and then no correction
 * data is produced, so second derivatives from the FP32 operators alone carry an error of order 1e-7 * L/h),
 * degenerate_d (n bytes, may be NULL); stream is a cudaStream_t (NULL = legacy default stream).  The family
 * arrays are checked on the device first; a malformed list gives PXB_ERR_INVALID and no build.  Working memory
 * is one fixed 4 MiB device array shared by all calls on a device, which limits n to
 * pxb_gbuild_noalloc_max_nodes(dim) (262,128 nodes in 2D, 131,064 in 3D); larger n is rejected with
 * PXB_ERR_INVALID.  Calls that overlap on the GPU race on the shared array.  The call synchronises its stream
 * (the input check and the degenerate counters are read back), so it cannot be captured into a CUDA graph. */
int pxb_gbuild_noalloc_d(int dim, int order, int precision, int n, long long nbtot, const int *neigh_off_d,
                         const int *neigh_id0_d, const double *coords3_d, const double *vols_d, const int *layer_d,
                         double delta, double dx_char, void *ops_d, float *defect_d, uint8_t *degenerate_d,
                         int *n_degenerate, int *first_degenerate, void *stream);
int pxb_gbuild_noalloc_max_nodes(int dim);

/* ---- family-sum derivative apply ---------------------------------------------------------------------------
 * out[i*nk + s] = sum_t g^{k_s}_it (u_j - u_i) for the nk operator slots in `slots` (0-based into the
 * multi-index table), for a scalar field u (N).  The adjoint maps ybar (N*nk) to ubar (N) (transpose). */
int pxb_apply(pxb_ctx *ctx, const double *u, int nk, const int *slots, double *out);
int pxb_apply_d(pxb_ctx *ctx, const double *u_d, int nk, const int *slots, double *out_d);
int pxb_apply_adjoint(pxb_ctx *ctx, const double *ybar, int nk, const int *slots, double *ubar);
int pxb_apply_adjoint_d(pxb_ctx *ctx, const double *ybar_d, int nk, const int *slots, double *ubar_d);

/* ---- explicit_pddo_frac (reference src/ElmtSystem/ExplicitPDDOFracElement.cpp:85-300) --------------------
 * Material: C11/C12/C66 Navier constants, rho, body force b[dim], uniform critical stretch sc (0 = no
 * damage), tension_only.  pxb_epf_setup builds the per-bond Navier operator cache (2D Gxx,Gyy,Gxy;
 * 3D Gxx,Gyy,Gzz,Gxy,Gxz,Gyz) with the g-build kernel and seeds health from `health0` (nbtot, 1/0; NULL =
 * all intact). */
int pxb_epf_setup(pxb_ctx *ctx, int precision, double C11, double C12, double C66, double rho, const double *b,
                  double sc, int tension_only, const uint8_t *health0);

/* Variable horizon: every bond breaks at its own critical stretch s_c(0.5 (delta_i + delta_j)) from the fracture
 * energy G0, Young's modulus E and (2D) plane stress (ExplicitPDDOFracElement.cpp:254-261 with
 * FractureCriterion.h:30-43), instead of the uniform sc of pxb_epf_setup.  Needs pxb_set_node_horizons; call after
 * pxb_epf_setup.  The staged step kernels do not read per-bond thresholds: their variants then run the lane-group
 * kernel. */
int pxb_epf_set_variable_horizon_stretch(pxb_ctx *ctx, double G0, double E, int plane_stress);
/* One rate evaluation at u (N*dim): damage then force, a = (L+b)/rho (the reference CUDA entry
 * assembleExplicitPDDOFracAccel).  *n_broken = bonds that broke in this call. */
int pxb_epf_rate(pxb_ctx *ctx, const double *u, double *accel, long long *n_broken);
/* The reference boundary's explicit drop-in call perix_cuda::assembleExplicitPDDOFracAccel
 * (include/PDSystem/CudaAssemble.h:251-254 of the reference; shim in include/perix_cuda_compat.h) as a plain C entry
 * for FFI callers: mesh (N, dim, 1-based families, xyz coords, volumes, delta, dx_char) and element constants as the
 * reference's AssembleMesh / ExplicitPDDOFracParams carry them, u (N*dim), health_inout (nbtot doubles, 1/0,
 * updated when a bond breaks), accel_out (N*dim), *health_changed.  Uses the shim's default context (its schedule is
 * tuned at the first call of a problem).  Returns 1 on success, 0 where the C++ call returns false (reason on
 * stderr); pxb_cuda_shutdown releases the shim's context (perix_cuda::shutdown). */
int pxb_cuda_explicit_accel(int n, int dim, const int *neigh_off, const int *neigh_id, const double *coords,
                            const double *vols, double delta, double dx_char, double C11, double C12, double C66,
                            double rho, const double *body, double sc, int tension_only, int damage_on,
                            const double *u, double *health_inout, double *accel_out, int *health_changed);
void pxb_cuda_shutdown(void);

/* Output projections of the explicit state, the device twin of ExplicitPDDOFracElement::computeNodalProjection
 * (src/ElmtSystem/ExplicitPDDOFracElement.cpp:324-405): per node damage = 1 - intact/all bonds, von Mises stress,
 * Cauchy stress and small strain (3x3 row-major, 9 values per node) from the PDDO displacement gradient over the
 * whole family, with lambda = C12 and mu = C66; 2D sigma_zz = lambda tr(eps) when plane_strain, else 0.  u (NULL:
 * the current state u^n) and the current bond health.  Outputs may be NULL.  The first call builds the FP64
 * order-2 operator cache of the context if it is absent. */
int pxb_epf_project_d(pxb_ctx *ctx, const double *u_d, int plane_strain, double *damage_d, double *von_mises_d,
                      double *stress_d, double *strain_d);
int pxb_epf_project(pxb_ctx *ctx, const double *u, int plane_strain, double *damage, double *von_mises,
                    double *stress, double *strain);

/* Boundary-condition program applied after every central-difference update, in list order (reference
 * BCSystem::presetSolution, src/BCSystem/BCSystem.cpp:114-129).  Entry e: kind 0 Dirichlet (reflect across
 * the mirror bulk, or direct when direct[e] or no mirror), kind 1 Neumann copy; comp_mask bit a selects
 * component a; value/velocity dim doubles each (g(t)=value+velocity*t); has_box/box (6 doubles xmin,xmax,
 * ymin,ymax,zmin,zmax, inclusive, on the xyz node coordinates with z = 0 in 2D; an axis whose min exceeds its max
 * is unconstrained, as DirichletBC::insideBox, src/BCSystem/DirichletBC.cpp:89-98); nodes 1-based in
 * node_off[e]..node_off[e+1].  A Neumann entry naming a node without a mirror bulk node is rejected
 * (PXB_ERR_INVALID), where the reference aborts the run. */
int pxb_epf_set_bcs(pxb_ctx *ctx, int nbc, const int *kind, const int *comp_mask, const int *direct,
                    const double *value, const double *velocity, const int *has_box, const double *box,
                    const int *node_off, const int *nodes);

/* Central-difference state: u0, v0 (N*dim, v0 may be NULL).  Evaluates a0 (this also applies damage at u0,
 * exactly like the reference's pre-loop rate call) and forms u^{-1} = u0 - dt v0 + dt^2/2 a0. */
int pxb_epf_start(pxb_ctx *ctx, const double *u0, const double *v0, double dt);
/* Advance nsteps uniform steps on the device (captured into CUDA graphs of `chunk` steps; chunk<=0 picks a
 * default).  Returns PXB_ERR_BLOWUP with *bad_step (1-based) if the reference blow-up guard trips. */
int pxb_epf_advance(pxb_ctx *ctx, int nsteps, int chunk, int *bad_step);
/* Advance to the end time t_end exactly as the reference's explicit loop does (TimeStepping::solveExplicitDynamics,
 * src/TimeStepping/TimeStepping.cpp:495-599): while t < t_end - 1e-12 t_end, the attempted step is min(dt, t_end - t);
 * a step of the previous step's length is a uniform central-difference step (graph-captured chunks as in
 * pxb_epf_advance), any other - the clamped last step - takes the variable-step form
 * u + (dt/dt_prev)(u - u_prev) + dt (dt + dt_prev)/2 a (TimeStepping.cpp:537-545), with the BC pass at its new time
 * and the blow-up guard.  *steps_taken (may be NULL) receives the number of steps.  pxb_epf_advance itself always
 * takes uniform steps of dt. */
int pxb_epf_advance_to(pxb_ctx *ctx, double t_end, int chunk, int *bad_step, long long *steps_taken);
/* Read back state: u (N*dim), u_prev (N*dim), health (nbtot, as 1/0 bytes), t.  Any pointer may be NULL. */
int pxb_epf_get_state(pxb_ctx *ctx, double *u, double *u_prev, uint8_t *health, double *t);
/* Overwrite state (u, u_prev, health may be NULL to keep). */
int pxb_epf_set_state(pxb_ctx *ctx, const double *u, const double *u_prev, const uint8_t *health, double t);
/* Number of broken bonds (health == 0). */
int pxb_epf_broken_count(pxb_ctx *ctx, long long *n_broken);

/* Bond-force adjoint with a frozen damage mask: given abar = dJ/da (N*dim) at the current u, returns
 * ubar = (da/du)^T abar (N*dim) and the derivatives of J with respect to C11, C12, C66 (dC[3]).  The
 * health mask is held fixed (no damage update). Device-pointer variant for torch. */
int pxb_epf_force_adjoint(pxb_ctx *ctx, const double *u, const double *abar, double *ubar, double *dC);
int pxb_epf_force_adjoint_d(pxb_ctx *ctx, const double *u_d, const double *abar_d, double *ubar_d, double *dC_d);
/* Adjoint of the explicit loop with the damage mask frozen at the current health (device pointers, N*dim each):
 * the forward is the loop of pxb_epf_start + pxb_epf_advance from (u0, v0) (v0 may be NULL) over nsteps steps of dt,
 * with the context's BC program after every step and no bond breaking.  Given ubar_N = dJ/du^N and ubar_Nm1 =
 * dJ/du^{N-1} (may be NULL: 0), returns u0bar = dJ/du0, v0bar = dJ/dv0 (may be NULL) and dC = dJ/d(C11, C12, C66)
 * (3 doubles, may be NULL).  The reverse sweep runs on the device: per step the transpose of the BC pass, then one
 * kernel for the bond-force adjoint fused with the central difference's transpose (the reverse bonds' operators come
 * from a bond-ordered copy built on first use, as large as the operator cache; without room for it they are
 * gathered).  The forward states it needs are kept every checkpoint_every steps and the others recomputed
 * (<= 0 or >= nsteps: every state kept, nsteps * N * dim doubles, nothing recomputed).  Leaves the context's
 * explicit state unchanged.  pxb_epf_adjoint_d = pxb_epf_record_d + pxb_epf_adjoint_recorded_d.  No counterpart
 * in the reference. */
int pxb_epf_adjoint_d(pxb_ctx *ctx, const double *u0_d, const double *v0_d, double dt, int nsteps, int checkpoint_every,
                      const double *ubar_N_d, const double *ubar_Nm1_d, double *u0bar_d, double *v0bar_d,
                      double *dC_d);
/* The forward half on its own: runs the frozen-mask loop from (u0, v0), keeps its checkpoints (or every state) in the
 * context and returns u^N and u^{N-1} (either may be NULL).  A differentiable caller runs it as its forward pass and
 * pxb_epf_adjoint_recorded_d as its backward pass, so the loop is not run a second time. */
int pxb_epf_record_d(pxb_ctx *ctx, const double *u0_d, const double *v0_d, double dt, int nsteps, int checkpoint_every,
                     double *uN_d, double *uNm1_d);
/* The per-step rate call (pxb_epf_rate) with pinned host buffers and a staged schedule variant runs pipelined: u
 * goes up in node chunks, each chunk's kernel starts once the chunk's neighbours have arrived, and its acceleration
 * goes down while the next chunk computes.  chunks: -1 (default) one chunk per 96 Ki nodes, at most 4 (meshes under
 * 192 Ki nodes: one); 1 no pipelining; 2..8 that many chunks.  No counterpart in the reference. */
int pxb_epf_set_rate_chunks(pxb_ctx *ctx, int chunks);
/* The reverse sweep's bond-force adjoint kernel: 0 a kernel that streams both the forward and the reverse bonds'
 * operators; 1 the reverse-only kernel: the frozen mask's own-bond operator sums are formed once per sweep, dJ/dC
 * is summed over the reverse bonds, and one operator stream is read per step; 2, 3, 4 (and -1, the default: 4) the
 * reverse-only kernel with the tiles' ids, reverse health and node rows staged by bulk copies through a
 * shared-memory ring (bounded waits: a wait that runs out fails the sweep with PXB_ERR_CUDA) and each reverse
 * bond's source node gathered as one interleaved (u, adjoint) row, in three launch configurations (3D: 2, 1 or 3
 * reverse bonds a lane per pass at 16 lanes a node; 2D: 4, 4 or 8 lanes a node).  The reverse-only
 * kernels apply when every bond has its reverse (symmetric families); other meshes fall back to 0.  Results agree
 * to rounding.  No counterpart in the reference. */
int pxb_epf_set_adjoint_schedule(pxb_ctx *ctx, int schedule);
/* The reverse sweep of the last pxb_epf_record_d (PXB_ERR_STATE when there is none); arguments as pxb_epf_adjoint_d. */
int pxb_epf_adjoint_recorded_d(pxb_ctx *ctx, const double *ubar_N_d, const double *ubar_Nm1_d, double *u0bar_d,
                               double *v0bar_d, double *dC_d);
/* Force (rate) with a frozen mask, device pointers, no damage update: a = (L(u)+b)/rho. */
int pxb_epf_force_frozen_d(pxb_ctx *ctx, const double *u_d, double *a_d);
/* Replaces C11, C12, C66 and rho of the explicit element without rebuilding the g-functions (the packed
 * per-bond coefficients are recomputed; captured step graphs are dropped).  No counterpart in the reference,
 * which reads the constants from the element parameters (ExplicitPDDOFracElement.cpp:38-53); it serves
 * sweeps and finite-difference checks of d/dE. */
int pxb_epf_set_constants(pxb_ctx *ctx, double C11, double C12, double C66, double rho);

/* ---- explicit-state snapshot and schedule autotuning --------------------------------------------------------
 * Device-side copy of the explicit state (u, u_prev, health, t) and its restore. */
int pxb_epf_snapshot(pxb_ctx *ctx);
int pxb_epf_restore(pxb_ctx *ctx);
/* Schedule variants of the explicit kernel: 0-2 lane groups (lanes per node x bonds per lane per pass), 3-4
 * CSR-stream tiles, 5 and up TMA-staged tiles (time step only; the other modes of a staged variant run
 * variant 1).  pxb_epf_variant_count() gives their number.  pxb_epf_autotune times every variant that fits
 * for `steps` steps from a private copy of the current state (L2 flushed before each step), restores the
 * state, selects the fastest and caches the choice per problem signature (dim, precision, nodes, bonds,
 * largest family); use_cache=1 returns a cached choice without timing.  ms_per_variant (may be NULL;
 * pxb_epf_variant_count() entries) receives the mean step time of each variant, -1 for one that does not fit. */
int pxb_epf_variant_count(void);
int pxb_epf_autotune(pxb_ctx *ctx, int steps, size_t flush_bytes, int use_cache, int *best, float *ms_per_variant);
/* The same for the per-step rate call (pxb_epf_rate: damage, force, acceleration out) at the caller's
 * displacement u (host, N*dim): every fitting variant's kernel is timed over reps launches, the bond health and
 * counters are restored around them (the state is unchanged), and the choice is cached per signature.  Needs
 * pxb_epf_setup, not pxb_epf_start; the perix_cuda:: shim runs it once per problem at its first call. */
int pxb_epf_autotune_rate(pxb_ctx *ctx, const double *u, int reps, int use_cache, int *best, float *ms_per_variant);
int pxb_epf_set_variant(pxb_ctx *ctx, int variant);
int pxb_epf_get_variant(pxb_ctx *ctx, int *variant, int *lanes_per_node);

/* ---- batched clouds ----------------------------------------------------------------------------------------
 * Many independent node clouds (2D and 3D mixed, boundary-truncated families of uneven size) in one
 * concatenated numbering: cloud k owns nodes [node_off[k], node_off[k+1]); neigh_off is the CSR over all nodes
 * (neigh_off[N] bonds); neigh_id holds 1-based ids WITHIN the node's own cloud (the reference's per-mesh
 * convention, PDMeshData per cloud as in tests/ExplicitPDDOFracElementTests.cpp:35-64); coords3 is xyz per
 * node; delta / dx_char per cloud (PDOperators::calcAMatrixCompute, CalcPDOperators.cpp:108-226).
 * pxb_batch_gbuild builds the order-2 g-functions of every cloud (nop 5 in 2D, 9 in 3D) in one persistent
 * launch (or one per dimension, as the schedule says) and fails with PXB_ERR_DEGENERATE naming the cloud and
 * node of a degenerate family.  pxb_batch_apply computes all nop derivatives of a scalar field (N) per node:
 * out[out_off(k) + (i - node_off[k]) * nop + s], clouds back to back ([n_k][nop_k]; total length from
 * pxb_batch_info).  pxb_batch_get_ops returns one cloud's g-functions as double [nb_k][nop_k].
 * No single counterpart in the reference, which builds and applies one mesh at a time. */
int pxb_batch_set(pxb_ctx *ctx, int nclouds, const int *dims, const int *node_off, const double *coords3,
                  const double *vols, const int *neigh_off, const int *neigh_id, const double *delta,
                  const double *dx_char);
/* The same with every cloud's families built on the device (reference order, as pxb_set_geometry_points;
 * radius[k] is cloud k's family radius); pxb_batch_get_families copies one cloud's families out (1-based ids
 * within the cloud). */
int pxb_batch_set_points(pxb_ctx *ctx, int nclouds, const int *dims, const int *node_off, const double *coords3,
                         const double *vols, const double *radius, const double *delta, const double *dx_char);
int pxb_batch_get_families(pxb_ctx *ctx, int cloud, int *neigh_off, int *neigh_id);
int pxb_batch_info(pxb_ctx *ctx, long long *nodes, long long *bonds, long long *out_len, long long *ops_len);
int pxb_batch_gbuild(pxb_ctx *ctx, int precision, int *n_degenerate, int *first_degenerate);
int pxb_batch_apply(pxb_ctx *ctx, const double *u, double *out);
int pxb_batch_apply_d(pxb_ctx *ctx, const double *u_d, double *out_d);
int pxb_batch_get_ops(pxb_ctx *ctx, int cloud, double *ops);
/* Schedules (which 0: g-build, 1: apply): lanes per node for 2D and 3D clouds and one launch for both
 * dimensions or one per dimension; pxb_batch_variant_count() of each.  pxb_batch_autotune times every schedule
 * (`reps` launches, L2 flushed before each; the apply on device buffers u_d -> out_d) and keeps the fastest. */
int pxb_batch_variant_count(void);
int pxb_batch_set_variant(pxb_ctx *ctx, int which, int variant);
int pxb_batch_get_variant(pxb_ctx *ctx, int which, int *variant);
int pxb_batch_autotune(pxb_ctx *ctx, int what, int reps, size_t flush_bytes, const double *u_d, double *out_d,
                       int *best, float *ms_per_variant);

/* ---- CSR Jacobian value assembly ---------------------------------------------------------------------------
 * Sets the matrix pattern (from pxb_csr_pattern or the caller) and precomputes the bond -> CSR-slot map
 * on the device (no binary search per assembly). */
int pxb_csr_set_pattern(pxb_ctx *ctx, int ndof, const int *rowptr, const int *cols, long long nnz);
/* Builds the pattern pxb_csr_pattern computes (SparseMatrix::initFromPDMesh, src/MathUtils/SparseMatrix.cpp:73-185:
 * per node {i} u family u {mirror}, sorted, unique, ndof x ndof blocks) on the device from the context's families
 * and mirror map, and sets it as pxb_csr_set_pattern does; *nnz gets its size.  Node lists longer than 256 give
 * PXB_ERR_UNSUPPORTED.  pxb_csr_get_pattern copies the context's pattern to host arrays (rows + 1 and nnz ints). */
int pxb_csr_build_pattern(pxb_ctx *ctx, int ndof, long long *nnz);
int pxb_csr_get_pattern(pxb_ctx *ctx, int *rowptr, int *cols);
/* Poisson (type 0) / transient diffusion (type 1) residual + Jacobian with K = -dF/dU, RHS = +F (reference
 * PoissonElement.cpp:26-58, DiffusionElement, FormResidualAndJacobianParallel.cpp:114-171).  f_node: per-node
 * source (N) or NULL to use the constant f. uold may be NULL when dt == 0. */
int pxb_assemble_scalar(pxb_ctx *ctx, int type, double coef, double f, const double *f_node, double dt,
                        const double *u, const double *uold, double *kvals, double *rhs);
int pxb_assemble_scalar_d(pxb_ctx *ctx, int type, double coef, double f, const double *f_node_d, double dt,
                          const double *u_d, const double *uold_d, double *kvals_d, double *rhs_d);

/* Conservative Cahn-Hilliard (2 dof) assembly from a host-built lambda-corrected Laplacian lapbond[nbtot],
 * reverse-bond map rev[nbtot], ghost flags and Picard-frozen mobility (reference
 * src/PDSystem/CudaAssembleKernels.cu:1277-1323 boundary; physics CahnHilliardElement.cpp:178-292). */
int pxb_ch_set_geometry(pxb_ctx *ctx, const int *rev, const double *lapbond, const char *isghost);
/* The same geometry built on the device from the order-2 operator cache (the one-off part of
 * CahnHilliardElement::preprocessIteration, CahnHilliardElement.cpp:93-152): lapbond = g_xx + g_yy (+ g_zz),
 * times lambda = 2 dim / sum_j g2_ij (|x_j|^2 - |x_i|^2) on bonds to non-ghost nodes; rev = reverse-bond index
 * (0-based, -1 when absent); isghost from the mirror map.  pxb_ch_get_geometry reads them back. */
int pxb_ch_build_geometry(pxb_ctx *ctx);
int pxb_ch_get_geometry(pxb_ctx *ctx, int *rev, double *lapbond, char *isghost);
/* Picard-frozen mobility M(c) = M0 c (1 - c), c = u[2i] clamped to [1e-8, 1 - 1e-8] (CahnHilliardElement.cpp:45-50),
 * and the assembly on device buffers (no host copies). */
int pxb_ch_mobility_d(pxb_ctx *ctx, double M0, const double *u_d, double *mnode_d);
int pxb_assemble_ch_d(pxb_ctx *ctx, double kappa, double chi, double dt, const double *mnode_d, const double *u_d,
                      const double *uold_d, double *kvals_d, double *rhs_d);
int pxb_assemble_ch(pxb_ctx *ctx, double kappa, double chi, double dt, const double *mnode, const double *u,
                    const double *uold, double *kvals, double *rhs);

/* Implicit Cahn-Hilliard run on the device (spinodal decomposition end to end) and its adjoint.  Backward Euler with the
 * reference's transient CH solve per step: Newton on the conservative element's residual with the mobility
 * M0 c (1 - c) frozen per iteration at the current iterate (CahnHilliardElement.cpp:66-292), zero-Neumann ghost
 * rows as NeumannBC::apply (NeumannBC.cpp:127-150), each linear system solved on the device (BiCGStab, 2x2
 * block-Jacobi).  Needs a 2D geometry (mirror ghosts for the Neumann walls), an FP64 order-2 g-build, the CH
 * geometry (pxb_ch_build_geometry) and a 2-dof pattern holding the mirror columns.  c0[n]: initial c (ghost entries
 * are replaced by their mirror bulk values), mu0 = 0.  E = total free energy of the final state, the sum over bulk
 * nodes of V_i (f(c_i) + kappa/2 |grad c_i|^2), f(c) = c ln c + (1 - c) ln(1 - c) + chi c (1 - c), grad c the PDDO
 * first derivatives.  pxb_ch_gradient also returns dE/dkappa and dE/dc0 (bulk entries; ghost entries 0) by the
 * discrete adjoint of the converged steps (the mobility derivative the Picard Jacobian omits included); it keeps
 * every step's state on the device (2 n (nsteps + 1) doubles).  No counterpart in the reference (it has no GPU
 * solver and no gradient). */
typedef struct pxb_ch_run_params {
    double chi, kappa, M0, dt;
    int nsteps;
    double newton_rtol; /* stop when |F| <= newton_rtol |F| of the step's initial guess */
    int newton_max;
    double lin_rtol; /* BiCGStab relative residual */
    int lin_max;
} pxb_ch_run_params;
typedef struct pxb_ch_run_stats {
    int steps, newton_iters, lin_iters;
    double max_residual;   /* largest final relative Newton residual */
    double max_lin_relres; /* largest final BiCGStab relative residual */
    double energy;
} pxb_ch_run_stats;
int pxb_ch_run(pxb_ctx *ctx, const pxb_ch_run_params *p, const double *c0, double *u_final, double *E,
               pxb_ch_run_stats *stats);
int pxb_ch_gradient(pxb_ctx *ctx, const pxb_ch_run_params *p, const double *c0, double *E, double *dE_dkappa,
                    double *dE_dc0, pxb_ch_run_stats *stats);
/* E of u (2n, rows c, mu) and dE/du (may be NULL) */
int pxb_ch_energy(pxb_ctx *ctx, double kappa, double chi, const double *u, double *E, double *dE_du);

/* Stress-coupled (optionally fracturing) Cahn-Hilliard assembly, the boundary of the reference's
 * perix_cuda::assembleStressCahnHilliard (include/PDSystem/CudaAssemble.h:185-191; kernel
 * src/PDSystem/CudaAssembleKernels.cu:685-874).  Rows per node: c, mu, u_x, u_y[, u_z] (ndof = dim + 2).
 * Needs an FP64 order-2 g-build, the CH geometry (pxb_ch_set_geometry / pxb_ch_build_geometry) and a pattern
 * set with ndof = dim + 2.  health[nbtot] (may be NULL: every bond intact) gates the mechanical bond terms by
 * 1 or kres; vel[n*dim] (may be NULL) with rho > 0 adds the backward-Euler inertia on the u rows; uold may be
 * NULL (c_old = u_old = 0).  K = -dF/dU, rhs = +F; rows of degenerate nodes are zero. */
typedef struct pxb_stress_ch_params {
    double C11, C12, C66;  /* elastic stiffness */
    double A, Kh, Ch;      /* chemo-mechanical body force -A grad c; hydrostatic stress Kh tr(eps) + Ch (c - cref) */
    double Omega, cref;    /* swelling */
    double chi, kappa;     /* regular-solution interaction, gradient energy */
    double dt;             /* backward-Euler step */
    double kres;           /* stiffness floor of a broken bond */
    double rho;            /* > 0: inertia on the displacement rows */
} pxb_stress_ch_params;
int pxb_assemble_stress_ch_d(pxb_ctx *ctx, const pxb_stress_ch_params *p, const double *mnode_d,
                             const double *health_d, const double *vel_d, const double *u_d, const double *uold_d,
                             double *kvals_d, double *rhs_d);
int pxb_assemble_stress_ch(pxb_ctx *ctx, const pxb_stress_ch_params *p, const double *mnode, const double *health,
                           const double *vel, const double *u, const double *uold, double *kvals, double *rhs);

/* Implicit PDDO dynamic fracture, the boundary of the reference's perix_cuda::assembleCached
 * (include/PDSystem/CudaAssemble.h:216-219; kernel src/PDSystem/CudaAssembleKernels.cu:880-1024; physics
 * PDDODynamicFracElement.cpp:207-306).  Rows per node: u (ndof = dim).  Needs an FP64 order-2 g-build and a
 * pattern set with ndof = dim.  nodecache[i*ncache + a] = committed velocity (may be NULL: zero), bondcache
 * [t*nbcache] = frozen bond health (may be NULL: every bond 1; a bond with health <= 0 carries nothing); uold may
 * be NULL.  R = b - rho (u - u_old - v dt)/dt^2 + sum of health-scaled Navier bond terms; K = -dF/dU. */
typedef struct pxb_cached_params {
    double C11, C12, C66;  /* elastic stiffness */
    double rho, dt;        /* density, backward-Euler step */
    double b[3];           /* body force */
} pxb_cached_params;
int pxb_assemble_cached_d(pxb_ctx *ctx, const pxb_cached_params *p, const double *nodecache_d, int ncache,
                          const double *bondcache_d, int nbcache, const double *u_d, const double *uold_d,
                          double *kvals_d, double *rhs_d);
int pxb_assemble_cached(pxb_ctx *ctx, const pxb_cached_params *p, const double *nodecache, int ncache,
                        const double *bondcache, int nbcache, const double *u, const double *uold, double *kvals,
                        double *rhs);

#ifdef __cplusplus
}
#endif
#endif
