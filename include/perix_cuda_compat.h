/* Source-compatible replacement for PeriX's CUDA-assembly boundary (reference include/PDSystem/CudaAssemble.h,
 * namespace perix_cuda).  A PeriX build that lists this backend's sources in place of the reference's
 * PERIX_CUDA_ASSEMBLY_SOURCES (reference cmake/PeriXSources.cmake:106-109) compiles unchanged: the structs
 * carry the same members in the same order and the functions keep their signatures, because the reference's
 * callers (FormResidualAndJacobianCUDA.cpp, ExplicitPDDOFracElement.cpp:174-235) fill and pass exactly these.
 *
 * Behavioural differences, by design:
 *   - there is no CPU fallback inside the backend: a device failure prints the reason to stderr and returns
 *     false, which is where the reference's callers take their CPU path; a build that must never run on the CPU
 *     replaces that branch by an abort;
 *   - a per-node horizon (AssembleMesh::nodeHorizon / nodeSpacing) is honoured by every entry: the g-build uses
 *     node i's own horizon and spacing, and the explicit element breaks each bond at s_c(0.5 (delta_i + delta_j))
 *     computed from ExplicitPDDOFracParams::G0, E and plane_stress;
 *   - assembleExplicitPDDOFracAccel times its schedules once per problem at its first call and keeps FP64
 *     operators unless the environment sets PERIX_B200_PRECISION=mixed.
 * The device work runs on a lazily created default pxb_ctx (device 0), freed by shutdown().
 */
#pragma once

namespace perix_cuda {

/* element kinds with a device port (reference CudaAssemble.h:24-27) */
enum AssembleElmtType {
    ELMT_POISSON = 0,
    ELMT_DIFFUSION = 1
};

/* 0-based operator slots of the derivatives the kernels read; -1 when absent (CudaAssemble.h:34-44) */
struct OpSlots {
    int dx = -1, dy = -1, dz = -1;
    int dxx = -1, dxy = -1, dyy = -1;
    int dxz = -1, dyz = -1, dzz = -1;
};

/* per-element parameters (CudaAssemble.h:47-54) */
struct ElmtParams {
    int type = ELMT_POISSON;
    int ndof = 1;
    int dim = 2;
    double sigma = 0.0, f = 0.0;
    double D = 0.0;
    double dt = 0.0;
};

/* read-only mesh + multi-index tables (CudaAssemble.h:61-80) */
struct AssembleMesh {
    int N = 0;
    int nnz = 0;
    const int *csr_off = nullptr;
    const int *csr_col = nullptr;
    const int *neigh_off = nullptr;
    const int *neigh_id = nullptr;
    const double *coords = nullptr;
    const double *vols = nullptr;
    const int *qp = nullptr;
    const int *qq = nullptr;
    const int *qr = nullptr;
    const double *factprod = nullptr;
    int nop = 0;
    int dim = 2;
    double delta = 0.0;
    double dx_char = 0.0;
    const double *nodeHorizon = nullptr;
    const double *nodeSpacing = nullptr;
};

bool assemble(const AssembleMesh &m, const ElmtParams &p, const OpSlots &s,
              const double *u, const double *uold,
              double *out_Kvals, double *out_rhs);

/* conservative Cahn-Hilliard (CudaAssemble.h:100-142) */
struct CahnHilliardParams {
    double kappa = 0.0;
    double chi = 0.0;
    double dt = 1.0;
};

struct CahnHilliardMesh {
    int N = 0, nbtot = 0;
    const int *off = nullptr;
    const int *nbr = nullptr;
    const int *rev = nullptr;
    const double *lapbond = nullptr;
    const double *vol = nullptr;
    const char *isghost = nullptr;
    const double *mnode = nullptr;
};

bool assembleCahnHilliard(const CahnHilliardMesh &m, const CahnHilliardParams &p,
                          const int *csr_off, const int *csr_col, int nnz,
                          const double *u, const double *uold,
                          double *out_Kvals, double *out_rhs);

/* stress-coupled Cahn-Hilliard (CudaAssemble.h:150-191) */
struct StressCahnHilliardParams {
    int dim = 2, ndof = 4;
    double C11 = 0.0, C12 = 0.0, C66 = 0.0;
    double A = 0.0, Kh = 0.0, Ch = 0.0;
    double Omega = 0.0, cref = 0.0;
    double chi = 0.0, kappa = 0.0;
    double dt = 1.0;
    double kres = 1.0e-8;
    double rho = 0.0;
};

bool assembleStressCahnHilliard(const AssembleMesh &m, const StressCahnHilliardParams &p,
                                const OpSlots &s,
                                const int *rev, const double *lapbond,
                                const char *isghost, const double *mnode,
                                const double *health, const double *vel,
                                const double *u, const double *uold,
                                double *out_Kvals, double *out_rhs);

/* implicit dynamic fracture (CudaAssemble.h:194-219) */
struct CachedParams {
    int ndof = 2;
    int dim = 2;
    int ncache = 3;
    double dt = 0.0;
    double C11 = 0.0, C12 = 0.0, C66 = 0.0;
    double rho = 0.0;
    double bx = 0.0, by = 0.0, bz = 0.0;
    int nbcache = 1;
};

bool assembleCached(const AssembleMesh &m, const CachedParams &p, const OpSlots &s,
                    const double *nodecache, const double *bondcache,
                    const double *u, const double *uold,
                    double *out_Kvals, double *out_rhs);

/* explicit strong-form PDDO fracture (CudaAssemble.h:225-254) */
struct ExplicitPDDOFracParams {
    int dim = 2;
    double C11 = 0.0, C12 = 0.0, C66 = 0.0;
    double rho = 1.0;
    double bx = 0.0, by = 0.0, bz = 0.0;
    double sc = 0.0;
    int tension_only = 1, damage_on = 1;
    int plane_stress = 0;
    double G0 = 0.0, E = 0.0;
};

/* One acceleration evaluation: damage at u then force, a=(L+b)/rho (N*dim).  health_inout (nbtot, 1.0/0.0)
 * is uploaded on the first call (or after a size change), evolved on the device, and copied back only when
 * a bond broke (*health_changed = 1). */
bool assembleExplicitPDDOFracAccel(const AssembleMesh &m, const ExplicitPDDOFracParams &p,
                                   const OpSlots &s, const double *u,
                                   double *health_inout, double *accel_out,
                                   int *health_changed);

void shutdown();

}  // namespace perix_cuda
