// Test infrastructure only: a C-callable harness around the reference's OWN hot-path code, linked from the
// reference sources by oracle/Makefile into oracle/_ref/libperix_ref.so.  Only tests/, the smoke check and
// the bench's CPU-baseline / reference arm load it.  Nothing in the product links or calls it.
//
// Every value this harness returns is computed by reference code:
//   structured PD mesh      Lagrange2DQuad4/3DHex8 generators + PDMesh::createPDMesh (CreatePDMesh.cpp:30)
//   families                PDMesh::createNeighborNodes                              (CreatePDMesh.cpp:910)
//   g-functions             PDOperators::calcAMatrix / calcOperators                  (CalcPDOperators.cpp:85,245)
//   g-build timing          PDOperators::buildGeometryCache                           (CalcPDOperators.cpp:356)
//   CSR pattern             SparseMatrix::initFromPDMesh                              (SparseMatrix.cpp:73)
//   Poisson assembly        PoissonElement bond callback in the loop of
//                           PDSystem::formResidualAndJacobianParallel                 (FormResidualAndJacobianParallel.cpp:102-172)
//   explicit fracture rate  ExplicitPDDOFracElement::preprocessIteration              (ExplicitPDDOFracElement.cpp:85)
//   stress-coupled CH       StressCahnHilliardElement preprocess + nodal/bond callbacks (StressCahnHilliardElement.cpp:139-466)
//   implicit dyn. fracture  PDDODynamicFracElement preprocess (init + one commit) + callbacks (PDDODynamicFracElement.cpp:82-306)
//   ghost BC preset         DirichletBC::presetSolutionAtTime / NeumannBC::presetSolution, applied in list
//                           order like BCSystem::presetSolution                       (DirichletBC.cpp:107-147,
//                                                                                      NeumannBC.cpp:88-105,
//                                                                                      BCSystem.cpp:114-129)
//   scalar system assembly  PDSystem::formResidualAndJacobian with a registered PoissonElement or
//                           DiffusionElement                                          (FormResidualAndJacobian.cpp)
// The central-difference loop is a short restatement of TimeStepping.cpp:479-547 (that translation unit pulls in
// the whole run-time system).
//
// Built a second time with -DPERIX_CUDA_ASSEMBLE into oracle/_ref/libperix_ref_dropin.so, together with the
// reference's own callers of the CUDA-assembly boundary (PDSystem::formResidualAndJacobianCUDA and
// ExplicitPDDOFracElement's UseCuda branch, compiled unchanged against a forwarding PDSystem/CudaAssemble.h) and
// linked to libperix_b200.so: ref_system_assemble(..., use_cuda=1) and ref_epf_use_cuda then run the reference's
// callers through this backend's perix_cuda:: shim.

#include <algorithm>
#include <array>
#include <chrono>
#include <cmath>
#include <cstring>
#include <limits>
#include <memory>
#include <string>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

// The harness reads two private members (the element's flat health/op cache and the operator object's
// degenerate flag).  Access specifiers do not change GCC's class layout, so this only widens visibility.
#define private public
#include "ElmtSystem/ExplicitPDDOFracElement.h"
#include "PDOperators/PDOperators.h"
#undef private
#include "BCSystem/DirichletBC.h"
#include "BCSystem/NeumannBC.h"
#include "ElmtSystem/CahnHilliardElement.h"
#include "ElmtSystem/DiffusionElement.h"
#include "ElmtSystem/ElmtSystem.h"
#include "ElmtSystem/PDDODynamicFracElement.h"
#include "ElmtSystem/PoissonElement.h"
#include "PDSystem/PDSystem.h"
#include "ElmtSystem/StressCahnHilliardElement.h"
#include "MathUtils/SparseMatrix.h"
#include "Mesh/MeshGenerator.h"
#include "PDMesh/PDMesh.h"

namespace {

struct RefMesh {
    MeshData md;
    PDMesh pd;
    PDOperators ops;
    int dim = 2;
    int order = 2;
};

struct RefEpf {
    ExplicitPDDOFracElement el;
    RefMesh *mesh = nullptr;
    bool use_cuda = false;  // LocalElmtInfo::UseCuda of the rate calls (drop-in build only)
};

void setupOps(RefMesh *m) {
    m->ops.setDim(m->dim);
    m->ops.setOrder(m->order);
    m->ops.setup();
}

}  // namespace

extern "C" {

// ---- meshes ---------------------------------------------------------------------------------------------
// Structured lattice exactly as a deck's Mesh{type:quad4/hex8,nx,ny,nz,xmin..} + PDMesh block builds it.
void *ref_mesh_structured(int dim, int nx, int ny, int nz, const double *box /*xmin,xmax,ymin,ymax,zmin,zmax*/,
                          double horizon_factor, int order, int force_only, int ncracks, const double *cracks,
                          int nplanes, const double *planes) {
    auto *m = new RefMesh();
    m->dim = dim;
    m->order = order;
    m->md.Nx = nx;
    m->md.Ny = ny;
    m->md.Nz = (dim == 3) ? nz : 0;
    m->md.Xmin = box[0]; m->md.Xmax = box[1];
    m->md.Ymin = box[2]; m->md.Ymax = box[3];
    m->md.Zmin = (dim == 3) ? box[4] : 0.0;
    m->md.Zmax = (dim == 3) ? box[5] : 0.0;
    m->md.MeshDim = dim;
    m->md.BulkMeshTypeName = (dim == 3) ? "hex8" : "quad4";
    MeshGenerator gen;
    if (dim == 3) gen.Lagrange3DHex8MeshGenerator::generateMesh(m->md);
    else gen.Lagrange2DQuad4MeshGenerator::generateMesh(m->md);
    m->pd.createPDMesh(m->md);
    const auto &d = m->pd.getDataConstRef();
    m->pd.setHorizonRadiusFromFactor(horizon_factor, d.DX);
    for (int c = 0; c < ncracks; ++c)
        m->pd.addCrack(cracks[4 * c + 0], cracks[4 * c + 1], cracks[4 * c + 2], cracks[4 * c + 3]);
    for (int c = 0; c < nplanes; ++c) {
        const double *q = planes + 12 * c;
        m->pd.addCrackPlane({q[0], q[1], q[2]}, {q[3], q[4], q[5]}, {q[6], q[7], q[8]}, {q[9], q[10], q[11]});
    }
    m->pd.setForceOnlyCracks(force_only != 0);
    m->pd.createNeighborNodes();
    setupOps(m);
    return m;
}

// Free point cloud (no ghosts) built the way the reference tests build PDMeshData by hand
// (tests/ExplicitPDDOFracElementTests.cpp:35-64): coords/vols given, horizon set through the margin setter.
void *ref_mesh_cloud(int dim, int n, const double *coords3, const double *vols, double dx, double dy, double dz,
                     double horizon_radius_no_margin, int order, int volume_correction) {
    auto *m = new RefMesh();
    m->dim = dim;
    m->order = order;
    auto &d = m->pd.getDataRef();
    d.NodesNum = n;
    d.BulkElmtsNum = n;
    d.DX = dx; d.DY = dy; d.DZ = (dim == 3) ? dz : 0.0;
    d.NodeCoords.assign(coords3, coords3 + 3 * (size_t)n);
    d.NodeVolumes.assign(vols, vols + n);
    d.VolumeCorrection = volume_correction != 0;
    m->pd.setHorizonRadius(horizon_radius_no_margin);
    m->pd.createNeighborNodes();
    setupOps(m);
    return m;
}

// The same free cloud with the reference's variable horizon on (PDMeshData::VariableHorizon): every node is a bulk
// node (NodesElmtID = 1), PDMesh::computeVariableHorizon sets NodeHorizon / NodeSpacing from the volumes, then
// createNeighborNodes builds the dual families.
void *ref_mesh_cloud_vh(int dim, int n, const double *coords3, const double *vols, double dx, double dy, double dz,
                        double horizon_radius_no_margin, int order, int volume_correction) {
    auto *m = new RefMesh();
    m->dim = dim;
    m->order = order;
    auto &d = m->pd.getDataRef();
    d.NodesNum = n;
    d.BulkElmtsNum = n;
    d.DX = dx; d.DY = dy; d.DZ = (dim == 3) ? dz : 0.0;
    d.NodeCoords.assign(coords3, coords3 + 3 * (size_t)n);
    d.NodeVolumes.assign(vols, vols + n);
    d.NodesElmtID.assign((size_t)n, 1);
    d.VolumeCorrection = volume_correction != 0;
    m->pd.setHorizonRadius(horizon_radius_no_margin);
    m->pd.setVariableHorizon(true);
    m->pd.computeVariableHorizon();
    m->pd.createNeighborNodes();
    setupOps(m);
    return m;
}

// NodeHorizon / NodeSpacing of the mesh (n each; zeros when the variable horizon is off)
void ref_mesh_node_horizon(void *h, double *delta, double *spacing) {
    const auto &d = static_cast<RefMesh *>(h)->pd.getDataConstRef();
    for (int i = 0; i < d.NodesNum; ++i) {
        delta[i] = d.NodeHorizon.empty() ? 0.0 : d.NodeHorizon[(size_t)i];
        spacing[i] = d.NodeSpacing.empty() ? 0.0 : d.NodeSpacing[(size_t)i];
    }
}

void ref_mesh_free(void *h) { delete static_cast<RefMesh *>(h); }

int ref_mesh_nodes(void *h) { return static_cast<RefMesh *>(h)->pd.getNodesNum(); }

long long ref_mesh_bonds(void *h) {
    long long nb = 0;
    for (const auto &f : static_cast<RefMesh *>(h)->pd.getDataConstRef().NodesNeighNodesID) nb += (long long)f.size();
    return nb;
}

// scalars[0..5] = HorizonRadius, DX, DY, DZ, dx_char=max(DX,DY,DZ), nop
void ref_mesh_scalars(void *h, double *out) {
    auto *m = static_cast<RefMesh *>(h);
    const auto &d = m->pd.getDataConstRef();
    out[0] = d.HorizonRadius;
    out[1] = d.DX; out[2] = d.DY; out[3] = d.DZ;
    out[4] = std::max(d.DX, std::max(d.DY, d.DZ));
    out[5] = m->ops.getOperatorsVecSize();
}

void ref_mesh_get(void *h, double *coords3, double *vols, int *off, int *ids1, int *mirror) {
    auto *m = static_cast<RefMesh *>(h);
    const auto &d = m->pd.getDataConstRef();
    const int n = d.NodesNum;
    if (coords3) std::memcpy(coords3, d.NodeCoords.data(), sizeof(double) * 3 * (size_t)n);
    if (vols) std::memcpy(vols, d.NodeVolumes.data(), sizeof(double) * (size_t)n);
    if (off) {
        off[0] = 0;
        for (int i = 0; i < n; ++i) off[i + 1] = off[i] + (int)d.NodesNeighNodesID[i].size();
    }
    if (ids1) {
        size_t p = 0;
        for (int i = 0; i < n; ++i)
            for (int j : d.NodesNeighNodesID[i]) ids1[p++] = j;
    }
    if (mirror) {
        for (int i = 0; i < n; ++i)
            mirror[i] = (i < (int)d.GhostMirrorBulkID.size()) ? d.GhostMirrorBulkID[i] : 0;
    }
}

int ref_group_size(void *h, const char *name) {
    return (int)static_cast<RefMesh *>(h)->pd.getNodeIDsViaPhyName(name).size();
}

void ref_group_get(void *h, const char *name, int *ids1) {
    const auto &v = static_cast<RefMesh *>(h)->pd.getNodeIDsViaPhyName(name);
    std::copy(v.begin(), v.end(), ids1);
}

int ref_crack_cuts(void *h, int i1, int j1) { return static_cast<RefMesh *>(h)->pd.initialCrackCutsBond(i1, j1) ? 1 : 0; }

// ---- multi-index table -----------------------------------------------------------------------------------
void ref_qindices(void *h, int *pqr /*nop*3*/, int *factprod) {
    auto *m = static_cast<RefMesh *>(h);
    const auto &q = m->ops.getQIndices();
    auto fact = [](int n) { int r = 1; for (int k = 2; k <= n; ++k) r *= k; return r; };
    for (size_t k = 0; k < q.size(); ++k) {
        pqr[3 * k + 0] = q[k][0]; pqr[3 * k + 1] = q[k][1]; pqr[3 * k + 2] = q[k][2];
        if (factprod) factprod[k] = fact(q[k][0]) * fact(q[k][1]) * fact(q[k][2]);
    }
}

// ---- g-functions (full nop vector per bond, family order, [bond*nop+k]) -------------------------------------
// degenerate[i] = 1 where calcAMatrixCompute flagged the family (usable<nop or inconsistent system).
void ref_gbuild(void *h, double *ops_out, unsigned char *degenerate, int nthreads) {
    auto *m = static_cast<RefMesh *>(h);
    const auto &d = m->pd.getDataConstRef();
    const int n = d.NodesNum;
    const int nop = m->ops.getOperatorsVecSize();
    std::vector<long long> off(n + 1, 0);
    for (int i = 0; i < n; ++i) off[i + 1] = off[i] + (long long)d.NodesNeighNodesID[i].size();
#pragma omp parallel num_threads(nthreads > 0 ? nthreads : 1)
    {
        PDOperators local = m->ops;
        local.setAbortOnDegenerate(false);
#pragma omp for schedule(guided)
        for (int i = 1; i <= n; ++i) {
            local.calcAMatrix(i, d);
            if (degenerate) degenerate[i - 1] = local.m_LastFamilyDegenerate ? 1 : 0;
            const auto &fam = d.NodesNeighNodesID[i - 1];
            for (size_t t = 0; t < fam.size(); ++t) {
                local.calcOperators(i, fam[t], d);
                for (int k = 0; k < nop; ++k)
                    ops_out[(off[i - 1] + (long long)t) * nop + k] = local.getOperatorValue(k + 1);
            }
        }
    }
}

// Wall time (s) of the reference's own cache build, best of `reps`.
double ref_gbuild_time(void *h, int nthreads, int reps) {
    auto *m = static_cast<RefMesh *>(h);
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#endif
    double best = 1e300;
    for (int r = 0; r < reps; ++r) {
        PDOperators o = m->ops;
        auto t0 = std::chrono::steady_clock::now();
        o.buildGeometryCache(m->pd.getDataConstRef(), 64.0);
        auto t1 = std::chrono::steady_clock::now();
        best = std::min(best, std::chrono::duration<double>(t1 - t0).count());
    }
    return best;
}

// ---- family-sum derivative apply D^k u_i = sum_j g^k_ij (u_j - u_i), all nop derivatives --------------------
void ref_apply(void *h, const double *u, double *out /*N*nop*/, int nthreads) {
    auto *m = static_cast<RefMesh *>(h);
    const auto &d = m->pd.getDataConstRef();
    const int n = d.NodesNum;
    const int nop = m->ops.getOperatorsVecSize();
#pragma omp parallel num_threads(nthreads > 0 ? nthreads : 1)
    {
        PDOperators local = m->ops;
        local.setAbortOnDegenerate(false);
#pragma omp for schedule(guided)
        for (int i = 1; i <= n; ++i) {
            local.calcAMatrix(i, d);
            std::vector<double> acc(nop, 0.0);
            for (int j : d.NodesNeighNodesID[i - 1]) {
                local.calcOperators(i, j, d);
                const double du = u[j - 1] - u[i - 1];
                for (int k = 0; k < nop; ++k) acc[k] += local.getOperatorValue(k + 1) * du;
            }
            for (int k = 0; k < nop; ++k) out[(size_t)(i - 1) * nop + k] = acc[k];
        }
    }
}

// ---- CSR pattern ------------------------------------------------------------------------------------------
int ref_csr_nnz(void *h, int ndof) {
    SparseMatrix K;
    K.initFromPDMesh(static_cast<RefMesh *>(h)->pd.getDataConstRef(), ndof);
    return K.getNNZNum();
}

void ref_csr_pattern(void *h, int ndof, int *rowptr, int *cols) {
    SparseMatrix K;
    K.initFromPDMesh(static_cast<RefMesh *>(h)->pd.getDataConstRef(), ndof);
    const auto r = K.getCSRRowsIndexCopy();
    const auto c = K.getCSRColsIndexCopy();
    std::copy(r.begin(), r.end(), rowptr);
    std::copy(c.begin(), c.end(), cols);
}

// ---- Poisson residual/Jacobian (K=-dF/dU, RHS=+F) with a per-node source f_i --------------------------------
// The bond term is the reference PoissonElement callback; the nodal term is f_i (the reference element only
// takes a constant f; a per-node source is what the manufactured Poisson solution needs).  Accumulation order
// and signs follow FormResidualAndJacobianParallel.cpp:114-171.
double ref_poisson_assemble(void *h, double sigma, const double *fnode, const double *u, double *kvals,
                            double *rhs, int nthreads) {
    auto *m = static_cast<RefMesh *>(h);
    const auto &d = m->pd.getDataConstRef();
    const int n = d.NodesNum;
    SparseMatrix K;
    K.initFromPDMesh(d, 1);
    K.setToZeros();
    PoissonElement el(sigma, 0.0);
    el.setDim(m->dim);
    auto t0 = std::chrono::steady_clock::now();
    std::vector<double> r(n, 0.0);
#pragma omp parallel num_threads(nthreads > 0 ? nthreads : 1)
    {
        PDOperators ops = m->ops;
        ops.setAbortOnDegenerate(false);
        VectorXd R(1), UI(1), UJ(1), UoI(1), UoJ(1);
        MatrixXd KII(1, 1), KIJ(1, 1);
        LocalElmtInfo info;
#pragma omp for schedule(guided)
        for (int i = 1; i <= n; ++i) {
            ops.calcAMatrix(i, d);
            r[i - 1] += fnode ? fnode[i - 1] : 0.0;
            K.addValue(i, i, -0.0);
            UI(1) = u[i - 1];
            for (int j : d.NodesNeighNodesID[i - 1]) {
                ops.calcOperators(i, j, d);
                UJ(1) = u[j - 1];
                el.computeBondResidualAndJacobian(ops, info, i, j, UI, UJ, UoI, UoJ, d.NodeVolumes[i - 1], R, KII, KIJ);
                r[i - 1] += R(1);
                K.addValue(i, i, -KII(1, 1));
                K.addValue(i, j, -KIJ(1, 1));
            }
        }
    }
    auto t1 = std::chrono::steady_clock::now();
    std::memcpy(kvals, K.getCSRValuesPtr(), sizeof(double) * (size_t)K.getNNZNum());
    std::memcpy(rhs, r.data(), sizeof(double) * (size_t)n);
    return std::chrono::duration<double>(t1 - t0).count();
}

// ---- Cahn-Hilliard element (2 dof) ------------------------------------------------------------------------
// CahnHilliardElement::preprocessIteration (one-off lambda-corrected Laplacian, reverse bonds, ghost flags,
// then the Picard-frozen mobility) and its nodal/bond callbacks, accumulated like
// FormResidualAndJacobianParallel.cpp:100-172 (K = -dF/dU, RHS = +F, row-owned).  Returns the element's geometry
// (lapbond[nb], rev[nb] 0-based bond index or -1, isghost[n]) and mobility mnode[n] for the device assembler's
// inputs.  Wall time in seconds of the assembly loop.
double ref_ch_assemble(void *h, double chi, double kappa, double M0, double dt, const double *u, const double *uold,
                       double *kvals, double *rhs, double *lapbond, int *rev, char *isghost, double *mnode,
                       int nthreads) {
    auto *m = static_cast<RefMesh *>(h);
    const auto &d = m->pd.getDataConstRef();
    const int n = d.NodesNum;
    const int ndof = 2;
    CahnHilliardElement el;
    el.setDim(m->dim);
    el.setChi(chi);
    el.setKappa(kappa);
    el.setMobility(M0);
    VectorXd U(n * ndof), Uo(n * ndof);
    std::memcpy(U.getDataPtr(), u, sizeof(double) * (size_t)n * ndof);
    std::memcpy(Uo.getDataPtr(), uold, sizeof(double) * (size_t)n * ndof);
    LocalElmtInfo info;
    info.Dt = dt;
    info.UseParallel = nthreads != 1;
    PDOperators pops = m->ops;
    pops.setAbortOnDegenerate(false);
    el.preprocessIteration(m->pd, pops, info, ndof, U, Uo);
    SparseMatrix K;
    K.initFromPDMesh(d, ndof);
    K.setToZeros();
    std::vector<double> r((size_t)n * ndof, 0.0);
    auto t0 = std::chrono::steady_clock::now();
#pragma omp parallel num_threads(nthreads > 0 ? nthreads : 1)
    {
        PDOperators ops = m->ops;
        ops.setAbortOnDegenerate(false);
        VectorXd R(ndof), Rn(ndof), UI(ndof), UJ(ndof), UoI(ndof), UoJ(ndof);
        MatrixXd KII(ndof, ndof), KIJ(ndof, ndof), Kn(ndof, ndof);
#pragma omp for schedule(guided)
        for (int i = 1; i <= n; ++i) {
            ops.calcAMatrix(i, d);
            const int bi = (i - 1) * ndof;
            for (int a = 1; a <= ndof; ++a) {
                UI(a) = u[bi + a - 1];
                UoI(a) = uold[bi + a - 1];
            }
            el.computeNodalResidualAndJacobian(info, i, UI, UoI, d.NodeVolumes[i - 1], Rn, Kn);
            for (int a = 1; a <= ndof; ++a) {
                r[bi + a - 1] += Rn(a);
                for (int b = 1; b <= ndof; ++b) K.addValue(bi + a, bi + b, -Kn(a, b));
            }
            for (int j : d.NodesNeighNodesID[i - 1]) {
                ops.calcOperators(i, j, d);
                const int bj = (j - 1) * ndof;
                for (int a = 1; a <= ndof; ++a) {
                    UJ(a) = u[bj + a - 1];
                    UoJ(a) = uold[bj + a - 1];
                }
                el.computeBondResidualAndJacobian(ops, info, i, j, UI, UJ, UoI, UoJ, d.NodeVolumes[i - 1], R, KII, KIJ);
                for (int a = 1; a <= ndof; ++a) {
                    r[bi + a - 1] += R(a);
                    for (int b = 1; b <= ndof; ++b) {
                        K.addValue(bi + a, bi + b, -KII(a, b));
                        K.addValue(bi + a, bj + b, -KIJ(a, b));
                    }
                }
            }
        }
    }
    auto t1 = std::chrono::steady_clock::now();
    std::memcpy(kvals, K.getCSRValuesPtr(), sizeof(double) * (size_t)K.getNNZNum());
    std::memcpy(rhs, r.data(), sizeof(double) * r.size());
    const size_t nb = el.getLapBond().size();
    if (lapbond) std::memcpy(lapbond, el.getLapBond().data(), sizeof(double) * nb);
    if (rev) std::memcpy(rev, el.getRevBond().data(), sizeof(int) * nb);
    if (isghost)
        for (int i = 0; i < n; ++i) isghost[i] = el.getGhostFlags().empty() ? 0 : el.getGhostFlags()[(size_t)i];
    if (mnode) std::memcpy(mnode, el.getNodeMobility().data(), sizeof(double) * (size_t)n);
    return std::chrono::duration<double>(t1 - t0).count();
}

// Stress-coupled Cahn-Hilliard (ndof = dim + 2: c, mu, u): StressCahnHilliardElement's preprocessIteration and
// its nodal / bond callbacks accumulated as formResidualAndJacobianParallel does (K = -dF/dU, rhs = +F).
// consts[6] receives the element's derived C11, C12, C66, A, Kh, Ch; lapbond/rev/isghost/mnode its own arrays.
double ref_stress_ch_assemble(void *h, double E, double nu, int plane_stress, double Omega, double cref, double D,
                              double chi, double kappa, double dt, const double *u, const double *uold, double *kvals,
                              double *rhs, double *lapbond, int *rev, char *isghost, double *mnode, double *consts,
                              int nthreads) {
    auto *m = static_cast<RefMesh *>(h);
    const auto &d = m->pd.getDataConstRef();
    const int n = d.NodesNum;
    const int ndof = m->dim + 2;
    StressCahnHilliardElement el;
    el.setDim(m->dim);
    el.setE(E);
    el.setNu(nu);
    el.setState(plane_stress ? StressCahnHilliardElement::StressState::PlaneStress
                             : StressCahnHilliardElement::StressState::PlaneStrain);
    el.setOmega(Omega);
    el.setCref(cref);
    el.setDiffusivity(D);
    el.setChi(chi);
    el.setKappa(kappa);
    VectorXd U(n * ndof), Uo(n * ndof);
    std::memcpy(U.getDataPtr(), u, sizeof(double) * (size_t)n * ndof);
    std::memcpy(Uo.getDataPtr(), uold, sizeof(double) * (size_t)n * ndof);
    LocalElmtInfo info;
    info.Dt = dt;
    info.UseParallel = nthreads != 1;
    PDOperators pops = m->ops;
    pops.setAbortOnDegenerate(false);
    el.preprocessIteration(m->pd, pops, info, ndof, U, Uo);
    SparseMatrix K;
    K.initFromPDMesh(d, ndof);
    K.setToZeros();
    std::vector<double> r((size_t)n * ndof, 0.0);
    auto t0 = std::chrono::steady_clock::now();
#pragma omp parallel num_threads(nthreads > 0 ? nthreads : 1)
    {
        PDOperators ops = m->ops;
        ops.setAbortOnDegenerate(false);
        VectorXd R(ndof), Rn(ndof), UI(ndof), UJ(ndof), UoI(ndof), UoJ(ndof);
        MatrixXd KII(ndof, ndof), KIJ(ndof, ndof), Kn(ndof, ndof);
#pragma omp for schedule(guided)
        for (int i = 1; i <= n; ++i) {
            ops.calcAMatrix(i, d);
            const int bi = (i - 1) * ndof;
            for (int a = 1; a <= ndof; ++a) {
                UI(a) = u[bi + a - 1];
                UoI(a) = uold[bi + a - 1];
            }
            el.computeNodalResidualAndJacobian(info, i, UI, UoI, d.NodeVolumes[i - 1], Rn, Kn);
            for (int a = 1; a <= ndof; ++a) {
                r[bi + a - 1] += Rn(a);
                for (int b = 1; b <= ndof; ++b) K.addValue(bi + a, bi + b, -Kn(a, b));
            }
            for (int j : d.NodesNeighNodesID[i - 1]) {
                ops.calcOperators(i, j, d);
                const int bj = (j - 1) * ndof;
                for (int a = 1; a <= ndof; ++a) {
                    UJ(a) = u[bj + a - 1];
                    UoJ(a) = uold[bj + a - 1];
                }
                el.computeBondResidualAndJacobian(ops, info, i, j, UI, UJ, UoI, UoJ, d.NodeVolumes[i - 1], R, KII, KIJ);
                for (int a = 1; a <= ndof; ++a) {
                    r[bi + a - 1] += R(a);
                    for (int b = 1; b <= ndof; ++b) {
                        K.addValue(bi + a, bi + b, -KII(a, b));
                        K.addValue(bi + a, bj + b, -KIJ(a, b));
                    }
                }
            }
        }
    }
    auto t1 = std::chrono::steady_clock::now();
    std::memcpy(kvals, K.getCSRValuesPtr(), sizeof(double) * (size_t)K.getNNZNum());
    std::memcpy(rhs, r.data(), sizeof(double) * r.size());
    const size_t nb = el.getLapBond().size();
    if (lapbond) std::memcpy(lapbond, el.getLapBond().data(), sizeof(double) * nb);
    if (rev) std::memcpy(rev, el.getRevBond().data(), sizeof(int) * nb);
    if (isghost)
        for (int i = 0; i < n; ++i) isghost[i] = el.getGhostFlags().empty() ? 0 : el.getGhostFlags()[(size_t)i];
    if (mnode) std::memcpy(mnode, el.getNodeMobility().data(), sizeof(double) * (size_t)n);
    if (consts) {
        consts[0] = el.getC11();
        consts[1] = el.getC12();
        consts[2] = el.getC66();
        consts[3] = el.getCoupling();
        consts[4] = el.getKh();
        consts[5] = el.getCh();
    }
    return std::chrono::duration<double>(t1 - t0).count();
}

// Implicit PDDO dynamic fracture (ndof = dim): PDDODynamicFracElement initialised at step 1 from uprev, then
// committed at step 2 from uold (velocity (uold - uprev)/dt, bond failure by stretch at uold), then its nodal and
// bond callbacks at u accumulated as formResidualAndJacobianParallel does.  vel_out[n*dim] and health_out[nbtot]
// (family order) receive the committed velocity and health; consts[3] = C11, C12, C66.
double ref_dynfrac_assemble(void *h, double E, double nu, double rho, double G0, int plane_stress, int tension_only,
                            double bx, double by, double bz, double dt, const double *uprev, const double *uold,
                            const double *u, double *kvals, double *rhs, double *vel_out, double *health_out,
                            double *consts) {
    auto *m = static_cast<RefMesh *>(h);
    const auto &d = m->pd.getDataConstRef();
    const int n = d.NodesNum;
    const int ndof = m->dim;
    PDDODynamicFracElement el;
    el.setDim(m->dim);
    el.setE(E);
    el.setNu(nu);
    el.setRho(rho);
    el.setG0(G0);
    el.setState(plane_stress ? PDDODynamicFracElement::StressState::PlaneStress
                             : PDDODynamicFracElement::StressState::PlaneStrain);
    el.setTensionOnly(tension_only != 0);
    el.setDamageOn(true);
    el.setBodyForce(bx, by, bz);
    VectorXd U(n * ndof), Uo(n * ndof), Up(n * ndof);
    std::memcpy(U.getDataPtr(), u, sizeof(double) * (size_t)n * ndof);
    std::memcpy(Uo.getDataPtr(), uold, sizeof(double) * (size_t)n * ndof);
    std::memcpy(Up.getDataPtr(), uprev, sizeof(double) * (size_t)n * ndof);
    LocalElmtInfo info;
    info.Dt = dt;
    info.UseParallel = false;
    info.Timestep = 1;
    PDOperators pops = m->ops;
    pops.setAbortOnDegenerate(false);
    el.preprocessIteration(m->pd, pops, info, ndof, U, Up);
    info.Timestep = 2;
    el.preprocessIteration(m->pd, pops, info, ndof, U, Uo);
    SparseMatrix K;
    K.initFromPDMesh(d, ndof);
    K.setToZeros();
    std::vector<double> r((size_t)n * ndof, 0.0);
    auto t0 = std::chrono::steady_clock::now();
    {
        PDOperators ops = m->ops;
        ops.setAbortOnDegenerate(false);
        VectorXd R(ndof), Rn(ndof), UI(ndof), UJ(ndof), UoI(ndof), UoJ(ndof);
        MatrixXd KII(ndof, ndof), KIJ(ndof, ndof), Kn(ndof, ndof);
        for (int i = 1; i <= n; ++i) {
            ops.calcAMatrix(i, d);
            const int bi = (i - 1) * ndof;
            for (int a = 1; a <= ndof; ++a) {
                UI(a) = u[bi + a - 1];
                UoI(a) = uold[bi + a - 1];
            }
            el.computeNodalResidualAndJacobian(info, i, UI, UoI, d.NodeVolumes[i - 1], Rn, Kn);
            for (int a = 1; a <= ndof; ++a) {
                r[bi + a - 1] += Rn(a);
                for (int b = 1; b <= ndof; ++b) K.addValue(bi + a, bi + b, -Kn(a, b));
            }
            for (int j : d.NodesNeighNodesID[i - 1]) {
                ops.calcOperators(i, j, d);
                const int bj = (j - 1) * ndof;
                for (int a = 1; a <= ndof; ++a) {
                    UJ(a) = u[bj + a - 1];
                    UoJ(a) = uold[bj + a - 1];
                }
                el.computeBondResidualAndJacobian(ops, info, i, j, UI, UJ, UoI, UoJ, d.NodeVolumes[i - 1], R, KII, KIJ);
                for (int a = 1; a <= ndof; ++a) {
                    r[bi + a - 1] += R(a);
                    for (int b = 1; b <= ndof; ++b) {
                        K.addValue(bi + a, bi + b, -KII(a, b));
                        K.addValue(bi + a, bj + b, -KIJ(a, b));
                    }
                }
            }
        }
    }
    auto t1 = std::chrono::steady_clock::now();
    std::memcpy(kvals, K.getCSRValuesPtr(), sizeof(double) * (size_t)K.getNNZNum());
    std::memcpy(rhs, r.data(), sizeof(double) * r.size());
    if (vel_out) std::memcpy(vel_out, el.getVel().data(), sizeof(double) * el.getVel().size());
    if (health_out) {
        size_t t = 0;
        for (const auto &fam : el.getBondHealth())
            for (double x : fam) health_out[t++] = x;
    }
    if (consts) {
        consts[0] = el.getC11();
        consts[1] = el.getC12();
        consts[2] = el.getC66();
    }
    return std::chrono::duration<double>(t1 - t0).count();
}

// ---- explicit_pddo_frac element -------------------------------------------------------------------------
void *ref_epf_create(void *mesh, double E, double nu, double rho, double G0, int plane_stress, int tension_only,
                     int damage_on, double bx, double by, double bz) {
    auto *e = new RefEpf();
    e->mesh = static_cast<RefMesh *>(mesh);
    e->el.setDim(e->mesh->dim);
    e->el.setE(E);
    e->el.setNu(nu);
    e->el.setRho(rho);
    e->el.setG0(G0);
    e->el.setState(plane_stress ? ExplicitPDDOFracElement::StressState::PlaneStress
                                : ExplicitPDDOFracElement::StressState::PlaneStrain);
    e->el.setTensionOnly(tension_only != 0);
    e->el.setDamageOn(damage_on != 0);
    e->el.setBodyForce(bx, by, bz);
    return e;
}

void ref_epf_free(void *h) { delete static_cast<RefEpf *>(h); }

// One rate evaluation (damage at u, then Navier force -> accel), OpenMP over nthreads.
// Returns the wall time in seconds of preprocessIteration.
double ref_epf_rate(void *h, const double *u, double *accel, double *health_out, int nthreads) {
    auto *e = static_cast<RefEpf *>(h);
    auto *m = e->mesh;
    const int n = m->pd.getNodesNum();
    const int dim = m->dim;
    VectorXd U(n * dim), Uo(n * dim);
    std::memcpy(U.getDataPtr(), u, sizeof(double) * (size_t)n * dim);
    LocalElmtInfo info;
    info.UseParallel = nthreads != 1;
    info.UseCuda = e->use_cuda;
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#endif
    auto t0 = std::chrono::steady_clock::now();
    e->el.preprocessIteration(m->pd, m->ops, info, dim, U, Uo);
    auto t1 = std::chrono::steady_clock::now();
    if (accel) std::memcpy(accel, e->el.m_Accel.data(), sizeof(double) * (size_t)n * dim);
    if (health_out) std::memcpy(health_out, e->el.m_HealthFlat.data(), sizeof(double) * e->el.m_HealthFlat.size());
    return std::chrono::duration<double>(t1 - t0).count();
}

void ref_epf_set_health(void *h, const double *health) {
    auto *e = static_cast<RefEpf *>(h);
    std::memcpy(e->el.m_HealthFlat.data(), health, sizeof(double) * e->el.m_HealthFlat.size());
}

// ExplicitPDDOFracElement::computeNodalProjection (ExplicitPDDOFracElement.cpp:324-405) for every node at u, on
// the element's current op cache and health: which 0 damage (1 value), 1 vonMises (1), 2 stress (9), 3 strain (9).
void ref_epf_project(void *h, int which, const double *u, double *out) {
    auto *e = static_cast<RefEpf *>(h);
    auto *m = e->mesh;
    const int n = m->pd.getNodesNum();
    const int dim = m->dim;
    static const char *names[4] = {"damage", "vonMises", "stress", "strain"};
    const int k = which < 2 ? 1 : 9;
    VectorXd U(n * dim);
    std::memcpy(U.getDataPtr(), u, sizeof(double) * (size_t)n * dim);
    std::vector<double> o((size_t)k);
    for (int i = 1; i <= n; ++i) {
        e->el.computeNodalProjection(names[which], m->pd, m->ops, U, i, dim, o);
        std::memcpy(out + (size_t)(i - 1) * k, o.data(), sizeof(double) * (size_t)k);
    }
}

// [sc, C11, C12, C66, stable_dt]
void ref_epf_constants(void *h, double *out) {
    auto *e = static_cast<RefEpf *>(h);
    out[0] = e->el.m_Sc; out[1] = e->el.m_C11; out[2] = e->el.m_C12; out[3] = e->el.m_C66;
    out[4] = e->el.estimateStableDt(e->mesh->pd);
}

// cached per-bond op vector of the element (5 or 9 per bond: dx,dy,[dz],dxx,dyy,[dzz],dxy,[dxz,dyz])
void ref_epf_opcache(void *h, double *out) {
    auto *e = static_cast<RefEpf *>(h);
    std::memcpy(out, e->el.m_OpCache.data(), sizeof(double) * e->el.m_OpCache.size());
}

// ---- ghost BC preset + central-difference loop ------------------------------------------------------------
// A BC program is a list of entries applied in order, as BCSystem::presetSolution does (BCSystem.cpp:114-129),
// each by the reference's own DirichletBC / NeumannBC object.  Entry e:
//   kind[e]    0 = Dirichlet (reflect, or direct when direct[e]!=0 or no mirror), 1 = Neumann copy
//   comp_mask  bit a set => component a (0-based) is constrained (the objects take 1-based components)
//   val/vel    dim values each: g(t) = value + velocity*t
//   box        has_box[e] and 6 bounds (xlo,xhi,ylo,yhi,zlo,zhi): DirichletBC::setBox
//   nodes      1-based ids (node_off[e]..node_off[e+1])
void ref_bc_preset(void *h, int nbc, const int *kind, const int *comp_mask, const int *direct, const double *val,
                   const double *vel, const int *has_box, const double *box, const int *node_off, const int *nodes,
                   double t, double *u) {
    auto *m = static_cast<RefMesh *>(h);
    const int dim = m->dim;
    const int n = m->pd.getNodesNum();
    VectorXd U(n * dim);
    std::memcpy(U.getDataPtr(), u, sizeof(double) * (size_t)n * dim);
    for (int e = 0; e < nbc; ++e) {
        std::vector<int> comps;
        std::vector<double> v, w;
        for (int a = 0; a < dim; ++a)
            if (comp_mask[e] & (1 << a)) {
                comps.push_back(a + 1);
                v.push_back(val[e * dim + a]);
                w.push_back(vel[e * dim + a]);
            }
        if (comps.empty()) continue;  // an empty list would mean every component to the reference objects
        const std::vector<int> ids(nodes + node_off[e], nodes + node_off[e + 1]);
        if (kind[e] == 0) {
            DirichletBC bc;
            bc.setValues(v);
            bc.setVelocity(w);
            bc.setComponents(comps);
            bc.setDirect(direct[e] != 0);
            if (has_box[e]) {
                std::array<double, 6> b6;
                for (int k = 0; k < 6; ++k) b6[(size_t)k] = box[6 * e + k];
                bc.setBox(b6);
            }
            bc.presetSolutionAtTime(m->pd, ids, dim, U, t);
        } else {
            NeumannBC bc;
            bc.setComponents(comps);
            bc.presetSolutionAtTime(m->pd, ids, dim, U, t);
        }
    }
    std::memcpy(u, U.getDataPtr(), sizeof(double) * (size_t)n * dim);
}

// Central difference (TimeStepping.cpp:479-547): start u^{-1}=u0-dt v0+dt^2/2 a0, then nsteps uniform steps
// u^{n+1}=2u^n-u^{n-1}+dt^2 a^n followed by the BC preset at t_{n+1}.  u0 in, u/uold out (post-BC),
// health_out the per-bond health after the run; returns seconds spent in the nsteps steps (the start, whose rate
// call also builds the element's operator cache on a fresh element, is not counted).
double ref_epf_run(void *h, const double *u0, const double *v0, double dt, int nsteps, int nbc, const int *kind,
                   const int *comp_mask, const int *direct, const double *val, const double *vel, const int *has_box,
                   const double *box, const int *node_off, const int *nodes, double *u_out, double *uold_out,
                   double *health_out, int nthreads) {
    auto *e = static_cast<RefEpf *>(h);
    auto *m = e->mesh;
    const int n = m->pd.getNodesNum() * m->dim;
    std::vector<double> U(u0, u0 + n), Uo(n), A(n);
    ref_epf_rate(h, U.data(), A.data(), nullptr, nthreads);
    for (int k = 0; k < n; ++k) Uo[k] = U[k] - dt * (v0 ? v0[k] : 0.0) + 0.5 * dt * dt * A[k];
    auto t0 = std::chrono::steady_clock::now();
    double t = 0.0;
    const double dt2 = dt * dt;
    for (int s = 0; s < nsteps; ++s) {
        const double tNew = t + dt;
        ref_epf_rate(h, U.data(), A.data(), nullptr, nthreads);
        for (int k = 0; k < n; ++k) {
            const double un = 2.0 * U[k] - Uo[k] + dt2 * A[k];
            Uo[k] = U[k];
            U[k] = un;
        }
        ref_bc_preset(m, nbc, kind, comp_mask, direct, val, vel, has_box, box, node_off, nodes, tNew, U.data());
        t = tNew;
    }
    auto t1 = std::chrono::steady_clock::now();
    if (u_out) std::memcpy(u_out, U.data(), sizeof(double) * n);
    if (uold_out) std::memcpy(uold_out, Uo.data(), sizeof(double) * n);
    if (health_out) std::memcpy(health_out, e->el.m_HealthFlat.data(), sizeof(double) * e->el.m_HealthFlat.size());
    return std::chrono::duration<double>(t1 - t0).count();
}

// ---- scalar system assembly through the reference's PDSystem --------------------------------------------
// type 0: PoissonElement(sigma = coef, f), type 1: DiffusionElement(D = coef, f) with Info.Dt = dt and Uold.
// use_cuda 0 runs PDSystem::formResidualAndJacobian (the reference CPU assembly); use_cuda 1 runs
// PDSystem::formResidualAndJacobianCUDA, the reference's caller of perix_cuda::assemble (drop-in build only;
// returns -1 elsewhere).  K = -dF/dU, RHS = +F on the reference CSR pattern (SparseMatrix::initFromPDMesh).
// Returns seconds spent in the assembly call.
double ref_system_assemble(void *h, int type, double coef, double f, double dt, const double *u, const double *uold,
                           double *kvals, double *rhs, int use_cuda) {
    auto *m = static_cast<RefMesh *>(h);
    const auto &d = m->pd.getDataConstRef();
    const int n = d.NodesNum;
    ElmtSystem es;
    if (type == 0) {
        auto el = std::make_unique<PoissonElement>(coef, f);
        el->setDim(m->dim);
        es.addElement("poisson", std::move(el));
    } else {
        auto el = std::make_unique<DiffusionElement>();
        el->setDim(m->dim);
        el->setD(coef);
        el->setF(f);
        es.addElement("diffusion", std::move(el));
    }
    SparseMatrix K;
    K.initFromPDMesh(d, 1);
    K.setToZeros();
    VectorXd U(n), Uo(n), R(n);
    std::memcpy(U.getDataPtr(), u, sizeof(double) * (size_t)n);
    if (uold) std::memcpy(Uo.getDataPtr(), uold, sizeof(double) * (size_t)n);
    LocalElmtInfo info;
    info.Dt = dt;
    PDSystem sys;
    auto t0 = std::chrono::steady_clock::now();
    if (use_cuda) {
#ifdef PERIX_CUDA_ASSEMBLE
        sys.formResidualAndJacobianCUDA(m->pd, m->ops, es, info, U, Uo, K, R);
#else
        return -1.0;
#endif
    } else {
        sys.formResidualAndJacobian(m->pd, m->ops, es, info, U, Uo, K, R);
    }
    auto t1 = std::chrono::steady_clock::now();
    std::memcpy(kvals, K.getCSRValuesPtr(), sizeof(double) * (size_t)K.getNNZNum());
    std::memcpy(rhs, R.getDataPtr(), sizeof(double) * (size_t)n);
    return std::chrono::duration<double>(t1 - t0).count();
}

// LocalElmtInfo::UseCuda for the element's rate calls: the reference element then hands the damage and force
// to perix_cuda::assembleExplicitPDDOFracAccel (drop-in build only; returns -1 elsewhere).
int ref_epf_use_cuda(void *h, int on) {
#ifdef PERIX_CUDA_ASSEMBLE
    static_cast<RefEpf *>(h)->use_cuda = on != 0;
    return 0;
#else
    (void)h;
    (void)on;
    return -1;
#endif
}

// 1 when this library is the drop-in build (the reference's callers linked to libperix_b200.so)
int ref_is_dropin(void) {
#ifdef PERIX_CUDA_ASSEMBLE
    return 1;
#else
    return 0;
#endif
}

// The reference's explicit loop to an end time (TimeStepping.cpp:479-599, restated): the start of ref_epf_run, then
// while t < t_end - 1e-12 t_end: dt_attempt = min(dt, t_end - t), the uniform step when dt_attempt equals the
// previous step's dt, else the variable-step form u + (dt/dt_prev)(u - u_prev) + dt (dt + dt_prev)/2 a; the BC
// preset at the new time; the blow-up guard (50-step window: non-finite U, or max|U| above 1e3 max(1, max|U| 50
// steps before).  Returns the number of steps completed; *blowup_step receives the 1-based step at which the guard
// tripped (0 if it did not), and u/uold/health are the state after the last completed step.
int ref_epf_run_to(void *h, const double *u0, const double *v0, double dt, double t_end, int nbc, const int *kind,
                   const int *comp_mask, const int *direct, const double *val, const double *vel, const int *has_box,
                   const double *box, const int *node_off, const int *nodes, double *u_out, double *uold_out,
                   double *health_out, int *blowup_step, double *t_out, int nthreads) {
    auto *e = static_cast<RefEpf *>(h);
    auto *m = e->mesh;
    const int n = m->pd.getNodesNum() * m->dim;
    std::vector<double> U(u0, u0 + n), Uo(n), A(n);
    ref_epf_rate(h, U.data(), A.data(), nullptr, nthreads);
    for (int k = 0; k < n; ++k) Uo[k] = U[k] - dt * (v0 ? v0[k] : 0.0) + 0.5 * dt * dt * A[k];
    constexpr int kWindow = 50;
    double hist[kWindow] = {0.0};
    double t = 0.0, dt_prev = dt;
    const double t_eps = 1.0e-12 * t_end;
    int step = 0, tripped = 0;
    while (t < t_end - t_eps) {
        step++;
        const double dtA = std::min(dt, t_end - t);
        const double tNew = t + dtA;
        const double dt2 = dtA * dtA;
        std::vector<double> Un = U, Uon = Uo;
        ref_epf_rate(h, Un.data(), A.data(), nullptr, nthreads);
        if (dtA == dt_prev) {
            for (int k = 0; k < n; ++k) {
                const double un = 2.0 * Un[k] - Uon[k] + dt2 * A[k];
                Uon[k] = Un[k];
                Un[k] = un;
            }
        } else {
            const double rho = dtA / dt_prev;
            const double w = 0.5 * dtA * (dtA + dt_prev);
            for (int k = 0; k < n; ++k) {
                const double un = Un[k] + rho * (Un[k] - Uon[k]) + w * A[k];
                Uon[k] = Un[k];
                Un[k] = un;
            }
        }
        ref_bc_preset(m, nbc, kind, comp_mask, direct, val, vel, has_box, box, node_off, nodes, tNew, Un.data());
        const int slot = (step - 1) % kWindow;
        const double past = step > kWindow ? hist[slot] : -1.0;
        const double cap = past >= 0.0 ? 1.0e3 * std::max(1.0, past) : std::numeric_limits<double>::infinity();
        double umax = 0.0;
        bool finite = true;
        for (int k = 0; k < n; ++k) {
            const double av = std::fabs(Un[k]);
            if (!(av <= std::numeric_limits<double>::max())) finite = false;
            else if (av > umax) umax = av;
        }
        if (!finite || umax > cap) {
            tripped = step;
            step--;
            break;
        }
        hist[slot] = umax;
        U.swap(Un);
        Uo.swap(Uon);
        t = tNew;
        dt_prev = dtA;
    }
    if (u_out) std::memcpy(u_out, U.data(), sizeof(double) * n);
    if (uold_out) std::memcpy(uold_out, Uo.data(), sizeof(double) * n);
    if (health_out) std::memcpy(health_out, e->el.m_HealthFlat.data(), sizeof(double) * e->el.m_HealthFlat.size());
    if (blowup_step) *blowup_step = tripped;
    if (t_out) *t_out = t;
    return step;
}

int ref_max_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

}  // extern "C"
