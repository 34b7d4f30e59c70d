// perix_cuda:: drop-in shim over the pxb_* C-ABI (the boundary of reference include/PDSystem/CudaAssemble.h).
// Structure uploads are cached and redone only when the sizes change, like the reference
// (src/PDSystem/CudaAssembleKernels.cu:1121-1146); results are copied back into the caller's host arrays.
#include "../../include/perix_cuda_compat.h"

#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "../../include/perix_b200.h"

namespace {

struct ShimState {
    pxb_ctx *ctx = nullptr;
    // which structure is resident (0 none, 1 scalar assembly, 2 explicit fracture, 3 Cahn-Hilliard, 4 stress CH, 5 dynamic fracture)
    int kind = 0;
    int n = 0, nnz = 0, nbtot = 0, nop = 0, ndof = 0, dim = 0;
    int precision = PXB_FP64;
    const double *vh = nullptr;  // the caller's per-node horizon array of the resident structure (variable horizon)
};

ShimState g_shim;

bool report(const char *who) {
    std::fprintf(stderr, "[perix_b200] %s: %s\n", who, pxb_last_error());
    return false;
}

// Precision of the explicit element's device operators: FP64 unless PERIX_B200_PRECISION=mixed (FP32-stored Navier
// coefficients with FP64 arithmetic, state and stretch decisions; within 1e-6 of FP64).
int explicit_precision() {
    const char *v = std::getenv("PERIX_B200_PRECISION");
    return (v && (std::strcmp(v, "mixed") == 0 || std::strcmp(v, "MIXED") == 0)) ? PXB_MIXED : PXB_FP64;
}

bool ensure_ctx() {
    if (g_shim.ctx) return true;
    if (pxb_ctx_create(0, &g_shim.ctx) != PXB_OK) return report("context");
    return true;
}

int order_of(const perix_cuda::AssembleMesh &m) {
    int o = 0;
    for (int k = 0; k < m.nop; ++k) o = std::max(o, m.qp[k] + m.qq[k] + (m.qr ? m.qr[k] : 0));
    return o;
}

// the multi-index table the caller passes must be the one the device kernels are compiled for
// (reference order, src/PDOperators/PDOperators.cpp:51-75)
bool qtable_matches(const perix_cuda::AssembleMesh &m, int order) {
    int k = 0;
    auto check = [&](int p, int q, int r) {
        const bool ok = k < m.nop && m.qp[k] == p && m.qq[k] == q && (m.qr ? m.qr[k] : 0) == r;
        ++k;
        return ok;
    };
    for (int o = 1; o <= order; ++o)
        for (int p = o; p >= 0; --p) {
            if (m.dim == 3) {
                for (int q = o - p; q >= 0; --q)
                    if (!check(p, q, o - p - q)) return false;
            } else if (!check(p, o - p, 0)) {
                return false;
            }
        }
    return k == m.nop;
}

// the mesh, and with a variable horizon (AssembleMesh::nodeHorizon / nodeSpacing, the reference's
// PDMeshData::NodeHorizon / NodeSpacing) the per-node horizons the g-build uses
bool upload_mesh(const perix_cuda::AssembleMesh &m, int order) {
    if (pxb_set_geometry(g_shim.ctx, m.N, m.dim, m.coords, m.vols, m.neigh_off, m.neigh_id, m.delta, m.dx_char,
                         nullptr, nullptr) != PXB_OK)
        return report("set_geometry");
    if (m.nodeHorizon && pxb_set_node_horizons(g_shim.ctx, m.nodeHorizon, m.nodeSpacing) != PXB_OK)
        return report("node horizons");
    g_shim.vh = m.nodeHorizon;
    (void)order;
    return true;
}

}  // namespace

namespace perix_cuda {

void shutdown() {
    if (g_shim.ctx) pxb_ctx_destroy(g_shim.ctx);
    g_shim = ShimState{};
}

bool assemble(const AssembleMesh &m, const ElmtParams &p, const OpSlots &s, const double *u, const double *uold,
              double *out_Kvals, double *out_rhs) {
    if (m.N <= 0 || p.ndof != 1 || s.dxx < 0 || s.dyy < 0) return false;
    if (!ensure_ctx()) return false;
    const int order = order_of(m);
    if (!qtable_matches(m, order)) {
        std::fprintf(stderr, "[perix_b200] assemble: unexpected multi-index table\n");
        return false;
    }
    const int nbtot = m.neigh_off[m.N];
    if (g_shim.kind != 1 || g_shim.n != m.N || g_shim.nnz != m.nnz || g_shim.nbtot != nbtot || g_shim.nop != m.nop ||
        g_shim.vh != m.nodeHorizon) {
        if (!upload_mesh(m, order)) return false;
        int ndeg = 0, first = 0;
        const int st = pxb_gbuild(g_shim.ctx, order, PXB_FP64, &ndeg, &first);
        if (st == PXB_ERR_DEGENERATE)
            std::fprintf(stderr, "[perix_b200] assemble: %s (rows of those nodes are zeroed)\n", pxb_last_error());
        else if (st != PXB_OK)
            return report("gbuild");
        if (pxb_csr_set_pattern(g_shim.ctx, 1, m.csr_off, m.csr_col, m.nnz) != PXB_OK) return report("csr pattern");
        g_shim.kind = 1;
        g_shim.n = m.N;
        g_shim.nnz = m.nnz;
        g_shim.nbtot = nbtot;
        g_shim.nop = m.nop;
    }
    const bool diffusion = (p.type == ELMT_DIFFUSION);
    const int st = pxb_assemble_scalar(g_shim.ctx, diffusion ? 1 : 0, diffusion ? p.D : p.sigma, p.f, nullptr,
                                       diffusion ? p.dt : 0.0, u, uold, out_Kvals, out_rhs);
    if (st != PXB_OK) return report("assemble");
    return true;
}

bool assembleCahnHilliard(const CahnHilliardMesh &m, const CahnHilliardParams &p, const int *csr_off,
                          const int *csr_col, int nnz, const double *u, const double *uold, double *out_Kvals,
                          double *out_rhs) {
    if (m.N <= 0 || !(p.dt > 0.0)) return false;
    if (!ensure_ctx()) return false;
    if (g_shim.kind != 3 || g_shim.n != m.N || g_shim.nnz != nnz || g_shim.nbtot != m.nbtot) {
        // the conservative CH kernel needs topology, volumes and the host-built Laplacian, not coordinates
        std::vector<double> zeros((size_t)m.N * 3, 0.0);
        if (pxb_set_geometry(g_shim.ctx, m.N, 2, zeros.data(), m.vol, m.off, m.nbr, 1.0, 0.0, nullptr, nullptr) != PXB_OK)
            return report("set_geometry");
        if (pxb_ch_set_geometry(g_shim.ctx, m.rev, m.lapbond, m.isghost) != PXB_OK) return report("ch geometry");
        if (pxb_csr_set_pattern(g_shim.ctx, 2, csr_off, csr_col, nnz) != PXB_OK) return report("csr pattern");
        g_shim.kind = 3;
        g_shim.n = m.N;
        g_shim.nnz = nnz;
        g_shim.nbtot = m.nbtot;
    }
    if (pxb_assemble_ch(g_shim.ctx, p.kappa, p.chi, p.dt, m.mnode, u, uold, out_Kvals, out_rhs) != PXB_OK)
        return report("assembleCahnHilliard");
    return true;
}

bool assembleStressCahnHilliard(const AssembleMesh &m, const StressCahnHilliardParams &p, const OpSlots &s,
                                const int *rev, const double *lapbond, const char *isghost, const double *mnode,
                                const double *health, const double *vel, const double *u, const double *uold,
                                double *out_Kvals, double *out_rhs) {
    (void)s;  // the operator slots are resolved from the multi-index table, which must be the reference's
    if (m.N <= 0 || (p.dim != 2 && p.dim != 3) || p.ndof != p.dim + 2 || !(p.dt > 0.0)) return false;
    if (!ensure_ctx()) return false;
    if (order_of(m) != 2 || !qtable_matches(m, 2)) {
        std::fprintf(stderr, "[perix_b200] assembleStressCahnHilliard: needs the order-2 multi-index table\n");
        return false;
    }
    const int nbtot = m.neigh_off[m.N];
    if (g_shim.kind != 4 || g_shim.n != m.N || g_shim.nnz != m.nnz || g_shim.nbtot != nbtot || g_shim.dim != p.dim ||
        g_shim.vh != m.nodeHorizon) {
        if (!upload_mesh(m, 2)) return false;
        int ndeg = 0, first = 0;
        const int st = pxb_gbuild(g_shim.ctx, 2, PXB_FP64, &ndeg, &first);
        if (st == PXB_ERR_DEGENERATE)
            std::fprintf(stderr, "[perix_b200] assembleStressCahnHilliard: %s (rows of those nodes are zeroed)\n",
                         pxb_last_error());
        else if (st != PXB_OK)
            return report("gbuild");
        if (pxb_ch_set_geometry(g_shim.ctx, rev, lapbond, isghost) != PXB_OK) return report("ch geometry");
        if (pxb_csr_set_pattern(g_shim.ctx, p.ndof, m.csr_off, m.csr_col, m.nnz) != PXB_OK) return report("csr pattern");
        g_shim.kind = 4;
        g_shim.n = m.N;
        g_shim.nnz = m.nnz;
        g_shim.nbtot = nbtot;
        g_shim.dim = p.dim;
    } else if (pxb_ch_set_geometry(g_shim.ctx, rev, lapbond, isghost) != PXB_OK) {
        return report("ch geometry");  // host-built per element; cheap to refresh
    }
    const pxb_stress_ch_params q{p.C11, p.C12, p.C66, p.A, p.Kh, p.Ch, p.Omega, p.cref, p.chi, p.kappa, p.dt, p.kres, p.rho};
    if (pxb_assemble_stress_ch(g_shim.ctx, &q, mnode, health, vel, u, uold, out_Kvals, out_rhs) != PXB_OK)
        return report("assembleStressCahnHilliard");
    return true;
}

bool assembleCached(const AssembleMesh &m, const CachedParams &p, const OpSlots &s, const double *nodecache,
                    const double *bondcache, const double *u, const double *uold, double *out_Kvals,
                    double *out_rhs) {
    (void)s;  // the operator slots are resolved from the multi-index table, which must be the reference's
    if (m.N <= 0 || (p.dim != 2 && p.dim != 3) || p.ndof != p.dim || !(p.dt > 0.0)) return false;
    if (!ensure_ctx()) return false;
    if (order_of(m) != 2 || !qtable_matches(m, 2)) {
        std::fprintf(stderr, "[perix_b200] assembleCached: needs the order-2 multi-index table\n");
        return false;
    }
    const int nbtot = m.neigh_off[m.N];
    if (g_shim.kind != 5 || g_shim.n != m.N || g_shim.nnz != m.nnz || g_shim.nbtot != nbtot || g_shim.dim != p.dim ||
        g_shim.vh != m.nodeHorizon) {
        if (!upload_mesh(m, 2)) return false;
        int ndeg = 0, first = 0;
        const int st = pxb_gbuild(g_shim.ctx, 2, PXB_FP64, &ndeg, &first);
        if (st == PXB_ERR_DEGENERATE)
            std::fprintf(stderr, "[perix_b200] assembleCached: %s (rows of those nodes are zeroed)\n", pxb_last_error());
        else if (st != PXB_OK)
            return report("gbuild");
        if (pxb_csr_set_pattern(g_shim.ctx, p.ndof, m.csr_off, m.csr_col, m.nnz) != PXB_OK) return report("csr pattern");
        g_shim.kind = 5;
        g_shim.n = m.N;
        g_shim.nnz = m.nnz;
        g_shim.nbtot = nbtot;
        g_shim.dim = p.dim;
    }
    const pxb_cached_params q{p.C11, p.C12, p.C66, p.rho, p.dt, {p.bx, p.by, p.bz}};
    if (pxb_assemble_cached(g_shim.ctx, &q, nodecache, p.ncache, bondcache, p.nbcache, u, uold, out_Kvals, out_rhs) !=
        PXB_OK)
        return report("assembleCached");
    return true;
}

bool assembleExplicitPDDOFracAccel(const AssembleMesh &m, const ExplicitPDDOFracParams &p, const OpSlots &s,
                                   const double *u, double *health_inout, double *accel_out, int *health_changed) {
    (void)s;
    if (health_changed) *health_changed = 0;
    if (m.N <= 0 || (p.dim != 2 && p.dim != 3)) return false;
    if (!ensure_ctx()) return false;
    const int nbtot = m.neigh_off[m.N];
    if (g_shim.kind != 2 || g_shim.n != m.N || g_shim.nbtot != nbtot || g_shim.dim != p.dim ||
        g_shim.vh != m.nodeHorizon) {
        if (pxb_set_geometry(g_shim.ctx, m.N, p.dim, m.coords, m.vols, m.neigh_off, m.neigh_id, m.delta, m.dx_char,
                             nullptr, nullptr) != PXB_OK)
            return report("set_geometry");
        if (m.nodeHorizon && pxb_set_node_horizons(g_shim.ctx, m.nodeHorizon, m.nodeSpacing) != PXB_OK)
            return report("node horizons");
        g_shim.vh = m.nodeHorizon;
        std::vector<uint8_t> h0((size_t)nbtot);
        for (int t = 0; t < nbtot; ++t) h0[(size_t)t] = health_inout[t] > 0.0 ? 1 : 0;
        const double b[3] = {p.bx, p.by, p.bz};
        const double sc = p.damage_on ? p.sc : 0.0;
        const int prec = explicit_precision();
        if (pxb_epf_setup(g_shim.ctx, prec, p.C11, p.C12, p.C66, p.rho, b, sc, p.tension_only, h0.data()) != PXB_OK)
            return report("epf setup");
        // variable horizon: each bond breaks at s_c(0.5 (delta_i + delta_j)) (ExplicitPDDOFracElement.cpp:254-261)
        if (m.nodeHorizon && p.damage_on &&
            pxb_epf_set_variable_horizon_stretch(g_shim.ctx, p.G0, p.E, p.plane_stress) != PXB_OK)
            return report("variable-horizon stretch");
        // the per-step call's schedule, timed once per problem signature at this displacement (state unchanged)
        if (pxb_epf_autotune_rate(g_shim.ctx, u, 3, 1, nullptr, nullptr) != PXB_OK) return report("epf autotune");
        g_shim.precision = prec;
        g_shim.kind = 2;
        g_shim.n = m.N;
        g_shim.nbtot = nbtot;
        g_shim.dim = p.dim;
    }
    long long broken = 0;
    if (pxb_epf_rate(g_shim.ctx, u, accel_out, &broken) != PXB_OK) return report("assembleExplicitPDDOFracAccel");
    if (broken > 0) {
        std::vector<uint8_t> h((size_t)nbtot);
        if (pxb_epf_get_state(g_shim.ctx, nullptr, nullptr, h.data(), nullptr) != PXB_OK) return report("health readback");
        for (int t = 0; t < nbtot; ++t) health_inout[t] = h[(size_t)t] ? 1.0 : 0.0;
        if (health_changed) *health_changed = 1;
    }
    return true;
}

}  // namespace perix_cuda

// C entry over the explicit drop-in call, for callers that bind C rather than C++ (ctypes, other FFIs): the
// arguments are the members of AssembleMesh / ExplicitPDDOFracParams the call reads, and the behaviour is
// perix_cuda::assembleExplicitPDDOFracAccel's (1 on success, 0 where that returns false).
extern "C" int pxb_cuda_explicit_accel(int n, int dim, const int *neigh_off, const int *neigh_id, const double *coords,
                                       const double *vols, double delta, double dx_char, double C11, double C12,
                                       double C66, double rho, const double *body, double sc, int tension_only,
                                       int damage_on, const double *u, double *health_inout, double *accel_out,
                                       int *health_changed) {
    perix_cuda::AssembleMesh m;
    m.N = n;
    m.dim = dim;
    m.neigh_off = neigh_off;
    m.neigh_id = neigh_id;
    m.coords = coords;
    m.vols = vols;
    m.delta = delta;
    m.dx_char = dx_char;
    perix_cuda::ExplicitPDDOFracParams p;
    p.dim = dim;
    p.C11 = C11;
    p.C12 = C12;
    p.C66 = C66;
    p.rho = rho;
    p.bx = body ? body[0] : 0.0;
    p.by = body ? body[1] : 0.0;
    p.bz = body && dim == 3 ? body[2] : 0.0;
    p.sc = sc;
    p.tension_only = tension_only;
    p.damage_on = damage_on;
    perix_cuda::OpSlots s;
    return perix_cuda::assembleExplicitPDDOFracAccel(m, p, s, u, health_inout, accel_out, health_changed) ? 1 : 0;
}

extern "C" void pxb_cuda_shutdown(void) { perix_cuda::shutdown(); }
