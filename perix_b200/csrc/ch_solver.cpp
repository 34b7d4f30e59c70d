// Implicit backward-Euler Cahn-Hilliard run on the device and its discrete adjoint.
//
// The forward run follows the reference's transient CH solve: per time step a Newton iteration on the conservative
// element's residual (CahnHilliardElement.cpp:178-292) with the mobility M(c) = M0 c (1 - c) frozen per Newton
// iteration at the current iterate (CahnHilliardElement::preprocessIteration, .cpp:66-175) and without its
// derivative in the Jacobian (a Picard-Newton iteration), zero-Neumann ghost rows replaced as NeumannBC::apply
// does (NeumannBC.cpp:127-150).  Each linear system K dU = F is solved on the device by BiCGStab with a 2x2
// block-Jacobi preconditioner, one cooperative kernel per solve (k_bicg.cu); assembly, solve and updates never leave
// the GPU, and the host reads the solve's outcome and the residual norm once per Newton iteration.
//
// The gradient of the total free energy E(U_N) (k_linalg.cu) with respect to kappa and the initial field c0 is the
// discrete adjoint of the converged steps: with F_n(U_n, U_{n-1}) = 0, dF_n/dU_n = -K_n + J_M (the mobility term the
// Picard Jacobian omits), each step backwards solves (K_n^T - J_M^T) lambda_n = g_n with g_N = dE/dU_N and
// g_{n-1} = (dF_n/dU_{n-1})^T lambda_n (the c_old term), and accumulates dE/dkappa += lambda_n . dF_n/dkappa.  The
// converged states are kept on the device (one per step).
#include <algorithm>
#include <cmath>
#include <string>
#include <vector>

#include "pxb_context.h"

namespace pxb {
namespace {

constexpr double kUpdateTol = 1e-14;  // Newton stops when |dU| <= kUpdateTol |U|
constexpr size_t kBicgScalarBytes = 128;  // BicgScalars, then the partial sums
static_assert(sizeof(BicgScalars) <= kBicgScalarBytes, "BiCGStab scalar block");
constexpr int kHostDots = 4;  // dot products read back with a solve's outcome

struct RunCtx {
    pxb_ctx *c;
    int n;
    long long rows;
    pxb_ch_run_params p;
};

int need_ch_run(pxb_ctx *c, const char *who) {
    if (!c || !c->g.ready) return fail(PXB_ERR_STATE, std::string(who) + ": geometry not set");
    if (c->g.dim != 2) return fail(PXB_ERR_UNSUPPORTED, std::string(who) + ": the implicit CH run is 2D");
    const OpsCache &o = c->ops;
    if (!o.ready || o.order != 2 || o.precision != PXB_FP64)
        return fail(PXB_ERR_STATE, std::string(who) + ": needs an FP64 order-2 g-build (pxb_gbuild)");
    if (!c->ch.ready) return fail(PXB_ERR_STATE, std::string(who) + ": needs the CH geometry (pxb_ch_build_geometry)");
    if (!c->csr.ready || c->csr.ndof != 2) return fail(PXB_ERR_STATE, std::string(who) + ": set a 2-dof pattern first");
    if (!c->csr.blocked2)
        return fail(PXB_ERR_UNSUPPORTED, std::string(who) + ": the pattern must consist of dense 2x2 node blocks");
    return PXB_OK;
}

int check(pxb_ctx *c, cudaError_t e, const char *what) {
    if (e != cudaSuccess) return fail(PXB_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
    c->launches++;
    return PXB_OK;
}

int alloc_run(RunCtx &r) {
    pxb_ctx *c = r.c;
    ChState &h = c->ch;
    const size_t rows = (size_t)r.rows, n = (size_t)r.n;
    PXB_TRY(dev_alloc(c, h.U, sizeof(double) * rows));
    PXB_TRY(dev_alloc(c, h.Uold, sizeof(double) * rows));
    PXB_TRY(dev_alloc(c, h.dU, sizeof(double) * rows));
    PXB_TRY(dev_alloc(c, h.rhs, sizeof(double) * rows));
    PXB_TRY(dev_alloc(c, h.kv, sizeof(double) * (size_t)c->csr.nnz));
    PXB_TRY(dev_alloc(c, h.mnode, sizeof(double) * n));
    PXB_TRY(dev_alloc(c, h.binv, sizeof(double) * 4 * n));
    PXB_TRY(dev_alloc(c, h.red, sizeof(double) * (size_t)(dot_scratch_doubles() + 8)));
    PXB_TRY(dev_alloc(c, h.nodal, sizeof(double) * 2 * n));
    for (auto &w : h.w) PXB_TRY(dev_alloc(c, w, sizeof(double) * rows));
    PXB_TRY(dev_alloc(c, h.bicg, kBicgScalarBytes + sizeof(double) * 6 * kBicgParts));
    PXB_TRY(ensure_pinned(h.bicg_h, kBicgScalarBytes + sizeof(double) * kHostDots));
    if (h.ones.bytes < sizeof(double) * n) {
        std::vector<double> one(n, 1.0);
        PXB_TRY(dev_upload(c, h.ones, one.data(), sizeof(double) * n));
    }
    return PXB_OK;
}

int dotp(RunCtx &r, long long len, const double *a, const double *b, double *out) {
    pxb_ctx *c = r.c;
    double *red = c->ch.red.as<double>();
    PXB_TRY(check(c, launch_dot(len, a, b, red, red + dot_scratch_doubles(), c->stream), "dot"));
    PXB_CUDA_TRY(cudaMemcpyAsync(out, red + dot_scratch_doubles(), sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    PXB_CUDA_TRY(cudaStreamSynchronize(c->stream));
    return PXB_OK;
}

int copy(RunCtx &r, double *dst, const double *src) {
    PXB_CUDA_TRY(cudaMemcpyAsync(dst, src, sizeof(double) * (size_t)r.rows, cudaMemcpyDeviceToDevice, r.c->stream));
    return PXB_OK;
}

// K (Picard Jacobian, Neumann ghost rows) and F at (U, Uold) into ch.kv / ch.rhs; the mobility at U into ch.mnode
int assemble(RunCtx &r, const double *U, const double *Uold) {
    pxb_ctx *c = r.c;
    ChState &h = c->ch;
    PXB_TRY(check(c, launch_ch_mobility(r.n, r.p.M0, U, h.mnode.as<double>(), c->stream), "ch mobility"));
    PXB_TRY(pxb_assemble_ch_d(c, r.p.kappa, r.p.chi, r.p.dt, h.mnode.as<double>(), U, Uold, h.kv.as<double>(),
                              h.rhs.as<double>()));
    if (c->g.mirror.p)
        PXB_TRY(check(c, launch_ch_ghost_rows(r.n, c->g.mirror.as<int>(), c->csr.rowptr.as<int>(), c->csr.cols.as<int>(),
                                              U, h.kv.as<double>(), h.rhs.as<double>(), c->stream),
                      "ch ghost rows"));
    return PXB_OK;
}

ChAdjArgs adj_args(RunCtx &r, const double *U, const double *x, double *y) {
    pxb_ctx *c = r.c;
    ChAdjArgs a;
    a.n = r.n;
    a.M0 = r.p.M0;
    a.off = c->g.off.as<int>();
    a.nbr = c->g.nbr.as<int>();
    a.rev = c->ch.rev.as<int>();
    a.mirror = c->g.mirror.p ? c->g.mirror.as<int>() : nullptr;
    a.ghost = c->ch.ghost.p ? c->ch.ghost.as<char>() : nullptr;
    a.lap = c->ch.lap.as<double>();
    a.vol = c->g.vol.as<double>();
    a.u = U;
    a.x = x;
    a.y = y;
    return a;
}

// Right-preconditioned BiCGStab for A x = b (x starts at 0) on the device, one cooperative kernel (k_bicg.cu); A = K
// (ch.kv) or, for adjoint solves, K'^T (ch.kvt through the transposed block view); the block-Jacobi inverse of A must
// be in ch.binv.  Launches only; bicg_outcome reads the result after the caller's next synchronisation.
int bicgstab_launch(RunCtx &r, bool adjoint, const double *b, double *x) {
    pxb_ctx *c = r.c;
    ChState &h = c->ch;
    BicgArgs a;
    a.n = r.n;
    a.bptr = (adjoint ? c->csr.tbptr : c->csr.bptr).as<int>();
    a.bcol = (adjoint ? c->csr.tbcol : c->csr.bcol).as<int>();
    a.val = (adjoint ? h.kvt : h.kv).as<double>();
    a.binv = h.binv.as<double>();
    a.b = b;
    a.x = x;
    a.r = h.w[0].as<double>();
    a.r0 = h.w[1].as<double>();
    a.rh = h.w[2].as<double>();
    a.v = h.w[3].as<double>();
    a.s = h.w[4].as<double>();
    a.t = h.w[5].as<double>();
    a.sh = h.w[6].as<double>();
    a.ph[0] = h.w[7].as<double>();
    a.ph[1] = h.w[8].as<double>();
    a.vh[0] = h.w[9].as<double>();
    a.vh[1] = h.w[10].as<double>();
    a.sc = h.bicg.as<BicgScalars>();
    a.part = reinterpret_cast<double *>(h.bicg.as<char>() + kBicgScalarBytes);
    PXB_TRY(check(c, launch_bicg_solve(a, r.p.lin_rtol, r.p.lin_max, c->stream), "bicgstab"));
    return PXB_OK;
}

// Host copies of the solve's outcome (pinned: BicgScalars, then kHostDots dot products); queue_readback enqueues the
// copies of the outcome and of the first ndots entries of ch.red's result slots.
BicgScalars *host_outcome(ChState &h) { return static_cast<BicgScalars *>(h.bicg_h.p); }
double *host_dots(ChState &h) { return reinterpret_cast<double *>(static_cast<char *>(h.bicg_h.p) + kBicgScalarBytes); }
double *dev_dots(ChState &h) { return h.red.as<double>() + dot_scratch_doubles(); }

int queue_readback(pxb_ctx *c, int ndots) {
    ChState &h = c->ch;
    PXB_CUDA_TRY(cudaMemcpyAsync(host_outcome(h), h.bicg.p, sizeof(BicgScalars), cudaMemcpyDeviceToHost, c->stream));
    if (ndots > 0)
        PXB_CUDA_TRY(cudaMemcpyAsync(host_dots(h), dev_dots(h), sizeof(double) * ndots, cudaMemcpyDeviceToHost,
                                     c->stream));
    return PXB_OK;
}

int bicg_outcome(ChState &h, int *its, double *relres) {
    const BicgScalars *hs = host_outcome(h);
    *its = hs->its;
    *relres = hs->relres;
    if (hs->status == kBicgDone) return PXB_OK;
    if (hs->abort) return fail(PXB_ERR_CUDA, "CH linear solve: a grid barrier of the BiCGStab kernel timed out");
    const char *why = hs->status == kBicgBreakdown ? " (breakdown)" : "";
    return fail(PXB_ERR_STATE, "CH linear solve: BiCGStab stopped at relative residual " + std::to_string(*relres) +
                                   " after " + std::to_string(*its) + " iterations" + why);
}

// dot product a . b into result slot k of ch.red (launch only)
int dot_into(RunCtx &r, long long len, const double *a, const double *b, int k) {
    pxb_ctx *c = r.c;
    double *red = c->ch.red.as<double>();
    return check(c, launch_dot(len, a, b, red, dev_dots(c->ch) + k, c->stream), "dot");
}

// the transposed block view and value permutation of the pattern, and room for K^T (adjoint solves)
int ensure_transpose(pxb_ctx *c) {
    CsrState &k = c->csr;
    if (!k.transposed) {
        if (k.h_bptr.empty()) {  // a pattern built on the device: its block view comes to the host once
            k.h_bptr.resize((size_t)c->g.n + 1);
            PXB_TRY(d2h(c, k.h_bptr.data(), k.bptr.p, sizeof(int) * k.h_bptr.size()));
            PXB_TRY(sync(c));
            k.h_bcol.resize((size_t)k.h_bptr.back());
            if (!k.h_bcol.empty()) PXB_TRY(d2h(c, k.h_bcol.data(), k.bcol.p, sizeof(int) * k.h_bcol.size()));
            PXB_TRY(sync(c));
        }
        std::vector<int> tbptr, tbcol, perm;
        block_transpose(c->g.n, k.h_bptr, k.h_bcol, tbptr, tbcol, perm);
        PXB_TRY(dev_upload(c, k.tbptr, tbptr.data(), sizeof(int) * tbptr.size()));
        PXB_TRY(dev_upload(c, k.tbcol, tbcol.data(), sizeof(int) * std::max<size_t>(1, tbcol.size())));
        PXB_TRY(dev_upload(c, k.tperm, perm.data(), sizeof(int) * std::max<size_t>(1, perm.size())));
        PXB_TRY(sync(c));
        k.transposed = true;
    }
    return dev_alloc(c, c->ch.kvt, sizeof(double) * (size_t)k.nnz);
}

// one backward-Euler step: U (in: initial guess, out: converged state) from Uold
int newton_step(RunCtx &r, double *U, const double *Uold, pxb_ch_run_stats *st) {
    pxb_ctx *c = r.c;
    ChState &h = c->ch;
    double res0 = -1.0;
    for (int it = 0; it <= r.p.newton_max; ++it) {
        PXB_TRY(assemble(r, U, Uold));
        double ff = 0.0;
        PXB_TRY(dotp(r, r.rows, h.rhs.as<double>(), h.rhs.as<double>(), &ff));
        const double res = std::sqrt(ff);
        if (!std::isfinite(res)) return fail(PXB_ERR_BLOWUP, "CH Newton: non-finite residual");
        if (it == 0) res0 = res;
        st->max_residual = std::max(st->max_residual, it == 0 ? 0.0 : res / std::max(res0, 1e-300));
        if (res == 0.0 || (it > 0 && res <= r.p.newton_rtol * res0)) {
            st->newton_iters += it;
            return PXB_OK;
        }
        if (it == r.p.newton_max) break;
        PXB_TRY(check(c, launch_block_inv(r.n, c->csr.diag.as<int>(), h.kv.as<double>(), false, h.binv.as<double>(),
                                          c->stream),
                      "block inverse"));
        PXB_TRY(bicgstab_launch(r, false, h.rhs.as<double>(), h.dU.as<double>()));
        PXB_TRY(dot_into(r, r.rows, h.dU.as<double>(), h.dU.as<double>(), 0));
        PXB_TRY(dot_into(r, r.rows, U, U, 1));
        PXB_TRY(check(c, launch_axpby(r.rows, 1.0, h.dU.as<double>(), 1.0, U, c->stream), "update"));
        PXB_TRY(queue_readback(c, 2));
        PXB_TRY(sync(c));
        int lits = 0;
        double lres = 0.0;
        PXB_TRY(bicg_outcome(h, &lits, &lres));
        st->lin_iters += lits;
        st->max_lin_relres = std::max(st->max_lin_relres, lres);
        const double dd = host_dots(h)[0], uu = host_dots(h)[1];
        // an update at the rounding level of the state ends the iteration (the residual of a small step can sit
        // at its evaluation floor, far above newton_rtol times its initial value)
        if (std::sqrt(dd) <= kUpdateTol * std::sqrt(uu)) {
            st->newton_iters += it + 1;
            return PXB_OK;
        }
    }
    return fail(PXB_ERR_STATE, "CH Newton did not reach the relative residual " + std::to_string(r.p.newton_rtol));
}

// U0 = (c0, 0) with ghost c copied from the mirror bulk node
int initial_state(RunCtx &r, const double *c0, double *U) {
    const Geometry &g = r.c->g;
    std::vector<double> u((size_t)r.rows, 0.0);
    for (int i = 0; i < r.n; ++i) {
        const int m = g.h_mirror.empty() ? 0 : g.h_mirror[(size_t)i];
        u[2 * (size_t)i] = m > 0 ? c0[(size_t)m - 1] : c0[(size_t)i];
    }
    return h2d(r.c, U, u.data(), sizeof(double) * u.size());
}

int validate(pxb_ctx *c, const pxb_ch_run_params *p, const double *c0, const char *who) {
    PXB_TRY(need_ch_run(c, who));
    if (!p || !c0 || p->nsteps < 0 || !(p->dt > 0.0) || !(p->M0 >= 0.0) || p->newton_max < 1 || p->lin_max < 1 ||
        !(p->newton_rtol > 0.0) || !(p->lin_rtol > 0.0))
        return fail(PXB_ERR_INVALID, std::string(who) + ": bad arguments");
    return PXB_OK;
}

// E(U) (returned) and, when dedu != NULL, dE/dU and dE/dkappa's explicit part
int energy(RunCtx &r, const double *U, double *E, double *dedk_explicit, double *dedu) {
    pxb_ctx *c = r.c;
    ChState &h = c->ch;
    const OpsCache &o = c->ops;
    auto slot = [&](int pp, int q) {
        for (int s = 0; s < o.nop; ++s)
            if (o.pqr[3 * s] == pp && o.pqr[3 * s + 1] == q && o.pqr[3 * s + 2] == 0) return s;
        return -1;
    };
    ChEnergyArgs a;
    a.n = r.n;
    a.nop = o.nop;
    a.sx = slot(1, 0);
    a.sy = slot(0, 1);
    a.kappa = r.p.kappa;
    a.chi = r.p.chi;
    a.off = c->g.off.as<int>();
    a.nbr = c->g.nbr.as<int>();
    a.rev = c->ch.rev.as<int>();
    a.mirror = c->g.mirror.p ? c->g.mirror.as<int>() : nullptr;
    a.vol = c->g.vol.as<double>();
    a.ops = o.ops.as<double>();
    a.u = U;
    a.e_out = h.nodal.as<double>();
    a.grad_e = h.nodal.as<double>() + r.n;
    a.gbar = h.w[0].as<double>();
    a.fprime = h.w[1].as<double>();
    PXB_TRY(check(c, launch_ch_energy(a, c->stream), "ch energy"));
    PXB_TRY(dotp(r, r.n, a.e_out, h.ones.as<double>(), E));
    if (dedk_explicit) PXB_TRY(dotp(r, r.n, a.grad_e, h.ones.as<double>(), dedk_explicit));
    if (dedu) PXB_TRY(check(c, launch_ch_energy_grad(a, dedu, c->stream), "ch energy gradient"));
    return PXB_OK;
}

}  // namespace
}  // namespace pxb

using namespace pxb;

extern "C" int pxb_ch_run(pxb_ctx *c, const pxb_ch_run_params *p, const double *c0, double *u_final, double *E,
                          pxb_ch_run_stats *stats) {
    PXB_TRY(validate(c, p, c0, "pxb_ch_run"));
    RunCtx r{c, c->g.n, 2LL * c->g.n, *p};
    PXB_TRY(alloc_run(r));
    ChState &h = c->ch;
    pxb_ch_run_stats st{};
    PXB_TRY(initial_state(r, c0, h.U.as<double>()));
    for (int s = 0; s < p->nsteps; ++s) {
        PXB_TRY(copy(r, h.Uold.as<double>(), h.U.as<double>()));
        PXB_TRY(newton_step(r, h.U.as<double>(), h.Uold.as<double>(), &st));
        st.steps++;
    }
    double e = 0.0;
    PXB_TRY(energy(r, h.U.as<double>(), &e, nullptr, nullptr));
    st.energy = e;
    if (E) *E = e;
    if (u_final) PXB_TRY(d2h(c, u_final, h.U.p, sizeof(double) * (size_t)r.rows));
    PXB_TRY(sync(c));
    if (stats) *stats = st;
    return PXB_OK;
}

extern "C" int pxb_ch_gradient(pxb_ctx *c, const pxb_ch_run_params *p, const double *c0, double *E, double *dE_dkappa,
                               double *dE_dc0, pxb_ch_run_stats *stats) {
    PXB_TRY(validate(c, p, c0, "pxb_ch_gradient"));
    RunCtx r{c, c->g.n, 2LL * c->g.n, *p};
    PXB_TRY(alloc_run(r));
    ChState &h = c->ch;
    const size_t rows = (size_t)r.rows;
    PXB_TRY(dev_alloc(c, h.hist, sizeof(double) * rows * ((size_t)p->nsteps + 1)));
    double *hist = h.hist.as<double>();
    pxb_ch_run_stats st{};
    PXB_TRY(initial_state(r, c0, hist));
    for (int s = 1; s <= p->nsteps; ++s) {
        double *Un = hist + rows * (size_t)s;
        PXB_TRY(copy(r, Un, Un - rows));
        PXB_TRY(newton_step(r, Un, Un - rows, &st));
        st.steps++;
    }
    // g_N = dE/dU_N (in ch.Uold), dE/dkappa explicit part
    double e = 0.0, dk = 0.0;
    double *g = h.Uold.as<double>(), *lam = h.dU.as<double>();
    PXB_TRY(energy(r, hist + rows * (size_t)p->nsteps, &e, &dk, g));
    PXB_TRY(ensure_transpose(c));
    for (int s = p->nsteps; s >= 1; --s) {
        const double *Un = hist + rows * (size_t)s;
        // A = (K - J_M)^T at (U_n, U_{n-1}): fold the mobility derivative into K, then transpose the values
        PXB_TRY(assemble(r, Un, Un - rows));
        const ChAdjArgs fa = adj_args(r, Un, nullptr, nullptr);
        PXB_TRY(check(c, launch_ch_fold_mobility(fa, c->csr.slot.as<int>(), c->csr.diag.as<int>(), h.kv.as<double>(),
                                                 c->stream),
                      "ch mobility fold"));
        PXB_TRY(check(c, launch_gather_values(c->csr.nnz, c->csr.tperm.as<int>(), h.kv.as<double>(), h.kvt.as<double>(),
                                              c->stream),
                      "transpose values"));
        PXB_TRY(check(c, launch_block_inv(r.n, c->csr.diag.as<int>(), h.kv.as<double>(), true, h.binv.as<double>(),
                                          c->stream),
                      "block inverse"));
        PXB_TRY(bicgstab_launch(r, true, g, lam));
        ChAdjArgs a = adj_args(r, Un, lam, h.nodal.as<double>());
        PXB_TRY(check(c, launch_ch_dkappa(a, c->stream), "ch dkappa"));
        PXB_TRY(dot_into(r, r.n, h.nodal.as<double>(), h.ones.as<double>(), 0));
        PXB_TRY(queue_readback(c, 1));
        PXB_TRY(sync(c));
        int lits = 0;
        double lres = 0.0;
        PXB_TRY(bicg_outcome(h, &lits, &lres));
        st.lin_iters += lits;
        st.max_lin_relres = std::max(st.max_lin_relres, lres);
        dk += host_dots(h)[0];
        PXB_TRY(check(c, launch_ch_prev_cot(r.n, a.mirror, lam, p->dt, g, c->stream), "ch previous cotangent"));
    }
    st.energy = e;
    if (E) *E = e;
    if (dE_dkappa) *dE_dkappa = dk;
    if (dE_dc0) {
        std::vector<double> gh(rows);
        PXB_TRY(d2h(c, gh.data(), g, sizeof(double) * rows));
        PXB_TRY(sync(c));
        for (int i = 0; i < r.n; ++i) dE_dc0[i] = gh[2 * (size_t)i];
    }
    PXB_TRY(sync(c));
    if (stats) *stats = st;
    return PXB_OK;
}

extern "C" int pxb_ch_energy(pxb_ctx *c, double kappa, double chi, const double *u, double *E, double *dE_du) {
    PXB_TRY(need_ch_run(c, "pxb_ch_energy"));
    if (!u || !E) return fail(PXB_ERR_INVALID, "pxb_ch_energy: NULL buffer");
    pxb_ch_run_params p{};
    p.kappa = kappa;
    p.chi = chi;
    RunCtx r{c, c->g.n, 2LL * c->g.n, p};
    PXB_TRY(alloc_run(r));
    ChState &h = c->ch;
    PXB_TRY(h2d(c, h.U.p, u, sizeof(double) * (size_t)r.rows));
    PXB_TRY(energy(r, h.U.as<double>(), E, nullptr, dE_du ? h.dU.as<double>() : nullptr));
    if (dE_du) PXB_TRY(d2h(c, dE_du, h.dU.p, sizeof(double) * (size_t)r.rows));
    return sync(c);
}
