// explicit_pddo_frac on the device (reference ExplicitPDDOFracElement::preprocessIteration,
// src/ElmtSystem/ExplicitPDDOFracElement.cpp:239-299, and the central-difference loop of
// src/TimeStepping/TimeStepping.cpp:479-547).
//
// One warp per source node; lanes walk the node's contiguous family (bond id, health byte and the SoA
// Navier operator streams are read fully coalesced; neighbour positions/displacements are gathers that hit
// L1/L2 because families are spatially local).  Per step, a single launch does
//   damage   irreversible tensile (or |s|) critical-stretch failure of every live bond, decided in FP64;
//   force    L_i = sum_j h_ij P_ij (u_j - u_i) with P from the cached Gxx,Gyy,(Gzz),Gxy,(Gxz,Gyz);
//   update   a_i = (L_i + b)/rho, u^{n+1} = 2u^n - u^{n-1} + dt^2 a_i  (STEP), written into the u^{n-1}
//            buffer (ping-pong: every thread reads u^n only, so no grid-wide sync is needed);
//   BC pass  ghost/boundary targets whose final value derives from this node's freshly integrated value
//            (reflection, Neumann copy) or from constants (direct pins) are written by this node's warp,
//            reproducing the reference's sequential BC application (compiled on the host);
//   guard    the per-step max |u^{n+1}| (NaN-propagating) for the reference blow-up test.
#include <type_traits>

#include <algorithm>

#include "k_kernels.h"
#include "pxb_common.cuh"

namespace pxb {

namespace {

// reference stretch s = (|xi+eta| - |xi|)/|xi| with the reference's operation order (no contraction)
// critical stretch of bond t and its squared thresholds (1 +- s_c)^2: the element's uniform s_c, or with a variable
// horizon the bond's own s_c(0.5 (delta_i + delta_j)) (ExplicitPDDOFracElement.cpp:239-266); s_c <= 0 never breaks
struct BondStretch {
    double sc, hi2, lo2;
};
__device__ __forceinline__ BondStretch bond_stretch(const EpfArgs &a, long long t) {
    if (!a.sc_bond) return BondStretch{a.sc, a.sc_hi2, a.sc_lo2};
    const double sc = a.sc_bond[t];
    return BondStretch{sc, (1.0 + sc) * (1.0 + sc), sc < 1.0 ? (1.0 - sc) * (1.0 - sc) : 0.0};
}

__device__ __forceinline__ double ref_stretch(double y2, double r2) {
    const double r = sqrt(r2);
    return __ddiv_rn(__dsub_rn(sqrt(y2), r), r);
}

template <int DIM>
__device__ __forceinline__ double dot_rn(const double *a, const double *b) {
    double s = __dmul_rn(a[0], b[0]);
    s = __dadd_rn(s, __dmul_rn(a[1], b[1]));
    if constexpr (DIM == 3) s = __dadd_rn(s, __dmul_rn(a[2], b[2]));
    return s;
}

template <int DIM, bool MIXED>
__device__ __forceinline__ void load_G(const void *G, long long nb, long long t, double *g) {
    constexpr int NC = (DIM == 3) ? 6 : 3;
#pragma unroll
    for (int c = 0; c < NC; ++c) {
        if constexpr (MIXED) g[c] = (double)__ldg(static_cast<const float *>(G) + (size_t)c * nb + t);
        else g[c] = __ldg(static_cast<const double *>(G) + (size_t)c * nb + t);
    }
}

// P * eta with the reference's coefficient formulas (ExplicitPDDOFracElement.cpp:276-295)
template <int DIM>
__device__ __forceinline__ void navier_apply(const double *g, double C11, double C12, double C66, const double *e,
                                             double *out) {
    if constexpr (DIM == 3) {
        const double Gxx = g[0], Gyy = g[1], Gzz = g[2], Gxy = g[3], Gxz = g[4], Gyz = g[5];
        const double p11 = C11 * Gxx + C66 * (Gyy + Gzz);
        const double p22 = C11 * Gyy + C66 * (Gxx + Gzz);
        const double p33 = C11 * Gzz + C66 * (Gxx + Gyy);
        const double ac = C12 + C66;
        const double p12 = ac * Gxy, p13 = ac * Gxz, p23 = ac * Gyz;
        out[0] = p11 * e[0] + p12 * e[1] + p13 * e[2];
        out[1] = p12 * e[0] + p22 * e[1] + p23 * e[2];
        out[2] = p13 * e[0] + p23 * e[1] + p33 * e[2];
    } else {
        const double Gxx = g[0], Gyy = g[1], Gxy = g[2];
        const double p11 = C11 * Gxx + C66 * Gyy;
        const double p22 = C66 * Gxx + C11 * Gyy;
        const double pxy = (C12 + C66) * Gxy;
        out[0] = p11 * e[0] + pxy * e[1];
        out[1] = pxy * e[0] + p22 * e[1];
    }
}

template <int DIM>
__device__ __forceinline__ double pick(const double *v, int d) {
    double r = v[0];
#pragma unroll
    for (int k = 1; k < DIM; ++k)
        if (d == k) r = v[k];
    return r;
}

}  // namespace

// Schedule: LPN lanes per node (GPW = 32/LPN nodes per warp in flight) and UNR bonds per lane per pass.
// Every per-bond stream (health byte, neighbour id, operator values) of the UNR bonds is loaded before any
// branch, then the neighbour gathers of all UNR bonds are issued together, so a node costs about one DRAM
// round trip plus one (mostly L2-resident) gather round trip, and GPW*UNR*LPN bonds per warp are in flight.
template <int DIM, bool MIXED, int MODE, int LPN, int UNR>
__global__ void __launch_bounds__(kEpfThreads) epf_kernel(EpfArgs a) {
    using PosT = typename Vec<DIM>::T;
    using GT = typename std::conditional<MIXED, float, double>::type;
    constexpr int NC = (DIM == 3) ? 6 : 3;
    constexpr int WPB = kEpfThreads / kWarp;
    constexpr int GPW = kWarp / LPN;
    __shared__ unsigned long long s_umax[WPB];
    __shared__ unsigned long long s_broken[WPB];

    const int lane = threadIdx.x & 31;
    const int wib = threadIdx.x >> 5;
    const int gl = lane & (LPN - 1);   // lane within the node group
    const int grp = lane / LPN;        // node group within the warp
    const PosT *pos = static_cast<const PosT *>(a.pos);
    const GT *G = static_cast<const GT *>(a.G);
    double t_new = 0.0;
    if constexpr (MODE == EPF_STEP) t_new = a.t_sched[a.step_in_chunk];

    unsigned long long broken = 0;
    double umax = 0.0;
    const long long stride = (long long)gridDim.x * WPB * GPW;

    for (long long base = ((long long)blockIdx.x * WPB + wib) * GPW; base < a.n; base += stride) {
        const int i = (int)(base + grp);
        const bool act = i < a.n;
        int b0 = 0, b1 = 0;
        PosT xi{};
        double ui[DIM];
#pragma unroll
        for (int d = 0; d < DIM; ++d) ui[d] = 0.0;
        if (act) {
            b0 = __ldg(a.off + i);
            b1 = __ldg(a.off + i + 1);
            xi = pos[i];
#pragma unroll
            for (int d = 0; d < DIM; ++d) ui[d] = a.u[(size_t)i * DIM + d];
        }
        double L[DIM];
#pragma unroll
        for (int d = 0; d < DIM; ++d) L[d] = 0.0;

        for (int t0 = b0; t0 < b1; t0 += LPN * UNR) {
            uint8_t h[UNR];
            int j[UNR];
            GT g[UNR][NC];
#pragma unroll
            for (int q = 0; q < UNR; ++q) {
                const int t = t0 + q * LPN + gl;
                const bool ok = t < b1;
                h[q] = ok ? a.health[t] : (uint8_t)0;
                j[q] = ok ? __ldg(a.nbr + t) : i;
#pragma unroll
                for (int c = 0; c < NC; ++c) g[q][c] = ok ? __ldg(G + (size_t)c * a.nb + t) : GT(0);
            }
            PosT xj[UNR];
            double uj[UNR][DIM];
#pragma unroll
            for (int q = 0; q < UNR; ++q) {
                xj[q] = pos[j[q]];
#pragma unroll
                for (int d = 0; d < DIM; ++d) uj[q][d] = a.u[(size_t)j[q] * DIM + d];
            }
#pragma unroll
            for (int q = 0; q < UNR; ++q) {
                if (h[q] == 0) continue;
                double e[DIM];
#pragma unroll
                for (int d = 0; d < DIM; ++d) e[d] = __dsub_rn(uj[q][d], ui[d]);
                if constexpr (MODE != EPF_FORCE_FROZEN) {
                    if (a.damage) {
                        double xv[DIM], yv[DIM];
                        xv[0] = __dsub_rn(xj[q].x, xi.x);
                        xv[1] = __dsub_rn(xj[q].y, xi.y);
                        if constexpr (DIM == 3) xv[2] = __dsub_rn(xj[q].z, xi.z);
#pragma unroll
                        for (int d = 0; d < DIM; ++d) yv[d] = __dadd_rn(xv[d], e[d]);
                        const double r2 = dot_rn<DIM>(xv, xv);
                        const BondStretch bs = bond_stretch(a, t0 + q * LPN + gl);
                        if (r2 > 0.0 && bs.sc > 0.0) {
                            const double y2 = dot_rn<DIM>(yv, yv);
                            // fast squared test; the reference's own arithmetic decides bonds near threshold
                            const double band = 1.0e-6 * r2;
                            const double qh = y2 - bs.hi2 * r2;
                            bool brk;
                            if (a.tension_only) {
                                if (qh > band) brk = true;
                                else if (qh < -band) brk = false;
                                else brk = ref_stretch(y2, r2) > bs.sc;
                            } else {
                                const double ql = bs.lo2 * r2 - y2;
                                if (qh > band || ql > band) brk = true;
                                else if (qh < -band && ql < -band) brk = false;
                                else brk = fabs(ref_stretch(y2, r2)) > bs.sc;
                            }
                            if (brk) {
                                a.health[t0 + q * LPN + gl] = 0;
                                ++broken;
                                continue;
                            }
                        }
                    }
                }
                double gd[NC];
#pragma unroll
                for (int c = 0; c < NC; ++c) gd[c] = (double)g[q][c];
                double f[DIM];
                navier_apply<DIM>(gd, a.C11, a.C12, a.C66, e, f);
#pragma unroll
                for (int d = 0; d < DIM; ++d) L[d] += f[d];
            }
        }
#pragma unroll
        for (int d = 0; d < DIM; ++d) L[d] = group_sum<LPN>(L[d]);

        // node update: lane d of the group owns component d
        double unew = 0.0;
        if (act && gl < DIM) {
            const int d = gl;
            const double acc = __ddiv_rn(__dadd_rn(pick<DIM>(L, d), a.b[d]), a.rho);
            const size_t k = (size_t)i * DIM + d;
            if constexpr (MODE == EPF_RATE || MODE == EPF_FORCE_FROZEN) {
                a.accel[k] = acc;
            } else if constexpr (MODE == EPF_START) {
                const double v = a.v0 ? a.v0[k] : 0.0;
                a.u_other[k] = __dadd_rn(__dsub_rn(pick<DIM>(ui, d), __dmul_rn(a.dt, v)), __dmul_rn(a.dt2, acc));
            } else {
                const double uprev = a.u_other[k];
                unew = cd_next(pick<DIM>(ui, d), uprev, acc, a.dt2, a.var_step, a.cv_rho, a.cv_w);
                const bool owned = a.bc_own && ((a.bc_own[i] >> d) & 1);
                if (!owned) {
                    a.u_other[k] = unew;
                    umax = max_nan(umax, fabs(unew));
                }
            }
        }
        if constexpr (MODE == EPF_STEP) {
            if (a.bc_off) {
                double un[DIM];
#pragma unroll
                for (int d = 0; d < DIM; ++d) un[d] = __shfl_sync(kFull, unew, grp * LPN + d);
                const int e0 = act ? a.bc_off[i] : 0, e1 = act ? a.bc_off[i + 1] : 0;
                for (int e = e0 + gl; e < e1; e += LPN) {
                    const int comp = a.bc_comp[e];
                    const int form = a.bc_form[e];
                    // g = value + velocity*t in the reference's order (DirichletBC.cpp:135-137)
                    const double g1 = __dadd_rn(a.bc_val[e], __dmul_rn(a.bc_vel[e], t_new));
                    double v;
                    if (form == 0) {
                        v = pick<DIM>(un, comp);
                    } else if (form == 1) {
                        v = g1;
                    } else if (form == 2) {
                        v = __dsub_rn(__dmul_rn(2.0, g1), pick<DIM>(un, comp));
                    } else {
                        const double g2 = __dadd_rn(a.bc_val2[e], __dmul_rn(a.bc_vel2[e], t_new));
                        v = __dsub_rn(__dmul_rn(2.0, g1), g2);
                    }
                    a.u_other[(size_t)a.bc_tgt[e] * DIM + comp] = v;
                    umax = max_nan(umax, fabs(v));
                }
            }
        }
    }

    // block reductions, one atomic per block
    if constexpr (MODE == EPF_STEP) {
        umax = group_max_nan<kWarp>(umax);
        if (lane == 0) s_umax[wib] = dbl_key(umax);
    }
    unsigned long long bsum = broken;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) bsum += __shfl_xor_sync(kFull, bsum, o);
    if (lane == 0) s_broken[wib] = bsum;
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned long long bb = 0, mm = 0;
        for (int w = 0; w < WPB; ++w) {
            bb += s_broken[w];
            if constexpr (MODE == EPF_STEP) mm = s_umax[w] > mm ? s_umax[w] : mm;
        }
        if (bb && a.n_broken) atomicAdd(a.n_broken, bb);
        if constexpr (MODE == EPF_STEP) {
            if (a.umax) atomicMax(a.umax + a.step_in_chunk, mm);
        }
    }
}

// ---- CSR-stream schedule ---------------------------------------------------------------------------------
// A block takes a tile of NB consecutive nodes; their families form one contiguous bond range, which all
// threads stream flat (bond t -> thread t mod blockDim), UNR bonds per thread per pass with every per-bond load
// issued before any branch.  A shared-memory map gives each bond its tile-local node; partial forces go to
// shared-memory FP64 accumulators.  A short node phase then does the update and the BC pass.  Every bond is
// independent, so registers stay low and many bonds are in flight per SM.
constexpr int kStreamMap = 4096;   // max bonds per tile (host checks NB * max family <= this)

template <int DIM, bool MIXED, int MODE, int NB, int UNR>
__global__ void __launch_bounds__(kEpfThreads) epf_stream_kernel(EpfArgs a) {
    using PosT = typename Vec<DIM>::T;
    using GT = typename std::conditional<MIXED, float, double>::type;
    constexpr int NC = (DIM == 3) ? 6 : 3;
    constexpr int WPB = kEpfThreads / kWarp;
    __shared__ int s_off[NB + 1];
    __shared__ PosT s_x[NB];
    __shared__ double s_u[NB][DIM];
    __shared__ double s_L[NB][DIM];
    __shared__ double s_un[NB][DIM];
    __shared__ unsigned char s_node[kStreamMap];
    __shared__ unsigned long long s_umax[WPB];
    __shared__ unsigned long long s_broken[WPB];

    const int tid = threadIdx.x;
    const int lane = tid & 31;
    const int wib = tid >> 5;
    const PosT *pos = static_cast<const PosT *>(a.pos);
    const GT *G = static_cast<const GT *>(a.G);
    double t_new = 0.0;
    if constexpr (MODE == EPF_STEP) t_new = a.t_sched[a.step_in_chunk];
    unsigned long long broken = 0;
    double umax = 0.0;
    const int ntiles = (a.n + NB - 1) / NB;

    for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const int n0 = tile * NB;
        const int cnt = min(NB, a.n - n0);
        // ---- phase A: node data of the tile ----
        if (tid <= cnt) s_off[tid] = __ldg(a.off + n0 + tid);
        if (tid < cnt) {
            s_x[tid] = pos[n0 + tid];
#pragma unroll
            for (int d = 0; d < DIM; ++d) {
                s_u[tid][d] = a.u[(size_t)(n0 + tid) * DIM + d];
                s_L[tid][d] = 0.0;
            }
        }
        __syncthreads();
        const int tb = s_off[0], te = s_off[cnt];
        // bond -> tile-local node map (warp per node, lanes over its bonds)
        for (int k = wib; k < cnt; k += WPB)
            for (int t = s_off[k] + lane; t < s_off[k + 1]; t += kWarp) s_node[t - tb] = (unsigned char)k;
        __syncthreads();
        // ---- phase B: the tile's bonds, flat ----
        for (int t0 = tb + tid; t0 < te; t0 += kEpfThreads * UNR) {
            uint8_t h[UNR];
            int j[UNR];
            GT g[UNR][NC];
#pragma unroll
            for (int q = 0; q < UNR; ++q) {
                const int t = t0 + q * kEpfThreads;
                const bool ok = t < te;
                h[q] = ok ? a.health[t] : (uint8_t)0;
                j[q] = ok ? __ldg(a.nbr + t) : n0;
#pragma unroll
                for (int c = 0; c < NC; ++c) g[q][c] = ok ? __ldg(G + (size_t)c * a.nb + t) : GT(0);
            }
            PosT xj[UNR];
            double uj[UNR][DIM];
#pragma unroll
            for (int q = 0; q < UNR; ++q) {
                xj[q] = pos[j[q]];
#pragma unroll
                for (int d = 0; d < DIM; ++d) uj[q][d] = a.u[(size_t)j[q] * DIM + d];
            }
#pragma unroll
            for (int q = 0; q < UNR; ++q) {
                if (h[q] == 0) continue;
                const int t = t0 + q * kEpfThreads;
                const int k = s_node[t - tb];
                const PosT xi = s_x[k];
                double e[DIM];
#pragma unroll
                for (int d = 0; d < DIM; ++d) e[d] = __dsub_rn(uj[q][d], s_u[k][d]);
                if constexpr (MODE != EPF_FORCE_FROZEN) {
                    if (a.damage) {
                        double xv[DIM], yv[DIM];
                        xv[0] = __dsub_rn(xj[q].x, xi.x);
                        xv[1] = __dsub_rn(xj[q].y, xi.y);
                        if constexpr (DIM == 3) xv[2] = __dsub_rn(xj[q].z, xi.z);
#pragma unroll
                        for (int d = 0; d < DIM; ++d) yv[d] = __dadd_rn(xv[d], e[d]);
                        const double r2 = dot_rn<DIM>(xv, xv);
                        const BondStretch bs = bond_stretch(a, t);
                        if (r2 > 0.0 && bs.sc > 0.0) {
                            const double y2 = dot_rn<DIM>(yv, yv);
                            const double band = 1.0e-6 * r2;
                            const double qh = y2 - bs.hi2 * r2;
                            bool brk;
                            if (a.tension_only) {
                                if (qh > band) brk = true;
                                else if (qh < -band) brk = false;
                                else brk = ref_stretch(y2, r2) > bs.sc;
                            } else {
                                const double ql = bs.lo2 * r2 - y2;
                                if (qh > band || ql > band) brk = true;
                                else if (qh < -band && ql < -band) brk = false;
                                else brk = fabs(ref_stretch(y2, r2)) > bs.sc;
                            }
                            if (brk) {
                                a.health[t] = 0;
                                ++broken;
                                continue;
                            }
                        }
                    }
                }
                double gd[NC];
#pragma unroll
                for (int c = 0; c < NC; ++c) gd[c] = (double)g[q][c];
                double f[DIM];
                navier_apply<DIM>(gd, a.C11, a.C12, a.C66, e, f);
#pragma unroll
                for (int d = 0; d < DIM; ++d) atomicAdd(&s_L[k][d], f[d]);
            }
        }
        __syncthreads();
        // ---- phase C: node update, one thread per (node, component) ----
        if (tid < cnt * DIM) {
            const int k = tid / DIM, d = tid - k * DIM;
            const int i = n0 + k;
            const double acc = __ddiv_rn(__dadd_rn(s_L[k][d], a.b[d]), a.rho);
            const size_t idx = (size_t)i * DIM + d;
            if constexpr (MODE == EPF_RATE || MODE == EPF_FORCE_FROZEN) {
                a.accel[idx] = acc;
            } else if constexpr (MODE == EPF_START) {
                const double v = a.v0 ? a.v0[idx] : 0.0;
                a.u_other[idx] = __dadd_rn(__dsub_rn(s_u[k][d], __dmul_rn(a.dt, v)), __dmul_rn(a.dt2, acc));
            } else {
                const double uprev = a.u_other[idx];
                const double unew = cd_next(s_u[k][d], uprev, acc, a.dt2, a.var_step, a.cv_rho, a.cv_w);
                s_un[k][d] = unew;
                const bool owned = a.bc_own && ((a.bc_own[i] >> d) & 1);
                if (!owned) {
                    a.u_other[idx] = unew;
                    umax = max_nan(umax, fabs(unew));
                }
            }
        }
        if constexpr (MODE == EPF_STEP) {
            if (a.bc_off) {
                __syncthreads();
                // BC entries executed by the tile: thread per node walks its (few) entries
                if (tid < cnt) {
                    const int i = n0 + tid;
                    for (int e = a.bc_off[i]; e < a.bc_off[i + 1]; ++e) {
                        const int comp = a.bc_comp[e];
                        const int form = a.bc_form[e];
                        const double g1 = __dadd_rn(a.bc_val[e], __dmul_rn(a.bc_vel[e], t_new));
                        double v;
                        if (form == 0) v = s_un[tid][comp];
                        else if (form == 1) v = g1;
                        else if (form == 2) v = __dsub_rn(__dmul_rn(2.0, g1), s_un[tid][comp]);
                        else v = __dsub_rn(__dmul_rn(2.0, g1), __dadd_rn(a.bc_val2[e], __dmul_rn(a.bc_vel2[e], t_new)));
                        a.u_other[(size_t)a.bc_tgt[e] * DIM + comp] = v;
                        umax = max_nan(umax, fabs(v));
                    }
                }
            }
        }
        __syncthreads();
    }

    if constexpr (MODE == EPF_STEP) {
        umax = group_max_nan<kWarp>(umax);
        if (lane == 0) s_umax[wib] = dbl_key(umax);
    }
    unsigned long long bsum = broken;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) bsum += __shfl_xor_sync(kFull, bsum, o);
    if (lane == 0) s_broken[wib] = bsum;
    __syncthreads();
    if (tid == 0) {
        unsigned long long bb = 0, mm = 0;
        for (int w = 0; w < WPB; ++w) {
            bb += s_broken[w];
            if constexpr (MODE == EPF_STEP) mm = s_umax[w] > mm ? s_umax[w] : mm;
        }
        if (bb && a.n_broken) atomicAdd(a.n_broken, bb);
        if constexpr (MODE == EPF_STEP) {
            if (a.umax) atomicMax(a.umax + a.step_in_chunk, mm);
        }
    }
}

// ---- bond-force adjoint with a frozen damage mask ---------------------------------------------------------
// Forward: a_i = (L_i + b)/rho, L_i = sum_t h_t P_t (u_j - u_i) with P_t symmetric.  For abar = dJ/da,
// Lbar = abar/rho and
//   ubar_m = sum_{t in fam(m)} ( h_rev(t) P_rev(t) Lbar_{j_t} - h_t P_t Lbar_m )      (gather via rev)
//   dJ/dC_k = sum_i sum_t h_t Lbar_i . (dP_t/dC_k) eta_t
// REV: the reverse-only mode (EpfAdjArgs::SG with GR and hrev), its own instantiation (fewer registers)
template <int DIM, bool MIXED, bool REV>
__global__ void __launch_bounds__(kEpfThreads, REV ? 4 : 1) epf_adjoint_kernel(EpfAdjArgs a) {
    constexpr int WPB = kEpfThreads / kWarp;
    constexpr int NC = (DIM == 3) ? 6 : 3;
    __shared__ double s_dC[WPB][3];
    const int lane = threadIdx.x & 31;
    const int wib = threadIdx.x >> 5;
    double dC[3] = {0.0, 0.0, 0.0};
    for (int m = blockIdx.x * WPB + wib; m < a.n; m += gridDim.x * WPB) {
        double Lm[DIM], um[DIM], U[DIM];
        const double lscale = a.scale * a.inv_rho;
#pragma unroll
        for (int d = 0; d < DIM; ++d) {
            Lm[d] = a.abar[(size_t)m * DIM + d] * lscale;
            um[d] = a.u[(size_t)m * DIM + d];
            U[d] = 0.0;
        }
        // dJ/dC of one bond: L (the source node's scaled adjoint) . dP/dC (G) e, e = u_target - u_source
        auto acc_dC = [&](const double *L, const double *g, const double *e) {
            if constexpr (DIM == 3) {
                const double Gxx = g[0], Gyy = g[1], Gzz = g[2], Gxy = g[3], Gxz = g[4], Gyz = g[5];
                dC[0] += L[0] * Gxx * e[0] + L[1] * Gyy * e[1] + L[2] * Gzz * e[2];
                dC[1] += L[0] * (Gxy * e[1] + Gxz * e[2]) + L[1] * (Gxy * e[0] + Gyz * e[2]) +
                         L[2] * (Gxz * e[0] + Gyz * e[1]);
                dC[2] += L[0] * ((Gyy + Gzz) * e[0] + Gxy * e[1] + Gxz * e[2]) +
                         L[1] * (Gxy * e[0] + (Gxx + Gzz) * e[1] + Gyz * e[2]) +
                         L[2] * (Gxz * e[0] + Gyz * e[1] + (Gxx + Gyy) * e[2]);
            } else {
                const double Gxx = g[0], Gyy = g[1], Gxy = g[2];
                dC[0] += L[0] * Gxx * e[0] + L[1] * Gyy * e[1];
                dC[1] += L[0] * Gxy * e[1] + L[1] * Gxy * e[0];
                dC[2] += L[0] * (Gyy * e[0] + Gxy * e[1]) + L[1] * (Gxy * e[0] + Gxx * e[1]);
            }
        };
        constexpr bool rev_only = REV;
        if constexpr (REV) {
            // the reverse bond (j -> m): its operators and health from the bond-ordered copies, the source's
            // adjoint and displacement gathered; its term of (da/du)^T and of dJ/dC
            for (int t = a.off[m] + lane; t < a.off[m + 1]; t += kWarp) {
                const int j = __ldg(a.nbr + t);
                double gr[NC], Lj[DIM], e[DIM], f[DIM];
                load_G<DIM, MIXED>(a.GR, a.nb, t, gr);
                const bool hr = a.hrev[t] != 0;
#pragma unroll
                for (int d = 0; d < DIM; ++d) {
                    Lj[d] = a.abar[(size_t)j * DIM + d] * lscale;
                    e[d] = um[d] - a.u[(size_t)j * DIM + d];
                }
                if (hr) {
                    navier_apply<DIM>(gr, a.C11, a.C12, a.C66, Lj, f);
#pragma unroll
                    for (int d = 0; d < DIM; ++d) U[d] += f[d];
                    acc_dC(Lj, gr, e);
                }
            }
        }
        for (int t = a.off[m] + lane; !REV && t < a.off[m + 1]; t += kWarp) {
            const int j = __ldg(a.nbr + t);
            const int r = a.hrev ? 0 : __ldg(a.rev + t);
            double g[NC], f[DIM];
            if (a.GR) {
                // the reverse bond's operators and health from bond-ordered copies (coalesced; zero without a
                // reverse bond): every load of the bond is issued up front, the masks applied afterwards
                double gr[NC], Lj[DIM];
                load_G<DIM, MIXED>(a.GR, a.nb, t, gr);
                const bool hr = a.hrev ? a.hrev[t] != 0 : (r >= 0 && a.health[r]);
#pragma unroll
                for (int d = 0; d < DIM; ++d) Lj[d] = a.abar[(size_t)j * DIM + d] * lscale;
                navier_apply<DIM>(gr, a.C11, a.C12, a.C66, Lj, f);
#pragma unroll
                for (int d = 0; d < DIM; ++d) U[d] += hr ? f[d] : 0.0;
            } else if (r >= 0 && a.health[r]) {
                double Lj[DIM];
#pragma unroll
                for (int d = 0; d < DIM; ++d) Lj[d] = a.abar[(size_t)j * DIM + d] * lscale;
                load_G<DIM, MIXED>(a.G, a.nb, r, g);
                navier_apply<DIM>(g, a.C11, a.C12, a.C66, Lj, f);
#pragma unroll
                for (int d = 0; d < DIM; ++d) U[d] += f[d];
            }
            if (a.health[t]) {
                load_G<DIM, MIXED>(a.G, a.nb, t, g);
                navier_apply<DIM>(g, a.C11, a.C12, a.C66, Lm, f);
#pragma unroll
                for (int d = 0; d < DIM; ++d) U[d] -= f[d];
                double e[DIM];
#pragma unroll
                for (int d = 0; d < DIM; ++d) e[d] = a.u[(size_t)j * DIM + d] - um[d];
                acc_dC(Lm, g, e);
            }
        }
#pragma unroll
        for (int d = 0; d < DIM; ++d) U[d] = group_sum<kWarp>(U[d]);
        if constexpr (rev_only) {  // the own bonds' term, - (sum_t h_t P_t) Lm, from the node's operator sums
            double sg[NC], f[DIM];
#pragma unroll
            for (int c = 0; c < NC; ++c) sg[c] = __ldg(a.SG + (size_t)m * NC + c);
            navier_apply<DIM>(sg, a.C11, a.C12, a.C66, Lm, f);
#pragma unroll
            for (int d = 0; d < DIM; ++d) U[d] -= f[d];
        }
        if (lane < DIM) {
            const size_t k = (size_t)m * DIM + lane;
            if (a.step) {
                const double w = a.abar[k];
                const double r = a.rin ? a.rin[k] : 0.0;
                if (a.rout) a.rout[k] = a.c_o * w;
                a.ubar[k] = a.c_r * r + a.c_w * w + pick<DIM>(U, lane);
            } else {
                a.ubar[k] = pick<DIM>(U, lane);
            }
        }
    }
#pragma unroll
    for (int k = 0; k < 3; ++k) dC[k] = group_sum<kWarp>(dC[k]);
    if (lane == 0) { s_dC[wib][0] = dC[0]; s_dC[wib][1] = dC[1]; s_dC[wib][2] = dC[2]; }
    __syncthreads();
    if (threadIdx.x < 3 && a.dC) {
        double v = 0.0;
        for (int w = 0; w < WPB; ++w) v += s_dC[w][threadIdx.x];
        atomicAdd(a.dC + threadIdx.x, v);
    }
}

// ---- the highest neighbour id of each node chunk (the pipelined rate call's upload dependencies) ---------------
constexpr int kReachBlocks = 256;  // blocks per chunk
__global__ void chunk_reach_kernel(const int *off, const int *nbr, const int *bounds, int *reach) {
    const int k = blockIdx.x / kReachBlocks, part = blockIdx.x % kReachBlocks;
    const int t0 = off[bounds[k]], t1 = off[bounds[k + 1]];
    int r = 0;
    for (int t = t0 + part * blockDim.x + threadIdx.x; t < t1; t += kReachBlocks * blockDim.x) r = max(r, nbr[t]);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) r = max(r, __shfl_xor_sync(kFull, r, o));
    if ((threadIdx.x & 31) == 0) atomicMax(reach + k, r);
}

cudaError_t launch_chunk_reach(const int *off, const int *nbr, const int *bounds, int nchunks, int *reach,
                               cudaStream_t s) {
    chunk_reach_kernel<<<(nchunks > 0 ? nchunks : 1) * kReachBlocks, 256, 0, s>>>(off, nbr, bounds, reach);
    return cudaGetLastError();
}

// ---- per-node sums of the healthy own bonds' operators (the adjoint's own-bond term under a frozen mask) --------
template <int NC, bool MIXED>
__global__ void own_sum_kernel(int n, const int *off, const int *rev, const uint8_t *health, const void *G,
                               long long ldb, double *SG, unsigned int *missing) {
    const int lane = threadIdx.x & 31;
    unsigned miss = 0;
    for (int m = (int)((blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5); m < n;
         m += (int)((gridDim.x * (long long)blockDim.x) >> 5)) {
        double s[NC];
#pragma unroll
        for (int c = 0; c < NC; ++c) s[c] = 0.0;
        for (int t = off[m] + lane; t < off[m + 1]; t += kWarp) {
            if (rev[t] < 0) ++miss;
            if (!health[t]) continue;
#pragma unroll
            for (int c = 0; c < NC; ++c) {
                if constexpr (MIXED) s[c] += (double)static_cast<const float *>(G)[(size_t)c * ldb + t];
                else s[c] += static_cast<const double *>(G)[(size_t)c * ldb + t];
            }
        }
#pragma unroll
        for (int c = 0; c < NC; ++c) {
            const double v = group_sum<kWarp>(s[c]);
            if (lane == c) SG[(size_t)m * NC + c] = v;
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) miss += __shfl_xor_sync(kFull, miss, o);
    if (lane == 0 && miss) atomicAdd(missing, miss);
}

cudaError_t launch_own_sums(int n, int dim, bool mixed, const int *off, const int *rev, const uint8_t *health,
                            const void *G, long long ldb, double *SG, unsigned int *missing, cudaStream_t s) {
    const int grid = (int)std::min<long long>(((long long)n * kWarp + 255) / 256, 148LL * 16);
    const int g = grid > 0 ? grid : 1;
    if (dim == 3) {
        if (mixed) own_sum_kernel<6, true><<<g, 256, 0, s>>>(n, off, rev, health, G, ldb, SG, missing);
        else own_sum_kernel<6, false><<<g, 256, 0, s>>>(n, off, rev, health, G, ldb, SG, missing);
    } else {
        if (mixed) own_sum_kernel<3, true><<<g, 256, 0, s>>>(n, off, rev, health, G, ldb, SG, missing);
        else own_sum_kernel<3, false><<<g, 256, 0, s>>>(n, off, rev, health, G, ldb, SG, missing);
    }
    return cudaGetLastError();
}

// ---- the Navier operators in reverse-bond order: GR[c][t] = G[c][rev t] (0 without a reverse bond) -------------
template <typename T>
__global__ void reverse_gather_kernel(const T *G, T *GR, const int *rev, long long nb, long long ldb, int nc) {
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < nb; t += (long long)gridDim.x * blockDim.x) {
        const int r = rev[t];
        for (int c = 0; c < nc; ++c) GR[(size_t)c * ldb + t] = r >= 0 ? G[(size_t)c * ldb + r] : T(0);
    }
}

__global__ void reverse_health_kernel(const uint8_t *health, const int *rev, uint8_t *hr, long long nb) {
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < nb; t += (long long)gridDim.x * blockDim.x) {
        const int r = rev[t];
        hr[t] = r >= 0 ? health[r] : (uint8_t)0;
    }
}

cudaError_t launch_reverse_health(const uint8_t *health, const int *rev, uint8_t *hr, long long nb, cudaStream_t s) {
    const int grid = (int)std::min<long long>((nb + 255) / 256, 148LL * 16);
    reverse_health_kernel<<<grid > 0 ? grid : 1, 256, 0, s>>>(health, rev, hr, nb);
    return cudaGetLastError();
}

cudaError_t launch_reverse_gather(const void *G, void *GR, const int *rev, long long nb, long long ldb, int dim,
                                  bool mixed, cudaStream_t s) {
    const int nc = dim == 3 ? 6 : 3;
    const int grid = (int)std::min<long long>((nb + 255) / 256, 148LL * 16);
    if (mixed)
        reverse_gather_kernel<float><<<grid > 0 ? grid : 1, 256, 0, s>>>(static_cast<const float *>(G),
                                                                       static_cast<float *>(GR), rev, nb, ldb, nc);
    else
        reverse_gather_kernel<double><<<grid > 0 ? grid : 1, 256, 0, s>>>(static_cast<const double *>(G),
                                                                         static_cast<double *>(GR), rev, nb, ldb, nc);
    return cudaGetLastError();
}

// ---- transpose of the BC program (the adjoint of a step's BC pass) --------------------------------------------
// The forward pass sets u^{n+1}[target] = coef w[src] + const per entry (form 0: coef +1, form 2: -1, forms 1 and 3:
// constants) and keeps w elsewhere; entries are grouped by the node that executes them, which for forms 0 and 2 is
// the source, so the transpose is a gather without atomics: thread per node.
template <int DIM>
__global__ void bc_transpose_kernel(EpfArgs b, int n, const double *a, double *w, const double *u, double *uw) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const unsigned own = b.bc_own ? b.bc_own[i] : 0u;
        double v[DIM];
#pragma unroll
        for (int d = 0; d < DIM; ++d) v[d] = ((own >> d) & 1u) ? 0.0 : a[(size_t)i * DIM + d];
        if (b.bc_off) {
            for (int e = b.bc_off[i]; e < b.bc_off[i + 1]; ++e) {
                const int form = b.bc_form[e];
                if (form != 0 && form != 2) continue;
                const int comp = b.bc_comp[e];
                const double x = a[(size_t)b.bc_tgt[e] * DIM + comp];
#pragma unroll
                for (int d = 0; d < DIM; ++d)
                    if (d == comp) v[d] += form == 0 ? x : -x;
            }
        }
#pragma unroll
        for (int d = 0; d < DIM; ++d) w[(size_t)i * DIM + d] = v[d];
        if (uw) {  // the staged adjoint's gather rows: (u_i, w_i) interleaved
#pragma unroll
            for (int d = 0; d < DIM; ++d) {
                uw[(size_t)i * 2 * DIM + d] = u[(size_t)i * DIM + d];
                uw[(size_t)i * 2 * DIM + DIM + d] = v[d];
            }
        }
    }
}

cudaError_t launch_bc_transpose(const EpfArgs &bc, int n, int dim, const double *a, double *w, cudaStream_t s,
                                const double *u, double *uw) {
    const int grid = (int)std::min<long long>(((long long)n + 255) / 256, 148LL * 16);
    if (dim == 3) bc_transpose_kernel<3><<<grid > 0 ? grid : 1, 256, 0, s>>>(bc, n, a, w, u, uw);
    else bc_transpose_kernel<2><<<grid > 0 ? grid : 1, 256, 0, s>>>(bc, n, a, w, u, uw);
    return cudaGetLastError();
}

// ---- packed Navier coefficients for the staged step kernels ----------------------------------------------
// Per bond the 2D operator is [[p11, pxy], [pxy, p22]] (3D: symmetric 3x3); the step kernels read it directly
// instead of forming it from (Gxx, Gyy, Gxy) and (C11, C12, C66) on every step.  The sums are evaluated in
// FP64 from the stored G and rounded once to the storage type.
template <int DIM, typename T>
__global__ void navier_pack_kernel(const T *G, T *P, long long ldb, double C11, double C12, double C66) {
    const double ac = C12 + C66;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < ldb; t += (long long)gridDim.x * blockDim.x) {
        if constexpr (DIM == 3) {
            const double Gxx = G[t], Gyy = G[ldb + t], Gzz = G[2 * ldb + t];
            P[t] = (T)(C11 * Gxx + C66 * (Gyy + Gzz));
            P[ldb + t] = (T)(C11 * Gyy + C66 * (Gxx + Gzz));
            P[2 * ldb + t] = (T)(C11 * Gzz + C66 * (Gxx + Gyy));
            P[3 * ldb + t] = (T)(ac * (double)G[3 * ldb + t]);
            P[4 * ldb + t] = (T)(ac * (double)G[4 * ldb + t]);
            P[5 * ldb + t] = (T)(ac * (double)G[5 * ldb + t]);
        } else {
            const double Gxx = G[t], Gyy = G[ldb + t];
            P[t] = (T)(C11 * Gxx + C66 * Gyy);
            P[ldb + t] = (T)(C66 * Gxx + C11 * Gyy);
            P[2 * ldb + t] = (T)(ac * (double)G[2 * ldb + t]);
        }
    }
}

template <int DIM>
__global__ void bond_vector_kernel(int n, const int *off, const int *nbr, const void *pos, long long ldb, float *xib,
                                   unsigned long long *r2min_key) {
    using PosT = typename Vec<DIM>::T;
    const PosT *p = static_cast<const PosT *>(pos);
    double r2min = __longlong_as_double(0x7ff0000000000000LL);  // +inf
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const PosT xi = p[i];
        for (int t = off[i]; t < off[i + 1]; ++t) {
            const PosT xj = p[nbr[t]];
            const double dx = __dsub_rn(xj.x, xi.x), dy = __dsub_rn(xj.y, xi.y);
            xib[t] = (float)dx;
            xib[ldb + t] = (float)dy;
            double r2 = __dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy));
            if constexpr (DIM == 3) {
                const double dz = __dsub_rn(xj.z, xi.z);
                xib[2 * ldb + t] = (float)dz;
                r2 = __dadd_rn(r2, __dmul_rn(dz, dz));
            }
            if (r2 > 0.0 && r2 < r2min) r2min = r2;
        }
    }
    if (r2min_key) {  // positive doubles order as their bit patterns
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) r2min = fmin(r2min, __shfl_xor_sync(kFull, r2min, o));
        if ((threadIdx.x & 31) == 0) atomicMin(r2min_key, dbl_key(r2min));
    }
}

cudaError_t launch_bond_vectors(int n, int dim, const int *off, const int *nbr, const void *pos, long long ldb,
                                float *xib, unsigned long long *r2min_key, cudaStream_t s) {
    const int grid = (int)std::min<long long>(((long long)n + 255) / 256, 148LL * 16);
    if (dim == 3) bond_vector_kernel<3><<<grid > 0 ? grid : 1, 256, 0, s>>>(n, off, nbr, pos, ldb, xib, r2min_key);
    else bond_vector_kernel<2><<<grid > 0 ? grid : 1, 256, 0, s>>>(n, off, nbr, pos, ldb, xib, r2min_key);
    return cudaGetLastError();
}

cudaError_t launch_navier_pack(const void *G, void *P, long long ldb, int dim, bool mixed, double C11, double C12,
                               double C66, cudaStream_t s) {
    const int grid = (int)std::min<long long>((ldb + 255) / 256, 148LL * 16);
    if (dim == 3) {
        if (mixed) navier_pack_kernel<3, float><<<grid, 256, 0, s>>>((const float *)G, (float *)P, ldb, C11, C12, C66);
        else navier_pack_kernel<3, double><<<grid, 256, 0, s>>>((const double *)G, (double *)P, ldb, C11, C12, C66);
    } else {
        if (mixed) navier_pack_kernel<2, float><<<grid, 256, 0, s>>>((const float *)G, (float *)P, ldb, C11, C12, C66);
        else navier_pack_kernel<2, double><<<grid, 256, 0, s>>>((const double *)G, (double *)P, ldb, C11, C12, C66);
    }
    return cudaGetLastError();
}


// schedule variants (LPN lanes per node, UNR bonds per lane per pass); index = EpfArgs-independent id
// persistent grid: every block resident (SM count x occupancy of this instantiation), capped by the work
template <typename K>
static int resident_grid(K kernel, int n, int nodes_per_block, int &cap) {
    if (cap == 0) {  // cap: the caller's cache, one per kernel instantiation
        int dev = 0, sms = 148, per_sm = 1;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, kEpfThreads, 0);
        cap = sms * (per_sm > 0 ? per_sm : 1);
    }
    const long long need = ((long long)n + nodes_per_block - 1) / nodes_per_block;
    return (int)(need < cap ? (need > 0 ? need : 1) : cap);
}

// the adjoint kernel's own resident grid (one warp per node, grid-stride), capped by the node count
template <int DIM, bool MIXED>
static cudaError_t launch_adj(const EpfAdjArgs &a, cudaStream_t s) {
    if (a.SG && a.GR && a.hrev) {
        auto k = epf_adjoint_kernel<DIM, MIXED, true>;
        static int cap = 0;
        const int grid = resident_grid(k, a.n, kEpfThreads / kWarp, cap);
        k<<<grid, kEpfThreads, 0, s>>>(a);
    } else {
        auto k = epf_adjoint_kernel<DIM, MIXED, false>;
        static int cap = 0;
        const int grid = resident_grid(k, a.n, kEpfThreads / kWarp, cap);
        k<<<grid, kEpfThreads, 0, s>>>(a);
    }
    return cudaGetLastError();
}

cudaError_t launch_epf_adjoint(const EpfAdjArgs &a, int dim, bool mixed, int, cudaStream_t s) {
    if (dim == 2) return mixed ? launch_adj<2, true>(a, s) : launch_adj<2, false>(a, s);
    return mixed ? launch_adj<3, true>(a, s) : launch_adj<3, false>(a, s);
}

template <int DIM, bool MIXED, int MODE, int LPN, int UNR>
static cudaError_t launch_m(const EpfArgs &a, cudaStream_t s) {
    auto k = epf_kernel<DIM, MIXED, MODE, LPN, UNR>;
    static int cap = 0;
    const int grid = resident_grid(k, a.n, (kEpfThreads / kWarp) * (kWarp / LPN), cap);
    k<<<grid, kEpfThreads, 0, s>>>(a);
    return cudaGetLastError();
}

template <int DIM, bool MIXED, int MODE, int NB, int UNR>
static cudaError_t launch_s(const EpfArgs &a, cudaStream_t s) {
    auto k = epf_stream_kernel<DIM, MIXED, MODE, NB, UNR>;
    static int cap = 0;
    const int grid = resident_grid(k, a.n, NB, cap);
    k<<<grid, kEpfThreads, 0, s>>>(a);
    return cudaGetLastError();
}

template <int DIM, bool MIXED, int NB, int UNR>
static cudaError_t launch_sv(const EpfArgs &a, int mode, cudaStream_t s) {
    switch (mode) {
        case EPF_RATE: return launch_s<DIM, MIXED, EPF_RATE, NB, UNR>(a, s);
        case EPF_START: return launch_s<DIM, MIXED, EPF_START, NB, UNR>(a, s);
        case EPF_STEP: return launch_s<DIM, MIXED, EPF_STEP, NB, UNR>(a, s);
        case EPF_FORCE_FROZEN: return launch_s<DIM, MIXED, EPF_FORCE_FROZEN, NB, UNR>(a, s);
        default: return cudaErrorInvalidValue;
    }
}

template <int DIM, bool MIXED, int LPN, int UNR>
static cudaError_t launch_v(const EpfArgs &a, int mode, cudaStream_t s) {
    switch (mode) {
        case EPF_RATE: return launch_m<DIM, MIXED, EPF_RATE, LPN, UNR>(a, s);
        case EPF_START: return launch_m<DIM, MIXED, EPF_START, LPN, UNR>(a, s);
        case EPF_STEP: return launch_m<DIM, MIXED, EPF_STEP, LPN, UNR>(a, s);
        case EPF_FORCE_FROZEN: return launch_m<DIM, MIXED, EPF_FORCE_FROZEN, LPN, UNR>(a, s);
        default: return cudaErrorInvalidValue;
    }
}

// 2D: families of ~12..30 bonds; 3D: ~40..122.  Variants 3/4 are the CSR-stream schedule (lanes per node
// reported as 0; tile sizes in nodes below).
static constexpr int kLpn2[5] = {32, 16, 8, 0, 0};
static constexpr int kLpn3[5] = {32, 32, 16, 0, 0};
static constexpr int kTile2[5] = {0, 0, 0, 64, 128};
static constexpr int kTile3[5] = {0, 0, 0, 16, 32};

template <int DIM, bool MIXED>
static cudaError_t launch_dm(const EpfArgs &a, int mode, int variant, cudaStream_t s) {
    if constexpr (DIM == 2) {
        switch (variant) {
            case 0: return launch_v<2, MIXED, 32, 1>(a, mode, s);
            case 1: return launch_v<2, MIXED, 16, 2>(a, mode, s);
            case 2: return launch_v<2, MIXED, 8, 4>(a, mode, s);
            case 3: return launch_sv<2, MIXED, 64, 2>(a, mode, s);
            default: return launch_sv<2, MIXED, 128, 2>(a, mode, s);
        }
    } else {
        switch (variant) {
            case 0: return launch_v<3, MIXED, 32, 1>(a, mode, s);
            case 1: return launch_v<3, MIXED, 32, 2>(a, mode, s);
            case 2: return launch_v<3, MIXED, 16, 2>(a, mode, s);
            case 3: return launch_sv<3, MIXED, 16, 2>(a, mode, s);
            default: return launch_sv<3, MIXED, 32, 2>(a, mode, s);
        }
    }
}

bool epf_is_tma(int variant) { return variant >= 5; }

int epf_tma_maxb(int dim, int variant, int max_family) {
    const int nt = epf_tma_tile_nodes(dim, variant - 5);
    const long long b = (long long)nt * max_family + 32;
    return (int)((b + 31) / 32 * 32);
}

cudaError_t launch_epf(const EpfArgs &a, int dim, bool mixed, int mode, int variant, cudaStream_t s) {
    if (a.sc_bond && epf_is_tma(variant)) variant = 1;  // per-bond critical stretch: the lane-group kernels read it
    if (epf_is_tma(variant)) {
        if (mode == EPF_STEP) return launch_epf_tma(a, dim, mixed, variant - 5, s);
        if (mode == EPF_RATE && a.accel) {
            EpfArgs r = a;
            r.rate = 1;
            return launch_epf_tma(r, dim, mixed, variant - 5, s);
        }
        variant = 1;  // the staged kernel implements the step and the rate; START / FORCE_FROZEN use variant 1
    }
    if (dim == 2) return mixed ? launch_dm<2, true>(a, mode, variant, s) : launch_dm<2, false>(a, mode, variant, s);
    return mixed ? launch_dm<3, true>(a, mode, variant, s) : launch_dm<3, false>(a, mode, variant, s);
}

int epf_lanes_per_node(int dim, int variant) {
    if (epf_is_tma(variant)) return epf_tma_lanes(dim, variant - 5);
    return dim == 3 ? kLpn3[variant] : kLpn2[variant];
}

int epf_tile_nodes(int dim, int variant) {
    if (epf_is_tma(variant)) return 0;
    return dim == 3 ? kTile3[variant] : kTile2[variant];
}

bool epf_variant_fits(int dim, int variant, int max_family) {
    if (epf_is_tma(variant)) {
        const int maxb = epf_tma_maxb(dim, variant, max_family);
        return epf_tma_smem(dim, false, variant - 5, maxb) <= 227u * 1024u;
    }
    const int nb = epf_tile_nodes(dim, variant);
    return nb == 0 || (long long)nb * max_family <= kStreamMap;
}

int epf_grid(int n, int dim, int variant) {
    static int sms = 0;
    if (sms == 0) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (sms <= 0) sms = 148;
    }
    const int lpn = epf_lanes_per_node(dim, variant);
    const int nodes_per_block = lpn ? (kEpfThreads / kWarp) * (kWarp / lpn) : epf_tile_nodes(dim, variant);
    const long long need = ((long long)n + nodes_per_block - 1) / nodes_per_block;
    const long long cap = (long long)sms * 8;
    const long long g = need < cap ? need : cap;
    return (int)(g > 0 ? g : 1);
}

}  // namespace pxb
