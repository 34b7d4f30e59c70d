// g-function build with one warp per node (reference PDOperators::calcAMatrixCompute / calcOperatorsCompute,
// src/PDOperators/CalcPDOperators.cpp:108-226 and 307-354), for moment systems of up to 32 monomials.
//
// The lane-group build (k_gbuild.cu) keeps the whole packed moment matrix in every lane while it accumulates and
// reduces, which at 3D order 2 (45 entries) takes ~250 registers a thread and leaves 2 blocks per SM.  Here:
//   pass 1  the family is walked in chunks of 32 bonds, one bond per lane: the lane forms its bond's weight bw
//           (cached in shared memory for pass 2) and monomials m, and the chunk's contribution to every entry
//           A[p][q] += (bw m_p) m_q is summed over the warp by a recursive-halving reduce-scatter whose products
//           are formed as the pairs are exchanged; after the five halvings each lane holds the chunk sums of at
//           most ceil(NE/32) entries and adds them to its accumulators;
//   solve   the entries go to shared memory, the warp factors A = L D L^T (right-looking, a row per lane), lane k
//           solves column k of X = A^-1 diag(q!) (with one step of iterative refinement above nine monomials) and
//           the reference's max-norm consistency test (src/MathUtils/MatrixXd.cpp:40-47) decides degeneracy;
//   pass 2  one bond per lane again: op_k = (sum_p X[p][k] m_p) bw / delta^|q_k| for every slot k, written as the
//           AoS operator vector and/or the SoA Navier subset; MIXED stores FP32 (sums stay FP64) and, at order 2,
//           the per-node first moments of the stored second-derivative operators (GBuildArgs::defect).
// With TC (up to nine monomials, the default there) the same three phases use the FP64 tensor cores
// (mma.sync.m8n8k4.f64): pass 1 accumulates the (0,0) tile of A = (W M)^T M from each chunk's transposed monomials
// (the ninth row per lane on the CUDA cores), the solve is Gauss-Jordan on [A | diag(q!)] with a row per lane in
// registers and its residual D - A X a tensor-core product, and pass 2 forms operators 0-7 as 8-bond tiles (the
// ninth per lane) staged in shared memory and stored as one coalesced block per chunk.
// Per-node horizons (GBuildArgs::node_delta / node_dxc) follow the reference's variable-horizon path: node i
// uses its own delta_i and spacing, and bonds longer than delta_i stay out of its moment system and get zero
// operators (CalcPDOperators.cpp:113-147, 307-354).
#include <cfloat>
#include <cstddef>

#include "k_kernels.h"
#include "pxb_common.cuh"

namespace pxb {

namespace {

constexpr int kWarpNodeThreads = 128;  // 4 warps (nodes) per block
constexpr int kBwCache = 256;          // bond weights per node cached for pass 2 (longer families recompute)
constexpr int kMonoStride = 36;        // row stride (doubles) of the transposed monomial tile: conflict-minimal reads
constexpr int kOpStride = 9;           // room (doubles) for one bond's staged operator row, up to nine monomials

// packed upper triangle (p <= q, row-major) of an NOP x NOP symmetric matrix
template <int NOP>
struct Tri {
    static constexpr int NE = NOP * (NOP + 1) / 2;
    int p[NE], q[NE];
    __host__ __device__ constexpr Tri() : p{}, q{} {
        int e = 0;
        for (int a = 0; a < NOP; ++a)
            for (int b = a; b < NOP; ++b) {
                p[e] = a;
                q[e] = b;
                ++e;
            }
    }
};

__host__ __device__ constexpr int halve(int n) { return (n + 1) / 2; }

// shared-memory loads the compiler may not hoist out of the bond loops (it would otherwise keep the whole
// loop-invariant X, A or L D L^T in registers)
__device__ __forceinline__ unsigned smem_addr(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }
__device__ __forceinline__ double lds(const double *p) {
    double v;
    asm volatile("ld.shared.f64 %0, [%1];" : "=d"(v) : "r"(smem_addr(p)));
    return v;
}
__device__ __forceinline__ double2 lds2(const double *p) {
    double2 v;
    asm volatile("ld.shared.v2.f64 {%0, %1}, [%2];" : "=d"(v.x), "=d"(v.y) : "r"(smem_addr(p)));
    return v;
}

// one halving of a reduce-scatter: lanes whose bit MASK is clear keep the first half of the list, their partners
// the second; each sends the other half and adds what it receives (a missing odd element counts as 0)
template <int N, int MASK>
__device__ __forceinline__ void rs_level(const double (&in)[N], double (&out)[halve(N)], bool upper) {
    constexpr int H = halve(N);
#pragma unroll
    for (int k = 0; k < H; ++k) {
        const double lo = in[k];
        const double hi = (H + k < N) ? in[(H + k < N) ? H + k : 0] : 0.0;
        const double send = upper ? lo : hi;
        const double keep = upper ? hi : lo;
        out[k] = keep + __shfl_xor_sync(kFull, send, MASK);
    }
}

// entry index held in final slot s by this lane after the five halvings of an NE-long list (-1: padding)
template <int NE>
__device__ __forceinline__ int rs_entry(int lane, int s) {
    constexpr int L0 = NE, L1 = halve(L0), L2 = halve(L1), L3 = halve(L2), L4 = halve(L3);
    int p = s;
    p = (lane & 1) ? halve(L4) + p : p;
    if (p >= L4) return -1;
    p = (lane & 2) ? halve(L3) + p : p;
    if (p >= L3) return -1;
    p = (lane & 4) ? halve(L2) + p : p;
    if (p >= L2) return -1;
    p = (lane & 8) ? halve(L1) + p : p;
    if (p >= L1) return -1;
    p = (lane & 16) ? halve(L0) + p : p;
    if (p >= L0) return -1;
    return p;
}

// D += A B on the FP64 tensor cores (m8n8k4): lane l holds A[l/4][l%4], B[l%4][l/4] and D[l/4][2(l%4) + {0,1}]
__device__ __forceinline__ void dmma(double (&d)[2], double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
                 : "+d"(d[0]), "+d"(d[1])
                 : "d"(a), "d"(b));
}

struct BondGeo {
    double dx, dy, dz, bw;
};

// per-node constants of the weight: delta, 4/delta^2, the rim spacing and the squared inner radius of the rim
// (delta - dx_char/2)^2 (-1 when that radius is not positive: every bond is a rim bond)
struct NodeWeight {
    double delta, four_inv_d2, dxc, rim2;
    __device__ __forceinline__ NodeWeight(double d, double dx) : delta(d), four_inv_d2(4.0 / (d * d)), dxc(dx) {
        const double ri = d - 0.5 * dx;
        rim2 = (dx > 0.0 && ri > 0.0) ? ri * ri : -1.0;
    }
};

// bond t of node i: the bond vector and the weight bw = w(|xi|) vc(|xi|) V_j (0 when the bond is skipped: zero
// length, outside the node's own horizon, or a non-positive weight).  w = exp(-(2|xi|/delta)^2) is evaluated from
// |xi|^2 (a few ulps from the reference's rounding of 2|xi|/delta); |xi| itself is formed only for rim bonds and
// for the own-horizon test
template <int DIM, typename PosT>
__device__ __forceinline__ BondGeo bond_geo_at(const PosT &xj, double vj, const PosT &xi, const NodeWeight &nw,
                                               bool own_horizon) {
    BondGeo g{0.0, 0.0, 0.0, 0.0};
    g.dx = xj.x - xi.x;
    g.dy = xj.y - xi.y;
    if constexpr (DIM == 3) g.dz = xj.z - xi.z;
    const double r2 = g.dx * g.dx + g.dy * g.dy + g.dz * g.dz;
    if (r2 > 0.0 && !(own_horizon && sqrt(r2) > nw.delta)) {
        double bw = exp(-(r2 * nw.four_inv_d2));
        if (nw.dxc > 0.0 && r2 > nw.rim2) bw *= rim_correction(sqrt(r2), nw.delta, nw.dxc);
        bw *= vj;
        if (bw > 0.0) g.bw = bw;
    }
    return g;
}

template <int DIM, typename PosT>
__device__ __forceinline__ BondGeo bond_geo(const GBuildArgs &a, const PosT *pos, const PosT &xi, int t,
                                            const NodeWeight &nw, bool own_horizon) {
    const int j = a.nbr[t];
    return bond_geo_at<DIM>(pos[j - a.node_base], a.vol[j], xi, nw, own_horizon);
}

}  // namespace

// Shared memory a warp needs for one node of NOP monomials (doubles): weight cache, A, L D L^T, X (rows padded
// to an even count so that rows load as double2).
template <int NOP, bool TC = false>
struct WarpNodeSmem {
    static constexpr int NP = (NOP + 1) & ~1;
    // bonds whose weight (and bond vector) pass 1 caches for pass 2: 128 with the tensor-core tiles, so that a
    // 2-warp block fits 8 times on an SM
    static constexpr int BWC = TC ? 128 : kBwCache;
    // bond vectors cached for pass 2 too (up to nine monomials; larger systems gather them again)
    static constexpr bool CACHE_X = NOP <= 9;
    static constexpr int XC = CACHE_X ? BWC : 2;
    // every section starts on a 16-byte boundary (X is read as double2)
    alignas(16) double bw[BWC];
    alignas(16) double xc[3 * XC];
    // TC (up to nine monomials): a chunk's monomials transposed [p][bond] (rows padded to 16, row stride kMonoStride),
    // its bond weights and its operator rows, and column 8 of X (the ninth operator is formed on the CUDA cores);
    // the L D L^T factors of the scalar path are not kept
    static constexpr bool TCA = TC && NOP <= 9;
    alignas(16) double A[NOP * NOP];
    alignas(16) double L[TCA ? 2 : NOP * NOP];
    alignas(16) double X[NOP * NP];
    alignas(16) double invD[TCA ? 2 : NP];  // 1 / D of the L D L^T factorisation
    alignas(16) double monoT[TCA ? 16 * kMonoStride : 2];
    alignas(16) double wk[TCA ? 32 : 2];
    alignas(16) double opb[TCA ? 32 * kOpStride : 2];
    alignas(16) double c8[TCA ? NP : 2];
};
static_assert(offsetof(WarpNodeSmem<14>, X) % 16 == 0 && offsetof(WarpNodeSmem<19>, X) % 16 == 0 &&
                  offsetof(WarpNodeSmem<9>, X) % 16 == 0 && offsetof(WarpNodeSmem<5>, X) % 16 == 0,
              "X rows are read as double2");

// TC (up to nine monomials): the moment sums and the per-bond operator products run on the FP64 tensor cores
// (mma m8n8k4): per 32-bond chunk the lanes store their bonds' monomials transposed in shared memory, the moment
// matrix accumulates as A += (W M)^T M over 4-bond k-steps in the (0,0) 8x8 tile (no cross-lane reduction; a
// ninth monomial's row is summed per lane), and in pass 2 each 8-bond tile of the chunk multiplies its monomials
// by X (held as B fragments in registers)
template <int DIM, int ORDER, bool MIXED, bool TC = false>
__device__ __forceinline__ void gbuild_warp_node(const GBuildArgs &a, int i, int lane,
                                                 WarpNodeSmem<nop_of(DIM, ORDER), TC> &sm) {
    constexpr QTable<DIM, ORDER> Q{};
    constexpr int NOP = Q.NOP;
    constexpr Tri<NOP> T{};
    constexpr int NE = Tri<NOP>::NE;
    constexpr int L1 = halve(NE), L2 = halve(L1), L3 = halve(L2), L4 = halve(L3), L5 = halve(L4);
    constexpr int NP = WarpNodeSmem<NOP, TC>::NP;
    static_assert(NOP <= 32, "one lane per solve column");
    using PosT = typename Vec<DIM>::T;
    const PosT *pos = static_cast<const PosT *>(a.pos);
    const bool own_h = a.node_delta != nullptr;
    const double delta = own_h ? a.node_delta[i - a.node_base] : a.delta;
    const double dxc = own_h ? a.node_dxc[i - a.node_base] : a.dx_char;
    const double inv_delta = 1.0 / delta;
    constexpr bool XCACHE = WarpNodeSmem<NOP, TC>::CACHE_X;
    constexpr int BWC = WarpNodeSmem<NOP, TC>::BWC;
    const int b0 = a.off[i], b1 = a.off[i + 1];
    const PosT xi = pos[i - a.node_base];

    // ---- pass 1: moment sums, chunk by chunk ----
    double acc[L5];
#pragma unroll
    for (int s = 0; s < L5; ++s) acc[s] = 0.0;
    static_assert(!TC || NOP <= 9, "tensor-core path: up to nine monomials");
    constexpr int MS = kMonoStride;
    const int grp = lane >> 2, tig = lane & 3;  // mma fragment coordinates
    // TC: the moment tile (0,0) on the tensor cores, four accumulators (k-steps modulo 4: shorter dependency
    // chains); with nine monomials the ninth row A[p][8] = sum bw m_p m_8 is summed per lane on the CUDA cores and
    // reduce-scattered once per node (an (0,8) and an (8,8) tile would use one column of eight)
    double c00[4][2] = {{0.0, 0.0}, {0.0, 0.0}, {0.0, 0.0}, {0.0, 0.0}};
    constexpr int N8 = NOP > 8 ? NOP : 1;
    double a8[N8];
#pragma unroll
    for (int p = 0; p < N8; ++p) a8[p] = 0.0;
    if constexpr (TC) {  // padding rows of the monomial tile stay zero for the node
#pragma unroll
        for (int p = NOP; p < 16; ++p) sm.monoT[p * MS + lane] = 0.0;
    }
    int usable = 0;
    {
    const NodeWeight nw(delta, dxc);
    // TC: the gathers run ahead of the chunk being summed (neighbour ids two chunks, their positions and volumes
    // one chunk), so that their latency overlaps the moment products of the chunk before
    int jn = -1;
    PosT xq{};
    double vq = 0.0;
    if constexpr (TC) {
        const int j0 = b0 + lane < b1 ? a.nbr[b0 + lane] : -1;
        if (j0 >= 0) {
            xq = pos[j0 - a.node_base];
            vq = a.vol[j0];
        }
        jn = b0 + kWarp + lane < b1 ? a.nbr[b0 + kWarp + lane] : -1;
    }
    for (int c0 = b0; c0 < b1; c0 += kWarp) {
        const int t = c0 + lane;
        BondGeo g{0.0, 0.0, 0.0, 0.0};
        if constexpr (TC) {
            const PosT xj = xq;
            const double vj = vq;
            if (jn >= 0) {
                xq = pos[jn - a.node_base];
                vq = a.vol[jn];
            }
            jn = t + 2 * kWarp < b1 ? a.nbr[t + 2 * kWarp] : -1;
            if (t < b1) g = bond_geo_at<DIM>(xj, vj, xi, nw, own_h);
        } else {
            if (t < b1) g = bond_geo<DIM>(a, pos, xi, t, nw, own_h);
        }
        if (t < b1 && t - b0 < BWC) {
            sm.bw[t - b0] = g.bw;
            if constexpr (XCACHE) {
                sm.xc[3 * (t - b0)] = g.dx;
                sm.xc[3 * (t - b0) + 1] = g.dy;
                sm.xc[3 * (t - b0) + 2] = g.dz;
            }
        }
        usable += g.bw > 0.0 ? 1 : 0;
        double m[NOP], wm[NOP];
        monomials<DIM, ORDER, double>(g.dx * inv_delta, g.dy * inv_delta, g.dz * inv_delta, m);
        if constexpr (TC) {
#pragma unroll
            for (int p = 0; p < (NOP < 8 ? NOP : 8); ++p) sm.monoT[p * MS + lane] = m[p];
            sm.wk[lane] = g.bw;
            if constexpr (NOP > 8) {
                const double wm8 = g.bw * m[8];
#pragma unroll
                for (int p = 0; p < NOP; ++p) a8[p] = fma(wm8, m[p], a8[p]);
            }
            __syncwarp();
#pragma unroll
            for (int kk = 0; kk < 8; ++kk) {  // k-steps of 4 bonds: A frag bw_b m_p(b), B frag m_q(b)
                const int b = 4 * kk + tig;
                const double w = sm.wk[b];
                const double mlo = sm.monoT[grp * MS + b];
                dmma(c00[kk & 3], w * mlo, mlo);
            }
            __syncwarp();
        } else {
#pragma unroll
        for (int k = 0; k < NOP; ++k) wm[k] = g.bw * m[k];
        // first halving with the products formed as they are exchanged
        double v1[L1];
        {
            const bool upper = (lane & 16) != 0;
#pragma unroll
            for (int k = 0; k < L1; ++k) {
                constexpr int dummy = 0;
                const int kh = (L1 + k < NE) ? L1 + k : dummy;
                const double lo = wm[T.p[k]] * m[T.q[k]];
                const double hi = (L1 + k < NE) ? wm[T.p[kh]] * m[T.q[kh]] : 0.0;
                const double send = upper ? lo : hi;
                const double keep = upper ? hi : lo;
                v1[k] = keep + __shfl_xor_sync(kFull, send, 16);
            }
        }
        double v2[L2], v3[L3], v4[L4], v5[L5];
        rs_level<L1, 8>(v1, v2, (lane & 8) != 0);
        rs_level<L2, 4>(v2, v3, (lane & 4) != 0);
        rs_level<L3, 2>(v3, v4, (lane & 2) != 0);
        rs_level<L4, 1>(v4, v5, (lane & 1) != 0);
#pragma unroll
        for (int s = 0; s < L5; ++s) acc[s] += v5[s];
        }
    }
    }
    usable = group_sum_int<kWarp>(usable);
    if constexpr (TC) {  // the tiles' upper triangle, mirrored (the matrix stays exactly symmetric)
        auto put = [&](int p, int q, double v) {
            if (p <= q && q < NOP) {
                sm.A[p * NOP + q] = v;
                sm.A[q * NOP + p] = v;
            }
        };
#pragma unroll
        for (int h = 0; h < 2; ++h) put(grp, 2 * tig + h, (c00[0][h] + c00[2][h]) + (c00[1][h] + c00[3][h]));
        if constexpr (NOP > 8) {  // the ninth row: five halvings leave entry rs_entry(lane) of a8 in lane
            static_assert(NOP == 9, "tensor-core path: up to nine monomials");
            double v1[5], v2[3], v3[2], v4[1], v5[1];
            rs_level<9, 16>(a8, v1, (lane & 16) != 0);
            rs_level<5, 8>(v1, v2, (lane & 8) != 0);
            rs_level<3, 4>(v2, v3, (lane & 4) != 0);
            rs_level<2, 2>(v3, v4, (lane & 2) != 0);
            rs_level<1, 1>(v4, v5, (lane & 1) != 0);
            const int e = rs_entry<9>(lane, 0);
            if (e >= 0) put(e, 8, v5[0]);
        }
    } else {
#pragma unroll
        for (int s = 0; s < L5; ++s) {
            const int e = rs_entry<NE>(lane, s);
            if (e >= 0) {
                sm.A[T.p[e] * NOP + T.q[e]] = acc[s];
                sm.A[T.q[e] * NOP + T.p[e]] = acc[s];
                sm.L[T.p[e] * NOP + T.q[e]] = acc[s];
                sm.L[T.q[e] * NOP + T.p[e]] = acc[s];
            }
        }
    }
    __syncwarp();

    double res = 0.0, maxA = 0.0, maxX = 0.0;
    bool degenerate;
    if constexpr (TC) {
        // ---- solve (up to nine monomials): Gauss-Jordan on [A | diag(q!)] with row r in lane r's registers; the
        // pivot row is broadcast by shuffles, so no shared-memory round trip or warp barrier per column.  A is
        // symmetric positive definite for a usable family (no pivoting, as in the L D L^T path); before step j the
        // right-hand side of row j is zero past column j.  Lane p < NOP ends with row p of X = A^-1 diag(q!).
        double ra[NOP], rb[NOP];
#pragma unroll
        for (int k = 0; k < NOP; ++k) {
            ra[k] = lane < NOP ? lds(&sm.A[(lane < NOP ? lane : 0) * NOP + k]) : 0.0;
            rb[k] = (k == lane) ? Q.fact[k] : 0.0;
        }
#pragma unroll
        for (int j = 0; j < NOP; ++j) {
            double pa[NOP], pb[NOP];
#pragma unroll
            for (int k = j; k < NOP; ++k) pa[k] = __shfl_sync(kFull, ra[k], j);
#pragma unroll
            for (int k = 0; k <= j; ++k) pb[k] = __shfl_sync(kFull, rb[k], j);
            const double inv = 1.0 / pa[j];
            const bool piv = lane == j;
            const double f = ra[j] * inv;
#pragma unroll
            for (int k = j + 1; k < NOP; ++k) ra[k] = piv ? pa[k] * inv : fma(-f, pa[k], ra[k]);
#pragma unroll
            for (int k = 0; k <= j; ++k) rb[k] = piv ? pb[k] * inv : fma(-f, pb[k], rb[k]);
        }
        // the consistency test's residual D - A X on the tensor cores (X rows through shared memory, 8x8 tiles)
        if (lane < NOP) {
#pragma unroll
            for (int k = 0; k < NP; ++k) sm.X[lane * NP + k] = k < NOP ? rb[k < NOP ? k : 0] : 0.0;
#pragma unroll
            for (int k = 0; k < NOP; ++k) maxX = max_nan(maxX, fabs(rb[k]));
        }
        __syncwarp();
        constexpr int RT = NOP > 8 ? 2 : 1, KS = (NOP + 3) / 4;
        double rt[RT][RT][2];
#pragma unroll
        for (int u = 0; u < RT; ++u)
#pragma unroll
            for (int v = 0; v < RT; ++v) rt[u][v][0] = rt[u][v][1] = 0.0;
#pragma unroll
        for (int ks = 0; ks < KS; ++ks) {
            const int kk = 4 * ks + tig;
            double af[RT], bf[RT];
#pragma unroll
            for (int u = 0; u < RT; ++u) {
                const int row = 8 * u + grp;
                af[u] = (row < NOP && kk < NOP) ? sm.A[row * NOP + kk] : 0.0;
                bf[u] = (kk < NOP && row < NOP) ? sm.X[kk * NP + row] : 0.0;  // B[kk][col = 8u + grp]
                maxA = fmax(maxA, fabs(af[u]));
            }
#pragma unroll
            for (int u = 0; u < RT; ++u)
#pragma unroll
                for (int v = 0; v < RT; ++v) dmma(rt[u][v], af[u], bf[v]);
        }
#pragma unroll
        for (int u = 0; u < RT; ++u)
#pragma unroll
            for (int v = 0; v < RT; ++v)
#pragma unroll
                for (int h = 0; h < 2; ++h) {
                    const int row = 8 * u + grp, col = 8 * v + 2 * tig + h;
                    if (row < NOP && col < NOP) {
                        double dv = 0.0;
#pragma unroll
                        for (int q = 0; q < NOP; ++q)
                            if (q == row && q == col) dv = Q.fact[q];
                        res = max_nan(res, fabs(dv - rt[u][v][h]));
                    }
                }
        maxA = group_max<kWarp>(maxA);
        res = group_max_nan<kWarp>(res);
        maxX = group_max_nan<kWarp>(maxX);
        double maxB = 0.0;
#pragma unroll
        for (int q = 0; q < NOP; ++q) maxB = fmax(maxB, Q.fact[q]);
        const double scale = fmax(fmax(maxB, maxA * maxX), DBL_MIN);
        const bool consistent = (res <= 1.0e-8 * scale);  // NaN-safe: NaN fails
        degenerate = (usable < NOP) || !consistent;
        __syncwarp();  // X is written again below, scaled
        // column k carries the operator's scale 1/delta^|q_k|, so that pass 2 only multiplies by the bond weight
        if (lane < NOP) {
#pragma unroll
            for (int k = 0; k < NOP; ++k) {
                double cs = inv_delta;
#pragma unroll
                for (int t2 = 1; t2 < Q.p[k] + Q.q[k] + Q.r[k]; ++t2) cs *= inv_delta;
                sm.X[lane * NP + k] = degenerate ? 0.0 : rb[k] * cs;
                if (k == 8) sm.c8[lane < NOP ? lane : 0] = degenerate ? 0.0 : rb[k] * cs;
            }
        }
    } else {
        // ---- solve: A = L D L^T right-looking in sm.L (row r in lane r; D on the diagonal, L below) ----
        for (int j = 0; j < NOP; ++j) {
            const double d = sm.L[j * NOP + j];
            const double cr = (lane > j && lane < NOP) ? sm.L[lane * NOP + j] : 0.0;  // column j before scaling
            __syncwarp();
            if (lane > j && lane < NOP) {
                const double l = cr / d;
                for (int k = j + 1; k <= lane; ++k) sm.L[lane * NOP + k] -= l * sm.L[k * NOP + j];
            }
            __syncwarp();
            if (lane > j && lane < NOP) sm.L[lane * NOP + j] = cr / d;
            __syncwarp();
        }
        if constexpr (NOP <= 9) {
            if (lane < NOP) sm.invD[lane] = 1.0 / sm.L[lane * NOP + lane];
            __syncwarp();
        }
        // lane k < NOP: column k of X = A^-1 diag(q!), one refinement step, the consistency test's residual
        const int kc = lane < NOP ? lane : 0;
        double fk = 0.0;
#pragma unroll
        for (int q = 0; q < NOP; ++q)
            if (q == kc) fk = Q.fact[q];
        auto solve = [&](double *x) {
#pragma unroll
            for (int r = 0; r < NOP; ++r) {
#pragma unroll
                for (int l = 0; l < r; ++l) x[r] -= lds(&sm.L[r * NOP + l]) * x[l];
            }
#pragma unroll
            for (int r = 0; r < NOP; ++r) {
                // up to nine monomials by the reciprocals (formed once per node); the larger systems divide (fewer
                // live registers there)
                if constexpr (NOP <= 9) x[r] *= lds(&sm.invD[r]);
                else x[r] /= lds(&sm.L[r * NOP + r]);
            }
#pragma unroll
            for (int r = NOP - 1; r >= 0; --r) {
#pragma unroll
                for (int l = r + 1; l < NOP; ++l) x[r] -= lds(&sm.L[l * NOP + r]) * x[l];
            }
        };
        double x[NOP];
#pragma unroll
        for (int q = 0; q < NOP; ++q) x[q] = (q == kc) ? fk : 0.0;
        solve(x);
        double r[NOP];
#pragma unroll
        for (int p = 0; p < NOP; ++p) {
            double sres = (p == kc) ? fk : 0.0;
#pragma unroll
            for (int q = 0; q < NOP; ++q) {
                const double apq = lds(&sm.A[p * NOP + q]);
                sres -= apq * x[q];
                maxA = fmax(maxA, fabs(apq));
            }
            r[p] = sres;
            res = fmax(res, fabs(sres));
            maxX = fmax(maxX, fabs(x[p]));
        }
        // one step of iterative refinement for the larger systems (14, 19 monomials); up to nine monomials the plain
        // solve is already ~1e-14 (family-scaled) from the reference's FullPivLU result, and a refinement step changes
        // nothing measurable there
        if constexpr (NOP > 9) {
            solve(r);
#pragma unroll
            for (int q = 0; q < NOP; ++q) x[q] += r[q];
        }
        if (lane >= NOP) {
            maxX = 0.0;
            res = 0.0;
        }
        res = group_max<kWarp>(res);
        maxX = group_max<kWarp>(maxX);
        double maxB = 0.0;
#pragma unroll
        for (int q = 0; q < NOP; ++q) maxB = fmax(maxB, Q.fact[q]);
        const double scale = fmax(fmax(maxB, maxA * maxX), DBL_MIN);
        const bool consistent = (res <= 1.0e-8 * scale);  // NaN-safe: NaN fails
        degenerate = (usable < NOP) || !consistent;
        // column k carries the operator's scale 1/delta^|q_k|, so that pass 2 only multiplies by the bond weight
        int ord = 1;  // |q_k| of this lane's column: the monomials are ordered by total degree
        while (ord < ORDER && kc >= nop_of(DIM, ord)) ++ord;
        double colscale = inv_delta;
        for (int t2 = 1; t2 < ord; ++t2) colscale *= inv_delta;
        if (lane < NP) {
#pragma unroll
            for (int p = 0; p < NOP; ++p) sm.X[p * NP + lane] = (degenerate || lane >= NOP) ? 0.0 : x[p] * colscale;
        }
    }
    const bool deep_ghost = (a.layer != nullptr) && (a.layer[i] > 1);
    if (lane == 0) {
        if (a.degenerate) a.degenerate[i] = degenerate ? 1 : 0;
        if (degenerate && !deep_ghost) {
            atomicAdd(a.n_degenerate, 1u);
            atomicMin(a.first_degenerate, i);
        }
    }
    __syncwarp();

    // ---- pass 2: per-bond operators ----
    constexpr bool DEF = MIXED && ORDER == 2;
    constexpr int ND = DEF ? (NOP - DIM) * DIM : 1;
    // scalar path: per-lane defect sums; TC: a tensor-core tile D[k - DIM][d] (two accumulators)
    double dsum[TC ? 1 : ND];
#pragma unroll
    for (int e = 0; e < (TC ? 1 : ND); ++e) dsum[e] = 0.0;
    double dfc[2][2] = {{0.0, 0.0}, {0.0, 0.0}};
    // the bond's geometry in pass 2: cached in pass 1, or formed again past the cache
    auto geo2 = [&](int t) -> BondGeo {
        BondGeo g;
        if (t - b0 < BWC) {
            if constexpr (XCACHE) {
                g.dx = sm.xc[3 * (t - b0)];
                g.dy = sm.xc[3 * (t - b0) + 1];
                g.dz = sm.xc[3 * (t - b0) + 2];
            } else {
                const int j = a.nbr[t];
                const PosT xj = pos[j - a.node_base];
                g.dx = xj.x - xi.x;
                g.dy = xj.y - xi.y;
                g.dz = 0.0;
                if constexpr (DIM == 3) g.dz = xj.z - xi.z;
            }
            g.bw = sm.bw[t - b0];
        } else {  // past the weight cache (families longer than BWC): formed again
            g = bond_geo<DIM>(a, pos, xi, t, NodeWeight(delta, dxc), own_h);
        }
        return g;
    };
    // the defect's first moments of one bond's stored (FP32) second-derivative operators and its Navier subset
    auto emit_rest = [&](int t, const BondGeo &g, const double *op) {
        if constexpr (DEF && !TC) {
            if (a.ops) {
#pragma unroll
                for (int k = DIM; k < NOP; ++k) {
                    const float gk = (float)op[k];
                    dsum[(k - DIM) * DIM + 0] += (double)gk * g.dx;
                    dsum[(k - DIM) * DIM + 1] += (double)gk * g.dy;
                    if constexpr (DIM == 3) dsum[(k - DIM) * DIM + 2] += (double)gk * g.dz;
                }
            }
        }
        if constexpr (ORDER >= 2) {
            if (a.G) {
                constexpr int NC = (DIM == 3) ? 6 : 3;
                int sl[NC];
                if constexpr (DIM == 3) {
                    sl[0] = Q.slot(2, 0, 0); sl[1] = Q.slot(0, 2, 0); sl[2] = Q.slot(0, 0, 2);
                    sl[3] = Q.slot(1, 1, 0); sl[4] = Q.slot(1, 0, 1); sl[5] = Q.slot(0, 1, 1);
                } else {
                    sl[0] = Q.slot(2, 0, 0); sl[1] = Q.slot(0, 2, 0); sl[2] = Q.slot(1, 1, 0);
                }
#pragma unroll
                for (int c = 0; c < NC; ++c) {
                    const double v = op[sl[c]];
                    if constexpr (MIXED) static_cast<float *>(a.G)[(size_t)c * a.nb + t] = (float)v;
                    else static_cast<double *>(a.G)[(size_t)c * a.nb + t] = v;
                }
            }
        }
    };
    // one bond's operator vector out: AoS operators (MIXED: FP32), then the defect moments and the Navier subset
    auto emit = [&](int t, const BondGeo &g, const double *op) {
        if (a.ops) {
            if constexpr (MIXED) {
                float *o = static_cast<float *>(a.ops) + (size_t)(t - a.bond_base) * NOP;
#pragma unroll
                for (int k = 0; k < NOP; ++k) o[k] = (float)op[k];
            } else {
                double *o = static_cast<double *>(a.ops) + (size_t)(t - a.bond_base) * NOP;
#pragma unroll
                for (int k = 0; k < NOP; ++k) o[k] = op[k];
            }
        }
        emit_rest(t, g, op);
    };
    // TC: X as B fragments (rows = monomials in k-steps of 4, columns = operators in tiles of 8), zero past NOP
    // (operators 0..7 on the tensor cores; the ninth, when there is one, per lane on the CUDA cores)
    constexpr int KS = (NOP + 3) / 4, NT2 = 1;
    constexpr int BTG = 4;  // 8-bond tiles whose DMMA chains run interleaved
    // the chunk's operator rows: FP64, or MIXED the stored FP32 values (rounded once, where they are staged)
    float *const opf = reinterpret_cast<float *>(sm.opb);
    auto stage = [&](int idx, double v) {
        if constexpr (MIXED) opf[idx] = (float)v;
        else sm.opb[idx] = v;
    };
    auto staged = [&](int idx) -> double {
        if constexpr (MIXED) return (double)opf[idx];
        else return sm.opb[idx];
    };
    constexpr int OS = NOP | 1;           // row stride (doubles) of the staged operator rows: odd, conflict-free
    double bx[TC ? KS : 1][TC ? NT2 : 1];
    if constexpr (TC) {
#pragma unroll
        for (int ks = 0; ks < KS; ++ks)
#pragma unroll
            for (int nt = 0; nt < NT2; ++nt) {
                const int pr = 4 * ks + tig, kc2 = 8 * nt + grp;
                bx[ks][nt] = (pr < NOP && kc2 < NOP) ? sm.X[pr * NP + kc2] : 0.0;
            }
    }
    for (int c0 = b0; c0 < b1; c0 += kWarp) {
        const int t = c0 + lane;
        if constexpr (TC) {
            BondGeo g{0.0, 0.0, 0.0, 0.0};
            if (t < b1) g = geo2(t);
            double m[NOP];
            monomials<DIM, ORDER, double>(g.dx * inv_delta, g.dy * inv_delta, g.dz * inv_delta, m);
#pragma unroll
            for (int p = 0; p < NOP; ++p) sm.monoT[p * MS + lane] = m[p];
            sm.wk[lane] = g.bw;
            if constexpr (NOP > 8) {  // op_8 = bw sum_p m_p X[p][8]
                double s8 = 0.0;
#pragma unroll
                for (int p = 0; p < NOP; p += 2) {
                    const double2 cp = lds2(&sm.c8[p]);  // c8 is padded to an even count
                    s8 = fma(m[p], cp.x, s8);
                    if (p + 1 < NOP) s8 = fma(m[p + 1 < NOP ? p + 1 : 0], cp.y, s8);
                }
                stage(lane * OS + 8, g.bw * s8);
            }
            __syncwarp();
            // 8-bond tiles D[bond][k] = sum_p m_p(bond) X[p][k], BTG tiles at a time so that their DMMA chains
            // interleave
#pragma unroll
            for (int bg = 0; bg < 4; bg += BTG) {
                double dd[BTG][NT2][2];
#pragma unroll
                for (int u = 0; u < BTG; ++u)
#pragma unroll
                    for (int nt = 0; nt < NT2; ++nt) dd[u][nt][0] = dd[u][nt][1] = 0.0;
#pragma unroll
                for (int ks = 0; ks < KS; ++ks) {
                    double am[BTG];
#pragma unroll
                    for (int u = 0; u < BTG; ++u) am[u] = sm.monoT[(4 * ks + tig) * MS + 8 * (bg + u) + grp];
#pragma unroll
                    for (int u = 0; u < BTG; ++u)
#pragma unroll
                        for (int nt = 0; nt < NT2; ++nt) dmma(dd[u][nt], am[u], bx[ks][nt]);
                }
#pragma unroll
                for (int u = 0; u < BTG; ++u) {
                    const double w = sm.wk[8 * (bg + u) + grp];
                    const int row = (8 * (bg + u) + grp) * OS;
#pragma unroll
                    for (int nt = 0; nt < NT2; ++nt)
#pragma unroll
                        for (int h = 0; h < 2; ++h) {
                            const int k = 8 * nt + 2 * tig + h;
                            if (k < NOP) stage(row + k, w * dd[u][nt][h]);
                        }
                }
            }
            __syncwarp();
            // the chunk's operator vectors are one contiguous AoS block: coalesced stores from the staged rows
            const int nval = b1 - c0 < kWarp ? b1 - c0 : kWarp;
            if (a.ops) {
                const size_t o0 = (size_t)(c0 - a.bond_base) * NOP + lane;
                float *const of = static_cast<float *>(a.ops) + o0;
                double *const od = static_cast<double *>(a.ops) + o0;
#pragma unroll
                for (int e0 = 0; e0 < NOP; ++e0) {
                    const int e = e0 * kWarp + lane;
                    if (e < nval * NOP) {
                        const int si = OS == NOP ? e : (e / NOP) * OS + e % NOP;
                        if constexpr (MIXED) of[e0 * kWarp] = opf[si];
                        else od[e0 * kWarp] = sm.opb[si];
                    }
                }
            }
            if constexpr (DEF) {
                // the defect's first moments sum_b g_k(b) xi_d(b) as (G^T M) over the chunk's 4-bond k-steps:
                // A[k - DIM][b] the stored (FP32) second-derivative operators, B[b][d] the first-order monomials
                // xi_d / delta of the tile (the factor delta is applied once at the end)
                if (a.ops && a.defect) {
#pragma unroll
                    for (int kk = 0; kk < 8; ++kk) {
                        const int b = 4 * kk + tig;
                        const double ga = grp < NOP - DIM
                                              ? (double)opf[b * OS + (grp < NOP - DIM ? DIM + grp : 0)]
                                              : 0.0;
                        const double xb = grp < DIM ? sm.monoT[(grp < DIM ? grp : 0) * MS + b] : 0.0;
                        dmma(dfc[kk & 1], ga, xb);
                    }
                }
            }
            if (t < b1 && a.G) {
                double op[NOP];
#pragma unroll
                for (int k = 0; k < NOP; ++k) op[k] = staged(lane * OS + k);
                emit_rest(t, g, op);
            }
            __syncwarp();
        } else {
            if (t >= b1) continue;
            const BondGeo g = geo2(t);
            double m[NOP];
            monomials<DIM, ORDER, double>(g.dx * inv_delta, g.dy * inv_delta, g.dz * inv_delta, m);
            double op[NOP];
#pragma unroll
            for (int k = 0; k < NOP; k += 2) {
                double s0 = 0.0, s1 = 0.0;
#pragma unroll
                for (int p = 0; p < NOP; ++p) {
                    const double2 xr = lds2(&sm.X[p * NP + k]);
                    s0 += xr.x * m[p];
                    s1 += xr.y * m[p];
                }
                // op_k = (sum_p X[p][k] m_p) bw / delta^|q_k| (the scale is in the column of X)
                op[k] = g.bw > 0.0 ? s0 * g.bw : 0.0;
                if (k + 1 < NOP) op[k + 1 < NOP ? k + 1 : 0] = g.bw > 0.0 ? s1 * g.bw : 0.0;
            }
            emit(t, g, op);
        }
    }
    if constexpr (DEF) {
        if (a.defect) {
            float *dst = a.defect + (size_t)(i - a.node_base) * ND;
            if constexpr (TC) {
                if (a.ops) {  // lane (grp, tig) holds D[grp][2 tig + h]
#pragma unroll
                    for (int h = 0; h < 2; ++h) {
                        const int d = 2 * tig + h;
                        if (grp < NOP - DIM && d < DIM) dst[grp * DIM + d] = (float)((dfc[0][h] + dfc[1][h]) * delta);
                    }
                } else {
                    if (lane < ND) dst[lane] = 0.0f;
                }
            } else {
#pragma unroll
                for (int e = 0; e < ND; ++e) {
                    const double v = group_sum<kWarp>(dsum[e]);
                    if (lane == (e & 31)) dst[e] = (float)v;
                }
            }
        }
    }
    __syncwarp();
}

// single geometry: one warp per node, grid-stride over the nodes; MINB resident blocks bound the registers
// (128 a thread at 4, where the 3D order-2 node spills a few dozen bytes)
// threads a block: 4 warps, 2 with the tensor-core tiles (whose per-warp shared memory is larger)
__host__ __device__ constexpr int warp_node_threads(bool tc) { return tc ? 64 : kWarpNodeThreads; }

template <int DIM, int ORDER, bool MIXED, int MINB, bool TC>
__global__ void __launch_bounds__(warp_node_threads(TC), MINB) gbuild_warp_kernel(GBuildArgs a) {
    constexpr int NOP = nop_of(DIM, ORDER);
    constexpr int WPB = warp_node_threads(TC) / kWarp;
    __shared__ WarpNodeSmem<NOP, TC> sm[WPB];
    const int lane = threadIdx.x & 31;
    const int w = threadIdx.x >> 5;
    for (long long i = (long long)blockIdx.x * WPB + w; i < a.n; i += (long long)gridDim.x * WPB)
        gbuild_warp_node<DIM, ORDER, MIXED, TC>(a, (int)i, lane, sm[w]);
}

// tensor-core products (TC) up to nine monomials; larger systems keep the scalar path
template <int DIM, int ORDER, bool TC0>
static cudaError_t launch_warp_order(const GBuildArgs &a, bool mixed, cudaStream_t s) {
    constexpr int NOP = nop_of(DIM, ORDER);
    constexpr bool TC = TC0 && NOP <= 9;
    constexpr int MINB = TC ? 8 : (NOP <= 5 ? 5 : (NOP <= 9 ? 4 : 2));  // TC: 8 blocks of 2 warps
    constexpr int THREADS = warp_node_threads(TC);
    auto k = mixed ? gbuild_warp_kernel<DIM, ORDER, true, MINB, TC> : gbuild_warp_kernel<DIM, ORDER, false, MINB, TC>;
    int dev = 0, sms = 148, per_sm = 1;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, THREADS, 0);
    constexpr int WPB = THREADS / kWarp;
    const long long need = ((long long)a.n + WPB - 1) / WPB;
    const long long cap = (long long)sms * (per_sm > 0 ? per_sm : 1);
    const int grid = (int)(need < cap ? (need > 0 ? need : 1) : cap);
    k<<<grid, THREADS, 0, s>>>(a);
    return cudaGetLastError();
}

template <bool TC>
static cudaError_t launch_warp_tc(const GBuildArgs &a, int dim, int order, bool mixed, cudaStream_t s) {
    if (dim == 2) {
        switch (order) {
            case 1: return launch_warp_order<2, 1, TC>(a, mixed, s);
            case 2: return launch_warp_order<2, 2, TC>(a, mixed, s);
            case 3: return launch_warp_order<2, 3, TC>(a, mixed, s);
            case 4: return launch_warp_order<2, 4, false>(a, mixed, s);
            default: return cudaErrorInvalidValue;
        }
    }
    switch (order) {
        case 1: return launch_warp_order<3, 1, TC>(a, mixed, s);
        case 2: return launch_warp_order<3, 2, TC>(a, mixed, s);
        case 3: return launch_warp_order<3, 3, false>(a, mixed, s);
        default: return cudaErrorInvalidValue;
    }
}

cudaError_t launch_gbuild_warp(const GBuildArgs &a, int dim, int order, bool mixed, bool tc, cudaStream_t s) {
    return tc ? launch_warp_tc<true>(a, dim, order, mixed, s) : launch_warp_tc<false>(a, dim, order, mixed, s);
}

// ---- batched clouds: persistent warps over the task table, one node at a time per warp (order 2) ----------------
template <int A, int B, bool TC>
union BatchWarpSmem {
    WarpNodeSmem<A, TC> s2;
    WarpNodeSmem<B, TC> s3;
};

template <bool MIXED, int DIMS, int MINB, bool TC>
__global__ void __launch_bounds__(warp_node_threads(TC), MINB) gbuild_batch_warp_kernel(BatchArgs b) {
    constexpr int WPB = warp_node_threads(TC) / kWarp;
    __shared__ BatchWarpSmem<5, 9, TC> sm[WPB];
    const int lane = threadIdx.x & 31;
    const int w = threadIdx.x >> 5;
    for (;;) {
        int task = 0;
        if (lane == 0) task = (int)atomicAdd(b.counter, 1u);
        task = __shfl_sync(kFull, task, 0);
        if (task >= b.ntasks) break;
        const BatchTask tk = b.tasks[b.task0 + task];
        const BatchCloud cd = b.clouds[tk.cloud];
        GBuildArgs a;
        a.n = cd.node0 + cd.n;
        a.off = b.off;
        a.nbr = b.nbr;
        a.pos = b.pos + cd.pos_off;
        a.vol = b.vol;
        a.delta = cd.delta;
        a.dx_char = cd.dx_char;
        a.ops = MIXED ? (void *)(static_cast<float *>(b.ops) + cd.ops_off)
                      : (void *)(static_cast<double *>(b.ops) + cd.ops_off);
        a.degenerate = b.degenerate;
        a.n_degenerate = b.n_degenerate;
        a.first_degenerate = b.first_degenerate;
        a.node_base = cd.node0;
        a.bond_base = cd.bond0;
        a.defect = (MIXED && b.defect) ? b.defect + cd.def_off : nullptr;
        for (int k = 0; k < tk.count; ++k) {
            if constexpr ((DIMS & 1) != 0) {
                if (tk.dim == 2) gbuild_warp_node<2, 2, MIXED, TC>(a, tk.first + k, lane, sm[w].s2);
            }
            if constexpr ((DIMS & 2) != 0) {
                if (tk.dim == 3) gbuild_warp_node<3, 2, MIXED, TC>(a, tk.first + k, lane, sm[w].s3);
            }
        }
        __syncwarp();
    }
}

template <bool MIXED, int DIMS, int MINB, bool TC>
static cudaError_t launch_gbw(const BatchArgs &a, cudaStream_t s) {
    auto k = gbuild_batch_warp_kernel<MIXED, DIMS, MINB, TC>;
    int dev = 0, sms = 148, per_sm = 1;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, warp_node_threads(TC), 0);
    const long long want = ((long long)a.ntasks + (warp_node_threads(TC) / kWarp) - 1) / (warp_node_threads(TC) / kWarp);
    const long long cap = (long long)sms * (per_sm > 0 ? per_sm : 1);
    const int grid = (int)(want < cap ? (want > 0 ? want : 1) : cap);
    k<<<grid, warp_node_threads(TC), 0, s>>>(a);
    return cudaGetLastError();
}

// split: one launch per dimension (dims 1: 2D tasks, 2: 3D tasks) with its own register bound
template <bool TC>
static cudaError_t launch_gbw_tc(const BatchArgs &a, bool mixed, bool split, int dims, cudaStream_t s) {
    constexpr int MB3 = TC ? 8 : 4;  // 3D (and joint): TC blocks are 2 warps
    if (!split) return mixed ? launch_gbw<true, 3, MB3, TC>(a, s) : launch_gbw<false, 3, MB3, TC>(a, s);
    constexpr int MB2 = TC ? 8 : 5;
    if (dims == 1) return mixed ? launch_gbw<true, 1, MB2, TC>(a, s) : launch_gbw<false, 1, MB2, TC>(a, s);
    return mixed ? launch_gbw<true, 2, MB3, TC>(a, s) : launch_gbw<false, 2, MB3, TC>(a, s);
}

// split: one launch per dimension (dims 1: 2D tasks, 2: 3D tasks) with its own register bound
cudaError_t launch_gbuild_batch_warp(const BatchArgs &a, bool mixed, bool split, int dims, bool tc, cudaStream_t s) {
    return tc ? launch_gbw_tc<true>(a, mixed, split, dims, s) : launch_gbw_tc<false>(a, mixed, split, dims, s);
}

bool gbuild_warp_supported(int dim, int order) {
    return (dim == 2 && order >= 1 && order <= 4) || (dim == 3 && order >= 1 && order <= 3);
}

}  // namespace pxb
