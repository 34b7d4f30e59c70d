// g-function build: per node i, the PDDO moment matrix over the horizon family, a small dense solve, and the
// per-bond operator values (reference PDOperators::calcAMatrixCompute / calcOperatorsCompute,
// src/PDOperators/CalcPDOperators.cpp:108-226 and 307-354).
//
// Schedule: a group of LPN lanes per node, 32/LPN nodes per warp (families are contiguous in the CSR, so the
// lanes of a group read consecutive bonds).
//   pass 1  lanes accumulate the upper triangle of A = sum_j bw * m m^T over a lane-strided slice of the
//           family; a butterfly reduction within the group leaves the full A in every lane of the group.
//   solve   every lane factors A = L D L^T redundantly in registers (nop <= 9 at order 2, so this is ~120
//           FMAs) and solves for column k = its group lane of X = A^-1 diag(q!), followed by one step of iterative
//           refinement against A kept in shared memory and the reference's max-norm consistency test
//           (src/MathUtils/MatrixXd.cpp:40-47).
//   pass 2  X goes to shared memory; lanes evaluate op_k(i,j) = (sum_a X[a][k] eta^{q_a}) * bw / delta^|q_k|
//           for their bonds and write the full op vector (AoS, [bond][nop]) and/or the Navier subset
//           (SoA, [c][bond]) used by the explicit fracture step.
// MIXED: bond weights, monomials and moment products in FP32 with two-sum compensated accumulation on
// delta-scaled bond vectors (the bond vector itself is formed in FP64); the factorisation, refinement and
// g-evaluation stay in FP64, the evaluation using the same FP32 weights and monomials that entered the moment
// sums (so sum_j g_j m(xi_j) reproduces diag(q!) for the matrix actually factored); g is stored in FP32, and
// at order 2 the first moments of the stored second-derivative operators are kept per node (the apply's
// defect correction).  MIXED with SUMS64: the same FP32 storage and defects, with the moment sums in FP64
// (on B200 an FP64 FMA costs less issue than an FP32 two-sum, so this variant is the faster and the more
// accurate one; the batch autotuner may pick it).
#include <cfloat>
#include <type_traits>

#include "k_kernels.h"
#include "pxb_common.cuh"

namespace pxb {

// One node per group of LPN lanes (a power of two >= nop; the caller maps 32/LPN groups onto a warp, all
// lanes of the warp call this together).  i is the node (act false: idle group); sA and sX are this group's
// nop x nop shared-memory slots.  Positions are read at pos[j - a.node_base] and the AoS operators written at
// ops[(t - a.bond_base) * nop], so a batch of clouds can address one cloud's slices with global ids.
template <int DIM, int ORDER, bool MIXED, int LPN, bool SUMS64 = false>
__device__ __forceinline__ void gbuild_group(const GBuildArgs &a, int i, bool act, int gl, double *sA, double *sX) {
    constexpr QTable<DIM, ORDER> Q{};
    constexpr int NOP = Q.NOP;
    constexpr int NE = NOP * (NOP + 1) / 2;
    static_assert(LPN >= NOP, "one lane per solve column");
    using PosT = typename Vec<DIM>::T;
    const PosT *pos = static_cast<const PosT *>(a.pos);
    const double inv_delta = 1.0 / a.delta;

    double idpow[NOP];
#pragma unroll
    for (int k = 0; k < NOP; ++k) {
        double v = 1.0;
#pragma unroll
        for (int t = 0; t < Q.p[k] + Q.q[k] + Q.r[k]; ++t) v *= inv_delta;
        idpow[k] = v;
    }
    {
        const int b0 = act ? a.off[i] : 0, b1 = act ? a.off[i + 1] : 0;
        const PosT xi = act ? pos[i - a.node_base] : PosT{};

        // ---- pass 1: moment sums ----
        double acc[NE];
        CompF cacc[(MIXED && !SUMS64) ? NE : 1];
#pragma unroll
        for (int e = 0; e < NE; ++e) acc[e] = 0.0;
        int usable = 0;
        // weights of this lane's first KC bonds, reused by pass 2 (0 marks a skipped bond)
        constexpr int KC = 4;
        using ET = typename std::conditional<MIXED && !SUMS64, float, double>::type;
        ET wcache[KC];
#pragma unroll
        for (int c = 0; c < KC; ++c) wcache[c] = ET(0);
        int cidx = 0;
        for (int t = b0 + gl; t < b1; t += LPN, ++cidx) {
            const int j = a.nbr[t];
            const PosT xj = pos[j - a.node_base];
            const double dx = xj.x - xi.x, dy = xj.y - xi.y;
            double dz = 0.0;
            if constexpr (DIM == 3) dz = xj.z - xi.z;
            const double xn = sqrt(dx * dx + dy * dy + dz * dz);
            if (xn <= 0.0) continue;
            if constexpr (MIXED && !SUMS64) {
                const float r = 2.0f * (float)(xn * inv_delta);
                const float w = expf(-r * r);
                float vc = 1.0f;
                if (a.dx_char > 0.0 && xn > a.delta - 0.5 * a.dx_char)
                    vc = fminf(fmaxf((float)((a.delta - xn + 0.5 * a.dx_char) / a.dx_char), 0.f), 1.f);
                const float bw = w * vc * (float)a.vol[j];
                if (!(bw > 0.f)) continue;
                ++usable;
#pragma unroll
                for (int c = 0; c < KC; ++c)
                    if (c == cidx) wcache[c] = bw;
                float m[NOP];
                monomials<DIM, ORDER, float>((float)(dx * inv_delta), (float)(dy * inv_delta),
                                             (float)(dz * inv_delta), m);
                int e = 0;
#pragma unroll
                for (int p = 0; p < NOP; ++p)
#pragma unroll
                    for (int q = p; q < NOP; ++q) cacc[e++].add(bw * m[p] * m[q]);
            } else {
                const double bw = bond_weight(xn, a.delta) * rim_correction(xn, a.delta, a.dx_char) * a.vol[j];
                if (!(bw > 0.0)) continue;
                ++usable;
#pragma unroll
                for (int c = 0; c < KC; ++c)
                    if (c == cidx) wcache[c] = bw;
                double m[NOP];
                monomials<DIM, ORDER, double>(dx * inv_delta, dy * inv_delta, dz * inv_delta, m);
                int e = 0;
#pragma unroll
                for (int p = 0; p < NOP; ++p)
#pragma unroll
                    for (int q = p; q < NOP; ++q) acc[e++] += bw * m[p] * m[q];
            }
        }
        if constexpr (MIXED && !SUMS64) {
#pragma unroll
            for (int e = 0; e < NE; ++e) acc[e] = cacc[e].value();
        }
#pragma unroll
        for (int e = 0; e < NE; ++e) acc[e] = group_sum<LPN>(acc[e]);
        usable = group_sum_int<LPN>(usable);

        // keep A (full, row-major) in shared memory for the refinement residual and the consistency test
        if (gl == 0) {
            int e = 0;
#pragma unroll
            for (int p = 0; p < NOP; ++p)
#pragma unroll
                for (int q = p; q < NOP; ++q) {
                    sA[p * NOP + q] = acc[e];
                    sA[q * NOP + p] = acc[e];
                    ++e;
                }
        }
        __syncwarp();

        // ---- solve: in-place L D L^T of the packed upper triangle (acc[e] holds row p, col q>=p) ----
        // index of (p,q), q>=p, in the packed upper triangle
        auto U = [&](int p, int q) -> int { return p * NOP - p * (p - 1) / 2 + (q - p); };
#pragma unroll
        for (int j = 0; j < NOP; ++j) {
            double d = acc[U(j, j)];
#pragma unroll
            for (int k = 0; k < j; ++k) d -= acc[U(k, j)] * acc[U(k, j)] * acc[U(k, k)];
            acc[U(j, j)] = d;
            const double invd = 1.0 / d;
#pragma unroll
            for (int i2 = j + 1; i2 < NOP; ++i2) {
                double s = acc[U(j, i2)];
#pragma unroll
                for (int k = 0; k < j; ++k) s -= acc[U(k, i2)] * acc[U(k, j)] * acc[U(k, k)];
                acc[U(j, i2)] = s * invd;  // L[i2][j] stored at packed (j, i2)
            }
        }
        const int kcol = (gl < NOP) ? gl : 0;
        double fk = 0.0;
#pragma unroll
        for (int q = 0; q < NOP; ++q)
            if (q == kcol) fk = Q.fact[q];
        auto ldl_solve = [&](double *x) {
            // x holds the rhs on entry
#pragma unroll
            for (int i2 = 0; i2 < NOP; ++i2) {
#pragma unroll
                for (int j = 0; j < i2; ++j) x[i2] -= acc[U(j, i2)] * x[j];
            }
#pragma unroll
            for (int i2 = 0; i2 < NOP; ++i2) x[i2] /= acc[U(i2, i2)];
#pragma unroll
            for (int i2 = NOP - 1; i2 >= 0; --i2) {
#pragma unroll
                for (int j = i2 + 1; j < NOP; ++j) x[i2] -= acc[U(i2, j)] * x[j];
            }
        };
        double x[NOP];
#pragma unroll
        for (int q = 0; q < NOP; ++q) x[q] = (q == kcol) ? fk : 0.0;
        ldl_solve(x);
        // consistency test of the direct solution (MatrixXd.cpp:40-47):
        //   max|A X - B| <= 1e-8 * max(max|B|, max|A| max|X|)
        // its residual r = b - A x then drives one step of iterative refinement: x += A^-1 r
        double r[NOP];
        double res = 0.0, maxA = 0.0, maxX = 0.0;
#pragma unroll
        for (int p = 0; p < NOP; ++p) {
            double sres = (p == kcol) ? fk : 0.0;
#pragma unroll
            for (int q = 0; q < NOP; ++q) {
                const double apq = sA[p * NOP + q];
                sres -= apq * x[q];
                maxA = fmax(maxA, fabs(apq));
            }
            r[p] = sres;
            res = fmax(res, fabs(sres));
            maxX = fmax(maxX, fabs(x[p]));
        }
        ldl_solve(r);
#pragma unroll
        for (int q = 0; q < NOP; ++q) x[q] += r[q];
        if (gl >= NOP) { res = 0.0; maxX = 0.0; }
        res = group_max<LPN>(res);
        maxX = group_max<LPN>(maxX);
        double maxB = 0.0;
#pragma unroll
        for (int q = 0; q < NOP; ++q) maxB = fmax(maxB, Q.fact[q]);
        const double scale = fmax(fmax(maxB, maxA * maxX), DBL_MIN);
        const bool consistent = (res <= 1.0e-8 * scale);  // NaN-safe: NaN fails
        const bool degenerate = (usable < NOP) || !consistent;
        const bool deep_ghost = act && (a.layer != nullptr) && (a.layer[i] > 1);
        const bool zero_ops = degenerate;
        if (act && gl == 0) {
            if (a.degenerate) a.degenerate[i] = degenerate ? 1 : 0;
            if (degenerate && !deep_ghost) {
                atomicAdd(a.n_degenerate, 1u);
                atomicMin(a.first_degenerate, i);
            }
        }
        // X (column kcol in lane kcol) to shared memory: sX[a][k]
        if (gl < NOP) {
#pragma unroll
            for (int p = 0; p < NOP; ++p) sX[p * NOP + gl] = zero_ops ? 0.0 : x[p];
        }
        __syncwarp();

        // ---- pass 2: per-bond operators, evaluated in FP64 (mixed mode stores them in FP32; its weights are
        //      the FP32 ones the moment sums used) ----
        // mixed, order 2: first moments of the stored second-derivative operators (see GBuildArgs::defect)
        constexpr bool DEF = MIXED && ORDER == 2;
        constexpr int ND = DEF ? (NOP - DIM) * DIM : 1;
        double dsum[ND];
#pragma unroll
        for (int e = 0; e < ND; ++e) dsum[e] = 0.0;
        cidx = 0;
        for (int t = b0 + gl; t < b1; t += LPN, ++cidx) {
            const int j = a.nbr[t];
            const PosT xj = pos[j - a.node_base];
            const double dx = xj.x - xi.x, dy = xj.y - xi.y;
            double dz = 0.0;
            if constexpr (DIM == 3) dz = xj.z - xi.z;
            ET bw = ET(0);
            if (cidx < KC) {
#pragma unroll
                for (int c = 0; c < KC; ++c)
                    if (c == cidx) bw = wcache[c];
            } else {
                const double xn = sqrt(dx * dx + dy * dy + dz * dz);
                if (xn > 0.0) {
                    if constexpr (MIXED && !SUMS64) {
                        const float rr = 2.0f * (float)(xn * inv_delta);
                        float vc = 1.0f;
                        if (a.dx_char > 0.0 && xn > a.delta - 0.5 * a.dx_char)
                            vc = fminf(fmaxf((float)((a.delta - xn + 0.5 * a.dx_char) / a.dx_char), 0.f), 1.f);
                        bw = expf(-rr * rr) * vc * (float)a.vol[j];
                    } else {
                        bw = bond_weight(xn, a.delta) * rim_correction(xn, a.delta, a.dx_char) * a.vol[j];
                    }
                }
            }
            const bool live = bw > ET(0);
            const double bwd = (double)bw;
            double m[NOP];
            if constexpr (MIXED && !SUMS64) {
                // the FP32 monomials pass 1 summed, so the moment conditions hold for the factored matrix
                float mf[NOP];
                monomials<DIM, ORDER, float>((float)(dx * inv_delta), (float)(dy * inv_delta), (float)(dz * inv_delta),
                                             mf);
#pragma unroll
                for (int k = 0; k < NOP; ++k) m[k] = (double)mf[k];
            } else {
                monomials<DIM, ORDER, double>(dx * inv_delta, dy * inv_delta, dz * inv_delta, m);
            }
            auto op = [&](int k) -> double {
                if (!live) return 0.0;
                double sum = 0.0;
#pragma unroll
                for (int p = 0; p < NOP; ++p) sum += sX[p * NOP + k] * m[p];
                return sum * bwd * idpow[k];
            };
            if (a.ops) {
                if constexpr (MIXED) {
                    float *o = static_cast<float *>(a.ops) + (size_t)(t - a.bond_base) * NOP;
#pragma unroll
                    for (int k = 0; k < NOP; ++k) {
                        const float gk = (float)op(k);
                        o[k] = gk;
                        if constexpr (DEF) {
                            if (k >= DIM) {
                                dsum[(k - DIM) * DIM + 0] += (double)gk * dx;
                                dsum[(k - DIM) * DIM + 1] += (double)gk * dy;
                                if constexpr (DIM == 3) dsum[(k - DIM) * DIM + 2] += (double)gk * dz;
                            }
                        }
                    }
                } else {
                    double *o = static_cast<double *>(a.ops) + (size_t)(t - a.bond_base) * NOP;
#pragma unroll
                    for (int k = 0; k < NOP; ++k) o[k] = op(k);
                }
            }
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
                    const double v = op(sl[c]);
                    if constexpr (MIXED) static_cast<float *>(a.G)[(size_t)c * a.nb + t] = (float)v;
                    else static_cast<double *>(a.G)[(size_t)c * a.nb + t] = v;
                }
            }
        }
        if constexpr (DEF) {
            if (a.defect) {
                float *dst = a.defect + (size_t)(i - a.node_base) * ND;
#pragma unroll
                for (int e = 0; e < ND; ++e) {
                    const double v = group_sum<LPN>(dsum[e]);
                    if (act && gl == (e & (LPN - 1))) dst[e] = (float)v;
                }
            }
        }
        __syncwarp();
    }
}

// single geometry: GPW = 32/LPN nodes per warp, grid-stride over the nodes
template <int DIM, int ORDER, bool MIXED, int LPN>
__global__ void __launch_bounds__(kGbuildThreads) gbuild_kernel(GBuildArgs a) {
    constexpr int NOP = QTable<DIM, ORDER>::NOP;
    constexpr int GPW = kWarp / LPN;
    constexpr int GPB = (kGbuildThreads / kWarp) * GPW;  // node groups per block
    __shared__ double sA[GPB][NOP * NOP];
    __shared__ double sX[GPB][NOP * NOP];
    const int lane = threadIdx.x & 31;
    const int gl = lane & (LPN - 1);
    const int wib = (threadIdx.x >> 5) * GPW + lane / LPN;  // node group index within the block
    const long long stride = (long long)gridDim.x * GPB;
    for (long long base = (long long)blockIdx.x * GPB + (threadIdx.x >> 5) * GPW; base < a.n + 0LL; base += stride) {
        const int i = (int)(base + lane / LPN);
        gbuild_group<DIM, ORDER, MIXED, LPN>(a, i, i < a.n, gl, sA[wib], sX[wib]);
    }
}

template <int DIM, int ORDER, int LPN>
static cudaError_t launch_order(const GBuildArgs &a, bool mixed, int grid, cudaStream_t s) {
    constexpr int GPB = (kGbuildThreads / kWarp) * (kWarp / LPN);
    const long long need = ((long long)a.n + GPB - 1) / GPB;
    const int g = (int)(need < grid ? (need > 0 ? need : 1) : grid);
    if (mixed) gbuild_kernel<DIM, ORDER, true, LPN><<<g, kGbuildThreads, 0, s>>>(a);
    else gbuild_kernel<DIM, ORDER, false, LPN><<<g, kGbuildThreads, 0, s>>>(a);
    return cudaGetLastError();
}

// lanes per node: 8 for 2D order <= 2 (families of ~12-30 bonds: ~4 bonds per lane, 4 nodes per warp), 16 when
// nop > 8, 32 for 3D order 2 (families of ~40-122 bonds)
cudaError_t launch_gbuild(const GBuildArgs &a, int dim, int order, bool mixed, int grid, cudaStream_t s) {
    if (dim == 2) {
        switch (order) {
            case 1: return launch_order<2, 1, 8>(a, mixed, grid, s);
            case 2: return launch_order<2, 2, 8>(a, mixed, grid, s);
            case 3: return launch_order<2, 3, 16>(a, mixed, grid, s);
            default: return cudaErrorInvalidValue;
        }
    }
    switch (order) {
        case 1: return launch_order<3, 1, 8>(a, mixed, grid, s);
        case 2: return launch_order<3, 2, 32>(a, mixed, grid, s);
        default: return cudaErrorInvalidValue;
    }
}

// ---- batched clouds: persistent warps over a task table (order 2) --------------------------------------------
// DIMS selects the task kinds this instantiation handles (1: 2D, 2: 3D, 3: both); a warp runs its task's nodes
// 32/LPN at a time with the single-geometry group code, addressing the cloud's slices through node_base /
// bond_base.
template <bool MIXED, int LPN2, int LPN3, int DIMS, bool SUMS64>
__global__ void __launch_bounds__(kGbuildThreads) gbuild_batch_kernel(BatchArgs b) {
    constexpr int WPB = kGbuildThreads / kWarp;
    constexpr int S2 = (kWarp / LPN2) * 25, S3 = (kWarp / LPN3) * 81;
    constexpr int SLOT = (DIMS & 2) ? ((DIMS & 1) ? (S2 > S3 ? S2 : S3) : S3) : S2;
    __shared__ double sA[WPB][SLOT];
    __shared__ double sX[WPB][SLOT];
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
        a.ops = MIXED ? (void *)(static_cast<float *>(b.ops) + cd.ops_off) : (void *)(static_cast<double *>(b.ops) + cd.ops_off);
        a.degenerate = b.degenerate;
        a.n_degenerate = b.n_degenerate;
        a.first_degenerate = b.first_degenerate;
        a.node_base = cd.node0;
        a.bond_base = cd.bond0;
        a.defect = (MIXED && b.defect) ? b.defect + cd.def_off : nullptr;
        if constexpr ((DIMS & 1) != 0) {
            if (tk.dim == 2) {
                constexpr int GPW = kWarp / LPN2;
                const int gl = lane & (LPN2 - 1), grp = lane / LPN2;
                for (int k0 = 0; k0 < tk.count; k0 += GPW) {
                    const bool act = k0 + grp < tk.count;
                    gbuild_group<2, 2, MIXED, LPN2, SUMS64>(a, tk.first + (act ? k0 + grp : 0), act, gl, &sA[w][grp * 25],
                                                    &sX[w][grp * 25]);
                }
            }
        }
        if constexpr ((DIMS & 2) != 0) {
            if (tk.dim == 3) {
                constexpr int GPW = kWarp / LPN3;
                const int gl = lane & (LPN3 - 1), grp = lane / LPN3;
                for (int k0 = 0; k0 < tk.count; k0 += GPW) {
                    const bool act = k0 + grp < tk.count;
                    gbuild_group<3, 2, MIXED, LPN3, SUMS64>(a, tk.first + (act ? k0 + grp : 0), act, gl, &sA[w][grp * 81],
                                                    &sX[w][grp * 81]);
                }
            }
        }
        __syncwarp();
    }
}

// schedules 4 and 5 (mixed only; identical to 2 and 3 in FP64) sum the moments in FP64 (SUMS64); 6 and 7 run one
// warp per node (FP64 moment sums in both precisions), in one launch or one per dimension
BatchSchedule batch_gbuild_schedule(int v) {
    switch (v) {
        case 0: return {8, 32, false};
        case 1: return {16, 32, false};
        case 2: return {8, 16, false};
        case 3: return {8, 32, true};
        case 4: return {8, 16, false};
        case 5: return {8, 32, true};
        case 6: return {32, 32, false, true};
        case 7: return {32, 32, true, true};
        case 8: return {32, 32, false, true, true};
        default: return {8, 32, true, true, false, true};
    }
}

template <bool MIXED, int LPN2, int LPN3, int DIMS, bool SUMS64 = false>
static cudaError_t launch_gb(const BatchArgs &a, cudaStream_t s) {
    auto k = gbuild_batch_kernel<MIXED, LPN2, LPN3, DIMS, SUMS64>;
    int dev = 0, sms = 148, per_sm = 1;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, kGbuildThreads, 0);
    const long long want = ((long long)a.ntasks + (kGbuildThreads / kWarp) - 1) / (kGbuildThreads / kWarp);
    const long long cap = (long long)sms * (per_sm > 0 ? per_sm : 1);
    const int grid = (int)(want < cap ? (want > 0 ? want : 1) : cap);
    k<<<grid, kGbuildThreads, 0, s>>>(a);
    return cudaGetLastError();
}

template <bool MIXED>
static cudaError_t launch_gb_m(const BatchArgs &a, int variant, int dims, cudaStream_t s) {
    switch (variant) {
        case 0: return launch_gb<MIXED, 8, 32, 3>(a, s);
        case 1: return launch_gb<MIXED, 16, 32, 3>(a, s);
        case 2: return launch_gb<MIXED, 8, 16, 3>(a, s);
        case 3: return dims == 1 ? launch_gb<MIXED, 8, 32, 1>(a, s) : launch_gb<MIXED, 8, 32, 2>(a, s);
        case 4: return launch_gb<MIXED, 8, 16, 3, MIXED>(a, s);
        default:
            return dims == 1 ? launch_gb<MIXED, 8, 32, 1, MIXED>(a, s) : launch_gb<MIXED, 8, 32, 2, MIXED>(a, s);
    }
}

cudaError_t launch_gbuild_batch(const BatchArgs &a, bool mixed, int variant, int dims, cudaStream_t s) {
    const BatchSchedule sch = batch_gbuild_schedule(variant);
    if (sch.hybrid && dims == 1)  // the 2D launch of the hybrid schedule: lane groups (FP64 sums for MIXED)
        return mixed ? launch_gb<true, 8, 32, 1, true>(a, s) : launch_gb<false, 8, 32, 1, false>(a, s);
    if (sch.warp) return launch_gbuild_batch_warp(a, mixed, sch.split, dims, sch.tc, s);
    return mixed ? launch_gb_m<true>(a, variant, dims, s) : launch_gb_m<false>(a, variant, dims, s);
}

bool gbuild_supported(int dim, int order) { return (dim == 2 && order >= 1 && order <= 3) || (dim == 3 && order >= 1 && order <= 2); }

}  // namespace pxb
