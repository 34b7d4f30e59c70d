// CSR Jacobian value assembly (reference PDSystem::formResidualAndJacobianParallel,
// src/PDSystem/FormResidualAndJacobianParallel.cpp:114-171, with the element callbacks of
// src/ElmtSystem/PoissonElement.cpp:26-58, DiffusionElement.cpp and CahnHilliardElement.cpp:178-292).
//
// Row ownership: node i owns its ndof rows, so no atomics.  The bond -> CSR slot map is computed once
// (csr_map_kernel, a binary search per bond at setup), replacing the per-assembly binary search of the
// reference (devFindSlot, src/PDSystem/CudaAssembleKernels.cu:157-168).  Sign convention K = -dF/dU,
// RHS = +F.
#include "k_kernels.h"
#include "pxb_common.cuh"

namespace pxb {

__device__ __forceinline__ double ch_clamp(double c) { return fmax(1.0e-8, fmin(1.0 - 1.0e-8, c)); }

__device__ __forceinline__ int find_slot(const int *cols, int lo, int hi, int target) {
    int l = lo, h = hi - 1;
    while (l <= h) {
        const int mid = l + ((h - l) >> 1);
        const int c = cols[mid];
        if (c == target) return mid;
        if (c < target) l = mid + 1; else h = mid - 1;
    }
    return -1;
}

__global__ void csr_map_kernel(CsrMapArgs a) {
    const int nd = a.ndof;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < a.n; i += gridDim.x * blockDim.x) {
        for (int r = 0; r < nd; ++r) {
            const int row = i * nd + r;
            const int lo = a.rowptr[row], hi = a.rowptr[row + 1];
            for (int c = 0; c < nd; ++c) {
                const int s = find_slot(a.cols, lo, hi, i * nd + c);
                a.diag[(size_t)i * nd * nd + r * nd + c] = s;
                if (s < 0) atomicAdd(a.missing, 1);
            }
            for (int t = a.off[i]; t < a.off[i + 1]; ++t) {
                const int j = a.nbr[t];
                for (int c = 0; c < nd; ++c) {
                    const int s = find_slot(a.cols, lo, hi, j * nd + c);
                    a.slot[(size_t)t * nd * nd + r * nd + c] = s;
                    if (s < 0) atomicAdd(a.missing, 1);
                }
            }
        }
        if (a.extra) {
            // the mirror block, when the mirror node is not a family member, and whether the rows hold anything else
            const int m = a.mirror ? a.mirror[i] - 1 : -1;
            bool in_fam = m == i;
            for (int t = a.off[i]; t < a.off[i + 1] && m >= 0 && !in_fam; ++t) in_fam = a.nbr[t] == m;
            const bool extra = m >= 0 && !in_fam;
            const int width = nd * (1 + (a.off[i + 1] - a.off[i]) + (extra ? 1 : 0));
            for (int r = 0; r < nd; ++r) {
                const int row = i * nd + r;
                const int lo = a.rowptr[row], hi = a.rowptr[row + 1];
                if (hi - lo != width) atomicAdd(a.inexact, 1);
                for (int c = 0; c < nd; ++c)
                    a.extra[(size_t)i * nd * nd + r * nd + c] = extra ? find_slot(a.cols, lo, hi, m * nd + c) : -1;
            }
        }
    }
}

cudaError_t launch_csr_map(const CsrMapArgs &a, cudaStream_t s) {
    const int g = (a.n + 127) / 128;
    csr_map_kernel<<<g > 0 ? g : 1, 128, 0, s>>>(a);
    return cudaGetLastError();
}

// ---- scalar elements: Poisson (type 0): coeff = sigma*Lap, R_n = f;  diffusion (type 1): coeff = -D*Lap,
//      R_n = (u-uold)/dt - f, K_n = 1/dt.  Bond: R = coeff (u_j-u_i), K_II = -coeff, K_IJ = coeff. ----------
template <bool MIXED>
__global__ void __launch_bounds__(256) assemble_scalar_kernel(ScalarAsmArgs a) {
    constexpr int WPB = 256 / kWarp;
    const int lane = threadIdx.x & 31;
    const int wib = threadIdx.x >> 5;
    for (int i = blockIdx.x * WPB + wib; i < a.n; i += gridDim.x * WPB) {
        const int r0 = a.rowptr[i], r1 = a.rowptr[i + 1];
        for (int s = r0 + lane; s < r1; s += kWarp) a.kvals[s] = 0.0;
        __syncwarp();
        if (a.degenerate && a.degenerate[i]) {  // reference GPU: a singular moment system zeroes the row
            if (lane == 0) a.rhs[i] = 0.0;
            continue;
        }
        const double ui = a.u[i];
        const int b0 = a.off[i], b1 = a.off[i + 1];
        double rsum = 0.0, dsum = 0.0;
        for (int t = b0 + lane; t < b1; t += kWarp) {
            const int j = __ldg(a.nbr + t);
            double lap;
            if constexpr (MIXED) {
                const float *g = static_cast<const float *>(a.ops) + (size_t)t * a.nop;
                lap = (double)g[a.s_xx] + (double)g[a.s_yy];
                if (a.dim >= 3) lap += (double)g[a.s_zz];
            } else {
                const double *g = static_cast<const double *>(a.ops) + (size_t)t * a.nop;
                lap = g[a.s_xx] + g[a.s_yy];
                if (a.dim >= 3) lap += g[a.s_zz];
            }
            const double coeff = (a.type == 0) ? a.coef * lap : -a.coef * lap;
            rsum += coeff * (a.u[j] - ui);
            dsum += coeff;                       // -K_II
            a.kvals[a.slot[t]] = -coeff;         // -K_IJ
        }
        rsum = group_sum<kWarp>(rsum);
        dsum = group_sum<kWarp>(dsum);
        if (lane == 0) {
            double rn, kn;
            const double fi = a.f_node ? a.f_node[i] : a.f;
            if (a.type == 0) { rn = fi; kn = 0.0; }
            else { rn = (ui - a.uold[i]) / a.dt - fi; kn = 1.0 / a.dt; }
            a.kvals[a.diag[i]] = -kn + dsum;
            a.rhs[i] = rn + rsum;
        }
    }
}

cudaError_t launch_assemble_scalar(const ScalarAsmArgs &a, cudaStream_t s) {
    const int g = (a.n + 7) / 8;
    if (a.mixed) assemble_scalar_kernel<true><<<g > 0 ? g : 1, 256, 0, s>>>(a);
    else assemble_scalar_kernel<false><<<g > 0 ? g : 1, 256, 0, s>>>(a);
    return cudaGetLastError();
}

// ---- stress-coupled Cahn-Hilliard (reference src/PDSystem/CudaAssembleKernels.cu:685-874): rows c, mu, u.
//      Per bond: the species flux w_ij = 0.5 (M_i g2_ij + V_j/V_i M_j g2_ji) (dropped on ghost bonds) on the
//      c-row, the gradient energy kappa g2_ij and the hydrostatic coupling Omega Kh grad(u) on the mu-row, the
//      Navier operators and the chemo-mechanical body force -A grad(c) on the u-rows; the mechanical terms are
//      gated by g = 1 (intact) or kres (broken).  Nodal: (c - c_old)/dt, mu - f'(c) + Omega Ch (c - cref), and
//      the optional backward-Euler inertia -rho (u - u_old - v dt)/dt^2.  K_IJ is stored per bond; the
//      diagonal block accumulates the nodal Jacobian plus the sum of K_IJ (K_II = -K_IJ per bond). ----------
template <int DIM>
__global__ void __launch_bounds__(256) assemble_stress_ch_kernel(StressChAsmArgs a) {
    constexpr int WPB = 256 / kWarp;
    constexpr int ND = DIM + 2;
    // distinct per-bond coefficients: coeff_c, kappaLap, cmu[DIM], cb[DIM], then the Navier block
    // 2D: p11 pxy p22;  3D: p11 p22 p33 p12 p13 p23
    constexpr int NK = 2 + 2 * DIM + (DIM == 3 ? 6 : 3);
    const int lane = threadIdx.x & 31;
    const int wib = threadIdx.x >> 5;
    const int *sl = a.sl;
    for (int i = blockIdx.x * WPB + wib; i < a.n; i += gridDim.x * WPB) {
        const int rb = i * ND;
        for (int s = a.rowptr[rb] + lane; s < a.rowptr[rb + ND]; s += kWarp) a.kvals[s] = 0.0;
        __syncwarp();
        if (a.degenerate && a.degenerate[i]) {  // singular moment system: the rows stay zero
            if (lane < ND) a.rhs[rb + lane] = 0.0;
            continue;
        }
        double uI[ND];
#pragma unroll
        for (int b = 0; b < ND; ++b) uI[b] = a.u[rb + b];
        const double Vi = a.vol[i], Mi = a.mnode[i];
        double R[ND], S[NK];
#pragma unroll
        for (int b = 0; b < ND; ++b) R[b] = 0.0;
#pragma unroll
        for (int k = 0; k < NK; ++k) S[k] = 0.0;
        for (int t = a.off[i] + lane; t < a.off[i + 1]; t += kWarp) {
            const int j = __ldg(a.nbr + t);
            const double *op = a.ops + (size_t)t * a.nop;
            const double g = a.health ? (a.health[t] > 0.0 ? 1.0 : a.kres) : 1.0;
            double G1[DIM];
#pragma unroll
            for (int d = 0; d < DIM; ++d) G1[d] = g * op[sl[d]];
            const double Gxx = g * op[sl[3]], Gxy = g * op[sl[4]], Gyy = g * op[sl[5]];
            const bool ghostJ = a.ghost && a.ghost[j];
            const double g2A = a.lap[t];
            double coeff_c = 0.0;
            if (!ghostJ) {
                const int r = a.rev[t];
                const double w = (r >= 0 && Vi > 0.0) ? 0.5 * (Mi * g2A + (a.vol[j] / Vi) * a.mnode[j] * a.lap[r])
                                                      : Mi * g2A;
                coeff_c = -w;
            }
            const double kappaLap = ghostJ ? 0.0 : a.kappa * g2A;
            double k[NK];
            k[0] = coeff_c;
            k[1] = kappaLap;
#pragma unroll
            for (int d = 0; d < DIM; ++d) {
                k[2 + d] = a.Omega * a.Kh * G1[d];
                k[2 + DIM + d] = -a.A * G1[d];
            }
            double du[DIM];
            const double dC = a.u[(size_t)j * ND] - uI[0], dMu = a.u[(size_t)j * ND + 1] - uI[1];
#pragma unroll
            for (int d = 0; d < DIM; ++d) du[d] = a.u[(size_t)j * ND + 2 + d] - uI[2 + d];
            double Kb[ND][ND];
#pragma unroll
            for (int r = 0; r < ND; ++r)
#pragma unroll
                for (int c = 0; c < ND; ++c) Kb[r][c] = 0.0;
            Kb[0][1] = coeff_c;
            Kb[1][0] = kappaLap;
#pragma unroll
            for (int d = 0; d < DIM; ++d) {
                Kb[1][2 + d] = k[2 + d];
                Kb[2 + d][0] = k[2 + DIM + d];
            }
            constexpr int P0 = 2 + 2 * DIM;
            if constexpr (DIM == 2) {
                k[P0 + 0] = a.C11 * Gxx + a.C66 * Gyy;          // p11
                k[P0 + 1] = (a.C12 + a.C66) * Gxy;              // pxy
                k[P0 + 2] = a.C66 * Gxx + a.C11 * Gyy;          // p22
                Kb[2][2] = k[P0];
                Kb[2][3] = Kb[3][2] = k[P0 + 1];
                Kb[3][3] = k[P0 + 2];
            } else {
                const double Gzz = g * op[sl[8]], Gxz = g * op[sl[6]], Gyz = g * op[sl[7]];
                const double cc = a.C12 + a.C66;
                k[P0 + 0] = a.C11 * Gxx + a.C66 * (Gyy + Gzz);  // p11
                k[P0 + 1] = a.C11 * Gyy + a.C66 * (Gxx + Gzz);  // p22
                k[P0 + 2] = a.C11 * Gzz + a.C66 * (Gxx + Gyy);  // p33
                k[P0 + 3] = cc * Gxy;                           // p12
                k[P0 + 4] = cc * Gxz;                           // p13
                k[P0 + 5] = cc * Gyz;                           // p23
                Kb[2][2] = k[P0];
                Kb[3][3] = k[P0 + 1];
                Kb[4][4] = k[P0 + 2];
                Kb[2][3] = Kb[3][2] = k[P0 + 3];
                Kb[2][4] = Kb[4][2] = k[P0 + 4];
                Kb[3][4] = Kb[4][3] = k[P0 + 5];
            }
            // residual of this bond: R = K_IJ (u_j - u_i) row by row
            R[0] += coeff_c * dMu;
            double r1 = kappaLap * dC;
#pragma unroll
            for (int d = 0; d < DIM; ++d) r1 += k[2 + d] * du[d];
            R[1] += r1;
#pragma unroll
            for (int d = 0; d < DIM; ++d) {
                double rd = k[2 + DIM + d] * dC;
#pragma unroll
                for (int e = 0; e < DIM; ++e) rd += Kb[2 + d][2 + e] * du[e];
                R[2 + d] += rd;
            }
#pragma unroll
            for (int q = 0; q < NK; ++q) S[q] += k[q];
            const int *st = a.slot + (size_t)t * ND * ND;
#pragma unroll
            for (int r = 0; r < ND; ++r)
#pragma unroll
                for (int c = 0; c < ND; ++c) a.kvals[st[r * ND + c]] = -Kb[r][c];
        }
#pragma unroll
        for (int b = 0; b < ND; ++b) R[b] = group_sum<kWarp>(R[b]);
#pragma unroll
        for (int q = 0; q < NK; ++q) S[q] = group_sum<kWarp>(S[q]);
        if (lane == 0) {
            const double c = uI[0], mu = uI[1], cold = a.uold ? a.uold[rb] : 0.0;
            const double cc = ch_clamp(c);
            const double fp = log(cc / (1.0 - cc)) + a.chi * (1.0 - 2.0 * cc);
            const double fpp = 1.0 / (cc * (1.0 - cc)) - 2.0 * a.chi;
            double rl[ND], kii[ND][ND];
#pragma unroll
            for (int r = 0; r < ND; ++r) {
                rl[r] = 0.0;
#pragma unroll
                for (int q = 0; q < ND; ++q) kii[r][q] = 0.0;
            }
            rl[0] = (c - cold) / a.dt;
            rl[1] = mu - fp + a.Omega * a.Ch * (c - a.cref);
            kii[0][0] = -(1.0 / a.dt);
            kii[1][0] = -(-fpp + a.Omega * a.Ch);
            kii[1][1] = -(1.0);
            if (a.rho > 0.0 && a.vel) {
                const double c0 = a.rho / (a.dt * a.dt);
#pragma unroll
                for (int d = 0; d < DIM; ++d) {
                    const double uo = a.uold ? a.uold[rb + 2 + d] : 0.0;
                    rl[2 + d] += -c0 * (uI[2 + d] - uo - a.vel[(size_t)i * DIM + d] * a.dt);
                    kii[2 + d][2 + d] += c0;
                }
            }
            // kii += sum over bonds of K_IJ (= -K_II)
            constexpr int P0 = 2 + 2 * DIM;
            kii[0][1] += S[0];
            kii[1][0] += S[1];
#pragma unroll
            for (int d = 0; d < DIM; ++d) {
                kii[1][2 + d] += S[2 + d];
                kii[2 + d][0] += S[2 + DIM + d];
            }
            if constexpr (DIM == 2) {
                kii[2][2] += S[P0];
                kii[2][3] += S[P0 + 1];
                kii[3][2] += S[P0 + 1];
                kii[3][3] += S[P0 + 2];
            } else {
                kii[2][2] += S[P0];
                kii[3][3] += S[P0 + 1];
                kii[4][4] += S[P0 + 2];
                kii[2][3] += S[P0 + 3];
                kii[3][2] += S[P0 + 3];
                kii[2][4] += S[P0 + 4];
                kii[4][2] += S[P0 + 4];
                kii[3][4] += S[P0 + 5];
                kii[4][3] += S[P0 + 5];
            }
            const int *dg = a.diag + (size_t)i * ND * ND;
#pragma unroll
            for (int r = 0; r < ND; ++r) {
#pragma unroll
                for (int q = 0; q < ND; ++q) a.kvals[dg[r * ND + q]] = kii[r][q];
                a.rhs[rb + r] = rl[r] + R[r];
            }
        }
    }
}

cudaError_t launch_assemble_stress_ch(const StressChAsmArgs &a, cudaStream_t s) {
    const int g = (a.n + 7) / 8;
    if (a.dim == 3) assemble_stress_ch_kernel<3><<<g > 0 ? g : 1, 256, 0, s>>>(a);
    else assemble_stress_ch_kernel<2><<<g > 0 ? g : 1, 256, 0, s>>>(a);
    return cudaGetLastError();
}

// ---- implicit PDDO dynamic fracture (reference src/PDSystem/CudaAssembleKernels.cu:880-1024, physics of
//      PDDODynamicFracElement.cpp:207-306): backward-Euler inertia R = b - rho (u - u_old - v dt)/dt^2 per node,
//      Navier bond blocks P scaled by the frozen bond health (a broken bond contributes nothing; its slots are
//      written as zero), zero-length bonds skipped.  K_IJ stored per bond, the diagonal block accumulates
//      rho/dt^2 plus the sum of K_IJ. -----------------------------------------------------------------------
template <int DIM>
__global__ void __launch_bounds__(256) assemble_cached_kernel(CachedAsmArgs a) {
    constexpr int WPB = 256 / kWarp;
    constexpr int NP = DIM == 3 ? 6 : 3;  // 2D p11 pxy p22; 3D p11 p22 p33 p12 p13 p23
    using PosT = typename Vec<DIM>::T;
    const PosT *pos = static_cast<const PosT *>(a.pos);
    const int lane = threadIdx.x & 31;
    const int wib = threadIdx.x >> 5;
    for (int i = blockIdx.x * WPB + wib; i < a.n; i += gridDim.x * WPB) {
        const int rb = i * DIM;
        for (int s = a.rowptr[rb] + lane; s < a.rowptr[rb + DIM]; s += kWarp) a.kvals[s] = 0.0;
        __syncwarp();
        if (a.degenerate && a.degenerate[i]) {  // singular moment system: the rows stay zero
            if (lane < DIM) a.rhs[rb + lane] = 0.0;
            continue;
        }
        double uI[DIM];
#pragma unroll
        for (int d = 0; d < DIM; ++d) uI[d] = a.u[rb + d];
        const PosT xi = pos[i];
        double R[DIM], S[NP];
#pragma unroll
        for (int d = 0; d < DIM; ++d) R[d] = 0.0;
#pragma unroll
        for (int q = 0; q < NP; ++q) S[q] = 0.0;
        for (int t = a.off[i] + lane; t < a.off[i + 1]; t += kWarp) {
            const int j = __ldg(a.nbr + t);
            const PosT xj = pos[j];
            double r2 = (xj.x - xi.x) * (xj.x - xi.x) + (xj.y - xi.y) * (xj.y - xi.y);
            if constexpr (DIM == 3) r2 += (xj.z - xi.z) * (xj.z - xi.z);
            if (!(r2 > 0.0)) continue;
            const double h = a.bondcache ? a.bondcache[(size_t)t * a.nbcache] : 1.0;
            double P[NP];
            if (h > 0.0) {
                const double *op = a.ops + (size_t)t * a.nop;
                const double Gxx = op[a.sl[0]], Gxy = op[a.sl[1]], Gyy = op[a.sl[2]];
                if constexpr (DIM == 2) {
                    P[0] = h * (a.C11 * Gxx + a.C66 * Gyy);
                    P[1] = h * (a.C12 + a.C66) * Gxy;
                    P[2] = h * (a.C66 * Gxx + a.C11 * Gyy);
                } else {
                    const double Gxz = op[a.sl[3]], Gyz = op[a.sl[4]], Gzz = op[a.sl[5]];
                    const double cc = a.C12 + a.C66;
                    P[0] = h * (a.C11 * Gxx + a.C66 * (Gyy + Gzz));
                    P[1] = h * (a.C11 * Gyy + a.C66 * (Gxx + Gzz));
                    P[2] = h * (a.C11 * Gzz + a.C66 * (Gxx + Gyy));
                    P[3] = h * cc * Gxy;
                    P[4] = h * cc * Gxz;
                    P[5] = h * cc * Gyz;
                }
            } else {
#pragma unroll
                for (int q = 0; q < NP; ++q) P[q] = 0.0;
            }
            double Kb[DIM][DIM];
            if constexpr (DIM == 2) {
                Kb[0][0] = P[0];
                Kb[0][1] = Kb[1][0] = P[1];
                Kb[1][1] = P[2];
            } else {
                Kb[0][0] = P[0];
                Kb[1][1] = P[1];
                Kb[2][2] = P[2];
                Kb[0][1] = Kb[1][0] = P[3];
                Kb[0][2] = Kb[2][0] = P[4];
                Kb[1][2] = Kb[2][1] = P[5];
            }
            double du[DIM];
#pragma unroll
            for (int d = 0; d < DIM; ++d) du[d] = a.u[(size_t)j * DIM + d] - uI[d];
#pragma unroll
            for (int r = 0; r < DIM; ++r) {
                double rr = 0.0;
#pragma unroll
                for (int c = 0; c < DIM; ++c) rr += Kb[r][c] * du[c];
                R[r] += rr;
            }
#pragma unroll
            for (int q = 0; q < NP; ++q) S[q] += P[q];
            const int *st = a.slot + (size_t)t * DIM * DIM;
#pragma unroll
            for (int r = 0; r < DIM; ++r)
#pragma unroll
                for (int c = 0; c < DIM; ++c) a.kvals[st[r * DIM + c]] = -Kb[r][c];
        }
#pragma unroll
        for (int d = 0; d < DIM; ++d) R[d] = group_sum<kWarp>(R[d]);
#pragma unroll
        for (int q = 0; q < NP; ++q) S[q] = group_sum<kWarp>(S[q]);
        if (lane == 0) {
            const double c0 = a.rho / (a.dt * a.dt);
            double kii[DIM][DIM];
            if constexpr (DIM == 2) {
                kii[0][0] = S[0];
                kii[0][1] = kii[1][0] = S[1];
                kii[1][1] = S[2];
            } else {
                kii[0][0] = S[0];
                kii[1][1] = S[1];
                kii[2][2] = S[2];
                kii[0][1] = kii[1][0] = S[3];
                kii[0][2] = kii[2][0] = S[4];
                kii[1][2] = kii[2][1] = S[5];
            }
            const int *dg = a.diag + (size_t)i * DIM * DIM;
#pragma unroll
            for (int r = 0; r < DIM; ++r) {
                const double uo = a.uold ? a.uold[rb + r] : 0.0;
                const double v = a.nodecache ? a.nodecache[(size_t)i * a.ncache + r] : 0.0;
                kii[r][r] += c0;
                a.rhs[rb + r] = (a.b[r] - c0 * (uI[r] - uo - v * a.dt)) + R[r];
#pragma unroll
                for (int c = 0; c < DIM; ++c) a.kvals[dg[r * DIM + c]] = kii[r][c];
            }
        }
    }
}

cudaError_t launch_assemble_cached(const CachedAsmArgs &a, cudaStream_t s) {
    const int g = (a.n + 7) / 8;
    if (a.dim == 3) assemble_cached_kernel<3><<<g > 0 ? g : 1, 256, 0, s>>>(a);
    else assemble_cached_kernel<2><<<g > 0 ? g : 1, 256, 0, s>>>(a);
    return cudaGetLastError();
}

// ---- conservative Cahn-Hilliard (2 dof: c, mu) ------------------------------------------------------------
// LPN lanes per node (a family of 12..28 bonds fills a group of 8 in a pass or four), so the per-node work (row
// zeroing, reductions, the nodal free-energy terms) runs for 32/LPN nodes at once instead of one per warp
template <int LPN>
__global__ void __launch_bounds__(256) assemble_ch_kernel(ChAsmArgs a) {
    constexpr int GPW = kWarp / LPN;
    const int lane = threadIdx.x & 31;
    const int gl = lane & (LPN - 1);
    const int grp = lane / LPN;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    for (int base = warp * GPW; base < a.n; base += nwarps * GPW) {
        const int i = base + grp;
        const bool act = i < a.n;
        const int rc = 2 * i, rm = 2 * i + 1;
        if (act) {
            if (a.extra) {  // exact pattern: every other entry of the two rows is written below
                if (gl < 4) {
                    const int e = a.extra[(size_t)i * 4 + gl];
                    if (e >= 0) a.kvals[e] = 0.0;
                }
            } else {
                for (int s = a.rowptr[rc] + gl; s < a.rowptr[rm + 1]; s += LPN) a.kvals[s] = 0.0;
            }
        }
        __syncwarp();
        double c = 0.0, mu = 0.0, Vi = 0.0, Mi = 0.0;
        int b0 = 0, b1 = 0;
        if (act) {
            c = a.u[rc];
            mu = a.u[rm];
            Vi = a.vol[i];
            Mi = a.mnode[i];
            b0 = a.off[i];
            b1 = a.off[i + 1];
        }
        double rcs = 0.0, rms = 0.0, k12 = 0.0, k21 = 0.0;
        for (int t = b0 + gl; t < b1; t += LPN) {
            const int j = __ldg(a.nbr + t);
            const double g2 = a.lap[t];
            double coeff_c = 0.0, coeff_mu = 0.0;
            if (a.lrv) {  // the geometry's bond-order streams: only the mobility and u of j are gathered
                const uint8_t f = a.bfl[t];
                if (!(f & 1)) {
                    double w;
                    if ((f & 2) && Vi > 0.0) w = 0.5 * (Mi * g2 + (a.lrv[t] / Vi) * a.mnode[j]);
                    else w = Mi * g2;
                    coeff_c = -w;
                    coeff_mu = a.kappa * g2;
                }
            } else {
                const bool ghostJ = a.ghost && a.ghost[j];
                if (!ghostJ) {
                    const int r = a.rev[t];
                    double w;
                    if (r >= 0 && Vi > 0.0) w = 0.5 * (Mi * g2 + (a.vol[j] / Vi) * a.mnode[j] * a.lap[r]);
                    else w = Mi * g2;
                    coeff_c = -w;
                    coeff_mu = a.kappa * g2;
                }
            }
            rcs += coeff_c * (a.u[2 * (size_t)j + 1] - mu);  // u may be only 8-byte aligned (a caller's pointer)
            rms += coeff_mu * (a.u[2 * (size_t)j] - c);
            k12 += coeff_c;
            k21 += coeff_mu;
            const int4 sl = reinterpret_cast<const int4 *>(a.slot)[t];
            a.kvals[sl.x] = -0.0;        // (c,  c_j)
            a.kvals[sl.y] = -coeff_c;    // (c,  mu_j)
            a.kvals[sl.z] = -coeff_mu;   // (mu, c_j)
            a.kvals[sl.w] = -0.0;        // (mu, mu_j)
        }
        rcs = group_sum<LPN>(rcs);
        rms = group_sum<LPN>(rms);
        k12 = group_sum<LPN>(k12);
        k21 = group_sum<LPN>(k21);
        if (act && gl == 0) {
            const double cold = a.uold[rc];
            const double cc = ch_clamp(c);
            const double fp = log(cc / (1.0 - cc)) + a.chi * (1.0 - 2.0 * cc);
            const double fpp = 1.0 / (cc * (1.0 - cc)) - 2.0 * a.chi;
            const int4 dg = reinterpret_cast<const int4 *>(a.diag)[i];
            a.kvals[dg.x] = -(1.0 / a.dt);
            a.kvals[dg.y] = -0.0 + k12;
            a.kvals[dg.z] = fpp + k21;
            a.kvals[dg.w] = -1.0;
            a.rhs[rc] = (c - cold) / a.dt + rcs;
            a.rhs[rm] = mu - fp + rms;
        }
    }
}

__global__ void ch_bond_streams_kernel(int n, const int *off, const int *nbr, const int *rev, const double *lap,
                                       const double *vol, const char *ghost, double *lrv, uint8_t *bfl) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        for (int t = off[i]; t < off[i + 1]; ++t) {
            const int j = nbr[t], r = rev[t];
            lrv[t] = r >= 0 ? vol[j] * lap[r] : 0.0;
            bfl[t] = (uint8_t)(((ghost && ghost[j]) ? 1 : 0) | (r >= 0 ? 2 : 0));
        }
    }
}

cudaError_t launch_ch_bond_streams(int n, const int *off, const int *nbr, const int *rev, const double *lap,
                                   const double *vol, const char *ghost, double *lrv, uint8_t *bfl, cudaStream_t s) {
    const int grid = (int)((n + 255) / 256 < 148 * 16 ? (n + 255) / 256 : 148 * 16);
    ch_bond_streams_kernel<<<grid > 0 ? grid : 1, 256, 0, s>>>(n, off, nbr, rev, lap, vol, ghost, lrv, bfl);
    return cudaGetLastError();
}

cudaError_t launch_assemble_ch(const ChAsmArgs &a, cudaStream_t s) {
    constexpr int LPN = 8;
    const long long warps = ((long long)a.n + (kWarp / LPN) - 1) / (kWarp / LPN);
    const long long g = (warps + 7) / 8;
    const int grid = (int)(g < 148 * 32 ? (g > 0 ? g : 1) : 148 * 32);
    assemble_ch_kernel<LPN><<<grid, 256, 0, s>>>(a);
    return cudaGetLastError();
}

// ---- Cahn-Hilliard geometry and mobility on the device -------------------------------------------------------
template <int DIM, typename GT>
__global__ void ch_geometry_kernel(int n, const int *off, const int *nbr, const void *pos, const int *mirror,
                                   const GT *ops, int nop, int sxx, int syy, int szz, double *lap, char *ghost) {
    using PosT = typename Vec<DIM>::T;
    const PosT *p = static_cast<const PosT *>(pos);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        ghost[i] = (mirror && mirror[i] > 0) ? 1 : 0;
        const PosT xi = p[i];
        double qi = xi.x * xi.x + xi.y * xi.y;
        if constexpr (DIM == 3) qi += xi.z * xi.z;
        double lapq = 0.0;
        const int b0 = off[i], b1 = off[i + 1];
        for (int t = b0; t < b1; ++t) {
            const GT *g = ops + (size_t)t * nop;
            double w = (double)g[sxx] + (double)g[syy];
            if constexpr (DIM == 3) w += (double)g[szz];
            lap[t] = w;
            const int j = nbr[t];
            if (!(mirror && mirror[j] > 0)) {
                const PosT xj = p[j];
                double qj = xj.x * xj.x + xj.y * xj.y;
                if constexpr (DIM == 3) qj += xj.z * xj.z;
                lapq += w * (qj - qi);
            }
        }
        const double lam = (lapq > 1.0e-12) ? (2.0 * DIM / lapq) : 1.0;
        for (int t = b0; t < b1; ++t)
            if (!(mirror && mirror[nbr[t]] > 0)) lap[t] *= lam;
    }
}

cudaError_t launch_ch_geometry(int n, int dim, const int *off, const int *nbr, const void *pos, const int *mirror,
                               const void *ops, bool mixed, int nop, int sxx, int syy, int szz, double *lap,
                               char *ghost, cudaStream_t s) {
    const int grid = (int)((n + 255) / 256 < 148 * 16 ? (n + 255) / 256 : 148 * 16);
    const int g = grid > 0 ? grid : 1;
    if (dim == 3) {
        if (mixed) ch_geometry_kernel<3, float><<<g, 256, 0, s>>>(n, off, nbr, pos, mirror, (const float *)ops, nop, sxx, syy, szz, lap, ghost);
        else ch_geometry_kernel<3, double><<<g, 256, 0, s>>>(n, off, nbr, pos, mirror, (const double *)ops, nop, sxx, syy, szz, lap, ghost);
    } else {
        if (mixed) ch_geometry_kernel<2, float><<<g, 256, 0, s>>>(n, off, nbr, pos, mirror, (const float *)ops, nop, sxx, syy, szz, lap, ghost);
        else ch_geometry_kernel<2, double><<<g, 256, 0, s>>>(n, off, nbr, pos, mirror, (const double *)ops, nop, sxx, syy, szz, lap, ghost);
    }
    return cudaGetLastError();
}

__global__ void ch_mobility_kernel(int n, double M0, const double *u, double *mnode) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const double c = fmax(1.0e-8, fmin(1.0 - 1.0e-8, u[2 * (size_t)i]));
        mnode[i] = M0 * c * (1.0 - c);
    }
}

cudaError_t launch_ch_mobility(int n, double M0, const double *u, double *mnode, cudaStream_t s) {
    const int grid = (int)((n + 255) / 256 < 148 * 16 ? (n + 255) / 256 : 148 * 16);
    ch_mobility_kernel<<<grid > 0 ? grid : 1, 256, 0, s>>>(n, M0, u, mnode);
    return cudaGetLastError();
}

}  // namespace pxb
