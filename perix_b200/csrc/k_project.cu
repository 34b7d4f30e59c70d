// Output projections of the explicit fracture state (reference ExplicitPDDOFracElement::computeNodalProjection,
// src/ElmtSystem/ExplicitPDDOFracElement.cpp:324-405), on the device so that output intervals need no copy of
// the full state: per node the damage 1 - (intact bonds)/(bonds), the displacement gradient from the FP64
// first-derivative operators over the whole family (broken bonds included, as in the reference), the small
// strain, the Cauchy stress with the Navier constants (lambda = C12, mu = C66; in 2D sigma_zz = lambda tr(eps)
// under plane strain, 0 under plane stress) and the von Mises stress.  One warp per node.
#include "k_kernels.h"
#include "pxb_common.cuh"

namespace pxb {

template <int DIM>
__global__ void __launch_bounds__(256) epf_project_kernel(ProjectArgs a) {
    constexpr int WPB = 256 / kWarp;
    const int lane = threadIdx.x & 31;
    const int wib = threadIdx.x >> 5;
    for (int i = blockIdx.x * WPB + wib; i < a.n; i += gridDim.x * WPB) {
        const int b0 = a.off[i], b1 = a.off[i + 1];
        double live = 0.0, gu[DIM][DIM];
#pragma unroll
        for (int r = 0; r < DIM; ++r)
#pragma unroll
            for (int c = 0; c < DIM; ++c) gu[r][c] = 0.0;
        double ui[DIM];
#pragma unroll
        for (int d = 0; d < DIM; ++d) ui[d] = a.u[(size_t)i * DIM + d];
        for (int t = b0 + lane; t < b1; t += kWarp) {
            const int j = __ldg(a.nbr + t);
            live += a.health[t] ? 1.0 : 0.0;
            const double *op = a.ops + (size_t)t * a.nop;
            double G[DIM];
#pragma unroll
            for (int c = 0; c < DIM; ++c) G[c] = op[a.sl[c]];
#pragma unroll
            for (int r = 0; r < DIM; ++r) {
                const double du = a.u[(size_t)j * DIM + r] - ui[r];
#pragma unroll
                for (int c = 0; c < DIM; ++c) gu[r][c] += du * G[c];
            }
        }
        live = group_sum<kWarp>(live);
#pragma unroll
        for (int r = 0; r < DIM; ++r)
#pragma unroll
            for (int c = 0; c < DIM; ++c) gu[r][c] = group_sum<kWarp>(gu[r][c]);
        if (lane != 0) continue;
        const int nb = b1 - b0;
        if (a.damage) a.damage[i] = nb <= 0 ? 0.0 : 1.0 - live / (double)nb;
        // eps = sym(grad u) as {xx, yy, zz, xy, xz, yz}
        double eps[6] = {gu[0][0], gu[1][1], 0.0, 0.5 * (gu[0][1] + gu[1][0]), 0.0, 0.0};
        if constexpr (DIM == 3) {
            eps[2] = gu[2][2];
            eps[4] = 0.5 * (gu[0][2] + gu[2][0]);
            eps[5] = 0.5 * (gu[1][2] + gu[2][1]);
        }
        const double lam = a.C12, mu = a.C66;
        const double tr = eps[0] + eps[1] + eps[2];
        double sig[6];
        sig[0] = lam * tr + 2.0 * mu * eps[0];
        sig[1] = lam * tr + 2.0 * mu * eps[1];
        sig[2] = DIM == 3 ? lam * tr + 2.0 * mu * eps[2] : (a.plane_strain ? lam * tr : 0.0);
        sig[3] = 2.0 * mu * eps[3];
        sig[4] = 2.0 * mu * eps[4];
        sig[5] = 2.0 * mu * eps[5];
        if (a.von_mises) {
            const double sm = (sig[0] + sig[1] + sig[2]) / 3.0;
            const double p = sig[0] - sm, q = sig[1] - sm, r = sig[2] - sm;
            a.von_mises[i] = sqrt(1.5 * (p * p + q * q + r * r + 2.0 * (sig[3] * sig[3] + sig[4] * sig[4] + sig[5] * sig[5])));
        }
        // 3x3 row-major tensors
        const int map[9] = {0, 3, 4, 3, 1, 5, 4, 5, 2};
        if (a.stress)
            for (int k = 0; k < 9; ++k) a.stress[(size_t)i * 9 + k] = sig[map[k]];
        if (a.strain)
            for (int k = 0; k < 9; ++k) a.strain[(size_t)i * 9 + k] = eps[map[k]];
    }
}

cudaError_t launch_epf_project(const ProjectArgs &a, cudaStream_t s) {
    const int g = (a.n + 7) / 8;
    if (a.dim == 3) epf_project_kernel<3><<<g > 0 ? g : 1, 256, 0, s>>>(a);
    else epf_project_kernel<2><<<g > 0 ? g : 1, 256, 0, s>>>(a);
    return cudaGetLastError();
}

}  // namespace pxb
