// Device linear algebra for the implicit Cahn-Hilliard run (ch_solver.cpp) and the Cahn-Hilliard-specific pieces
// of its Newton and adjoint steps.
//
// Generic: deterministic dot products (fixed-order two-stage reduction), vector updates, and the 2x2 block-Jacobi
// inverse built from the diagonal blocks of a 2-dof CSR matrix (the BiCGStab itself is in k_bicg.cu).
//
// Cahn-Hilliard (rows 2i = c, 2i+1 = mu; the conservative element of CahnHilliardElement.cpp:178-292):
//   * ghost rows: the reference's zero-Neumann row replacement (NeumannBC.cpp:127-150): row g becomes
//     s (dU_g - dU_b) = s (U_b - U_g), s = |K_gg| (1 when zero);
//   * the mobility term the Picard iteration leaves out of K (folded into K for the adjoint): dF/dU = -K + J_M with
//       J_M[c_i, c_i] = M'(c_i) sum_t -(paired ? g2_t / 2 : g2_t) (mu_j - mu_i),
//       J_M[c_i, c_j] = M'(c_j) (-1/2) (V_j / V_i) g2_rev(t) (mu_j - mu_i)  (paired bonds),
//     over bonds t = i -> j to non-ghost j of bulk rows i, M(c) = M0 cc (1 - cc), cc = clamp(c, 1e-8, 1 - 1e-8);
//   * dF_mu,i / dkappa = sum_t g2_t (c_j - c_i) over bonds to non-ghost j;
//   * the total free energy E = sum over bulk i of V_i (f(c_i) + kappa/2 |grad c_i|^2), f(c) = c ln c +
//     (1 - c) ln(1 - c) + chi c (1 - c), grad c_i = sum_t G1_t (c_j - c_i) (the PDDO first derivatives), and dE/dU.
#include "k_kernels.h"
#include "pxb_common.cuh"

namespace pxb {

namespace {
constexpr int kRedBlocks = 592;  // 4 x 148: partial sums of a dot product
}

__global__ void __launch_bounds__(256) dot_partial_kernel(long long n, const double *a, const double *b, double *part) {
    __shared__ double sh[8];
    double s = 0.0;
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x)
        s += a[k] * b[k];
    s = group_sum<kWarp>(s);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < 8; ++w) t += sh[w];
        part[blockIdx.x] = t;
    }
}

__global__ void dot_final_kernel(int nparts, const double *part, double *out) {
    __shared__ double sh[kWarp];
    double s = 0.0;
    for (int k = threadIdx.x; k < nparts; k += kWarp) s += part[k];
    sh[threadIdx.x] = s;
    __syncwarp();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < kWarp; ++w) t += sh[w];
        *out = t;
    }
}

int dot_scratch_doubles() { return kRedBlocks + 8; }

cudaError_t launch_dot(long long n, const double *a, const double *b, double *scratch, double *out, cudaStream_t s) {
    dot_partial_kernel<<<kRedBlocks, 256, 0, s>>>(n, a, b, scratch);
    dot_final_kernel<<<1, kWarp, 0, s>>>(kRedBlocks, scratch, out);
    return cudaGetLastError();
}

// y = alpha x + beta y  (beta == 0: y = alpha x)
__global__ void axpby_kernel(long long n, double alpha, const double *x, double beta, double *y) {
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x)
        y[k] = beta == 0.0 ? alpha * x[k] : alpha * x[k] + beta * y[k];
}

cudaError_t launch_axpby(long long n, double alpha, const double *x, double beta, double *y, cudaStream_t s) {
    axpby_kernel<<<148 * 8, 256, 0, s>>>(n, alpha, x, beta, y);
    return cudaGetLastError();
}

// inverse 2x2 diagonal blocks of a 2-dof CSR matrix (diag = slot map [n][4]); transpose stores the inverse of the
// transposed block.  A singular block falls back to the identity.
__global__ void block_inv_kernel(int n, const int *diag, const double *val, bool transpose, double *binv) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int *d = diag + (size_t)i * 4;
        double a = val[d[0]], b = val[d[1]], c = val[d[2]], e = val[d[3]];
        if (transpose) {
            const double t = b;
            b = c;
            c = t;
        }
        const double det = a * e - b * c;
        double *o = binv + (size_t)i * 4;
        if (det != 0.0 && isfinite(det)) {
            o[0] = e / det;
            o[1] = -b / det;
            o[2] = -c / det;
            o[3] = a / det;
        } else {
            o[0] = 1.0;
            o[1] = 0.0;
            o[2] = 0.0;
            o[3] = 1.0;
        }
    }
}

cudaError_t launch_block_inv(int n, const int *diag, const double *val, bool transpose, double *binv, cudaStream_t s) {
    block_inv_kernel<<<(n + 255) / 256 > 0 ? (n + 255) / 256 : 1, 256, 0, s>>>(n, diag, val, transpose, binv);
    return cudaGetLastError();
}

// ---- Cahn-Hilliard pieces ------------------------------------------------------------------------------------
// Neumann row replacement on the ghost rows of (K, rhs) at state U; rows must hold the mirror column
// warp per node; the lanes scan each ghost row for its diagonal and mirror columns and rewrite it in one pass
__global__ void __launch_bounds__(256) ch_ghost_rows_kernel(int n, const int *mirror, const int *rowptr,
                                                             const int *cols, const double *u, double *kv,
                                                             double *rhs) {
    constexpr int WPB = 256 / kWarp;
    const int lane = threadIdx.x & 31;
    for (int g = blockIdx.x * WPB + (threadIdx.x >> 5); g < n; g += gridDim.x * WPB) {
        const int b = mirror[g] - 1;
        if (b < 0) continue;
        for (int a = 0; a < 2; ++a) {
            const int row = 2 * g + a, mcol = 2 * b + a;
            const int lo = rowptr[row], hi = rowptr[row + 1];
            int sd = -1, sb = -1;
            double d = 0.0;
            for (int k = lo + lane; k < hi; k += kWarp) {
                const int col = cols[k];
                if (col == row) {
                    sd = k;
                    d = kv[k];
                }
                if (col == mcol) sb = k;
            }
            sd = __reduce_max_sync(kFull, sd);
            sb = __reduce_max_sync(kFull, sb);
            d = group_sum<kWarp>(d);  // one lane at most holds the diagonal
            double sc = sd >= 0 ? fabs(d) : 0.0;
            if (!(sc > 0.0)) sc = 1.0;
            for (int k = lo + lane; k < hi; k += kWarp) kv[k] = k == sd ? sc : (k == sb ? -sc : 0.0);
            if (lane == 0) rhs[row] = sc * (u[2 * (size_t)b + a] - u[2 * (size_t)g + a]);
        }
    }
}

cudaError_t launch_ch_ghost_rows(int n, const int *mirror, const int *rowptr, const int *cols, const double *u,
                                 double *kv, double *rhs, cudaStream_t s) {
    const int g = (n + 7) / 8;
    ch_ghost_rows_kernel<<<g < 148 * 16 ? (g > 0 ? g : 1) : 148 * 16, 256, 0, s>>>(n, mirror, rowptr, cols, u, kv,
                                                                                     rhs);
    return cudaGetLastError();
}

__device__ __forceinline__ double mob_prime(double c, double M0) {
    return (c > 1.0e-8 && c < 1.0 - 1.0e-8) ? M0 * (1.0 - 2.0 * c) : 0.0;
}

// K' = K - J_M on bulk rows i: for bonds t = i -> j to non-ghost j,
//   K'[c_i, c_i] -= M'(c_i) sum_t -(paired ? g2_t / 2 : g2_t) (mu_j - mu_i),
//   K'[c_i, c_j] -= M'(c_j) (-1/2) (V_j / V_i) g2_rev(t) (mu_j - mu_i)   (paired bonds),
// paired = the bond has a reverse and V_i > 0.  Each bond slot belongs to one bond, so the updates do not collide.
__global__ void __launch_bounds__(256) ch_fold_mobility_kernel(ChAdjArgs a, const int *slot, const int *diag,
                                                               double *kv) {
    constexpr int WPB = 256 / kWarp;
    const int lane = threadIdx.x & 31;
    const int wib = threadIdx.x >> 5;
    for (int i = blockIdx.x * WPB + wib; i < a.n; i += gridDim.x * WPB) {
        if (a.mirror && a.mirror[i] != 0) continue;
        const double mu_i = a.u[2 * (size_t)i + 1], Vi = a.vol[i];
        double acc = 0.0;
        for (int t = a.off[i] + lane; t < a.off[i + 1]; t += kWarp) {
            const int j = __ldg(a.nbr + t);
            if (a.ghost && a.ghost[j]) continue;
            const double dmu = a.u[2 * (size_t)j + 1] - mu_i;
            const int r = a.rev[t];
            const bool paired = r >= 0 && Vi > 0.0;
            acc += -(paired ? 0.5 : 1.0) * a.lap[t] * dmu;
            if (paired)
                kv[slot[4 * (size_t)t]] -= mob_prime(a.u[2 * (size_t)j], a.M0) * (-0.5 * (a.vol[j] / Vi) * a.lap[r] * dmu);
        }
        acc = group_sum<kWarp>(acc);
        if (lane == 0) kv[diag[4 * (size_t)i]] -= mob_prime(a.u[2 * (size_t)i], a.M0) * acc;
    }
}

cudaError_t launch_ch_fold_mobility(const ChAdjArgs &a, const int *slot, const int *diag, double *kv, cudaStream_t s) {
    const int g = (a.n + 7) / 8;
    ch_fold_mobility_kernel<<<g > 0 ? g : 1, 256, 0, s>>>(a, slot, diag, kv);
    return cudaGetLastError();
}

// out[i] = x_{mu_i} * sum_t g2_t (c_j - c_i) over bonds to non-ghost j, bulk rows i (summed by launch_dot)
__global__ void __launch_bounds__(256) ch_dkappa_kernel(ChAdjArgs a) {
    constexpr int WPB = 256 / kWarp;
    const int lane = threadIdx.x & 31;
    const int wib = threadIdx.x >> 5;
    for (int i = blockIdx.x * WPB + wib; i < a.n; i += gridDim.x * WPB) {
        const bool bulk = a.mirror == nullptr || a.mirror[i] == 0;
        const double ci = a.u[2 * (size_t)i];
        double s = 0.0;
        if (bulk)
            for (int t = a.off[i] + lane; t < a.off[i + 1]; t += kWarp) {
                const int j = __ldg(a.nbr + t);
                if (!(a.ghost && a.ghost[j])) s += a.lap[t] * (a.u[2 * (size_t)j] - ci);
            }
        s = group_sum<kWarp>(s);
        if (lane == 0) a.y[i] = bulk ? a.x[2 * (size_t)i + 1] * s : 0.0;
    }
}

cudaError_t launch_ch_dkappa(const ChAdjArgs &a, cudaStream_t s) {
    const int g = (a.n + 7) / 8;
    ch_dkappa_kernel<<<g > 0 ? g : 1, 256, 0, s>>>(a);
    return cudaGetLastError();
}

// per-node energy density times volume (bulk nodes; 0 elsewhere) and the gradient-energy cotangent
// ybar_i = kappa V_i grad c_i (for the transposed first-derivative apply); e_out[i], gbar[2*i], gbar[2*i+1]
__global__ void __launch_bounds__(256) ch_energy_kernel(ChEnergyArgs a) {
    constexpr int WPB = 256 / kWarp;
    const int lane = threadIdx.x & 31;
    const int wib = threadIdx.x >> 5;
    for (int i = blockIdx.x * WPB + wib; i < a.n; i += gridDim.x * WPB) {
        const bool bulk = a.mirror == nullptr || a.mirror[i] == 0;
        const double ci = a.u[2 * (size_t)i];
        double gx = 0.0, gy = 0.0;
        for (int t = a.off[i] + lane; t < a.off[i + 1]; t += kWarp) {
            const int j = __ldg(a.nbr + t);
            const double dc = a.u[2 * (size_t)j] - ci;
            gx += a.ops[(size_t)t * a.nop + a.sx] * dc;
            gy += a.ops[(size_t)t * a.nop + a.sy] * dc;
        }
        gx = group_sum<kWarp>(gx);
        gy = group_sum<kWarp>(gy);
        if (lane == 0) {
            const double V = a.vol[i];
            if (bulk) {
                const double c = fmin(fmax(ci, 1.0e-300), 1.0 - 1.0e-16);
                const double f = c * log(c) + (1.0 - c) * log(1.0 - c) + a.chi * c * (1.0 - c);
                a.e_out[i] = V * (f + 0.5 * a.kappa * (gx * gx + gy * gy));
                a.grad_e[i] = 0.5 * V * (gx * gx + gy * gy);  // dE/dkappa density
                if (a.gbar) {
                    a.gbar[2 * (size_t)i] = a.kappa * V * gx;
                    a.gbar[2 * (size_t)i + 1] = a.kappa * V * gy;
                }
                if (a.fprime) a.fprime[i] = V * (log(c / (1.0 - c)) + a.chi * (1.0 - 2.0 * c));
            } else {
                a.e_out[i] = 0.0;
                a.grad_e[i] = 0.0;
                if (a.gbar) a.gbar[2 * (size_t)i] = a.gbar[2 * (size_t)i + 1] = 0.0;
                if (a.fprime) a.fprime[i] = 0.0;
            }
        }
    }
}

cudaError_t launch_ch_energy(const ChEnergyArgs &a, cudaStream_t s) {
    const int g = (a.n + 7) / 8;
    ch_energy_kernel<<<g > 0 ? g : 1, 256, 0, s>>>(a);
    return cudaGetLastError();
}

// dE/dU: c rows = fprime_i (bulk) + (transposed first-derivative apply of gbar)_i, mu rows 0.
// The transposed apply: for bond t = i -> j: d(grad c_i)/dc_j = G1_t, d/dc_i = -G1_t.
__global__ void __launch_bounds__(256) ch_energy_grad_kernel(ChEnergyArgs a, double *dedu) {
    constexpr int WPB = 256 / kWarp;
    const int lane = threadIdx.x & 31;
    const int wib = threadIdx.x >> 5;
    for (int i = blockIdx.x * WPB + wib; i < a.n; i += gridDim.x * WPB) {
        double s = 0.0;
        for (int t = a.off[i] + lane; t < a.off[i + 1]; t += kWarp) {
            s -= a.ops[(size_t)t * a.nop + a.sx] * a.gbar[2 * (size_t)i] +
                 a.ops[(size_t)t * a.nop + a.sy] * a.gbar[2 * (size_t)i + 1];
            // the reverse contribution (row j of bond j -> i) is gathered through rev
            const int r = a.rev[t];
            if (r >= 0) {
                const int j = __ldg(a.nbr + t);
                s += a.ops[(size_t)r * a.nop + a.sx] * a.gbar[2 * (size_t)j] +
                     a.ops[(size_t)r * a.nop + a.sy] * a.gbar[2 * (size_t)j + 1];
            }
        }
        s = group_sum<kWarp>(s);
        if (lane == 0) {
            dedu[2 * (size_t)i] = a.fprime[i] + s;
            dedu[2 * (size_t)i + 1] = 0.0;
        }
    }
}

cudaError_t launch_ch_energy_grad(const ChEnergyArgs &a, double *dedu, cudaStream_t s) {
    const int g = (a.n + 7) / 8;
    ch_energy_grad_kernel<<<g > 0 ? g : 1, 256, 0, s>>>(a, dedu);
    return cudaGetLastError();
}

// cotangent of the previous state: g[c_i] = -lam[c_i]/dt on bulk rows (the c_old term of F_c), 0 elsewhere
__global__ void ch_prev_cot_kernel(int n, const int *mirror, const double *lam, double dt, double *g) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const bool bulk = mirror == nullptr || mirror[i] == 0;
        g[2 * (size_t)i] = bulk ? -lam[2 * (size_t)i] / dt : 0.0;
        g[2 * (size_t)i + 1] = 0.0;
    }
}

cudaError_t launch_ch_prev_cot(int n, const int *mirror, const double *lam, double dt, double *g, cudaStream_t s) {
    ch_prev_cot_kernel<<<(n + 255) / 256 > 0 ? (n + 255) / 256 : 1, 256, 0, s>>>(n, mirror, lam, dt, g);
    return cudaGetLastError();
}

}  // namespace pxb
