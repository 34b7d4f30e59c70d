// Device linear algebra for the implicit Cahn-Hilliard run (ch_solver.cpp) and the Cahn-Hilliard-specific pieces
// of its Newton and adjoint steps.
//
// Generic: CSR SpMV y = A x (warp per row), transposed SpMV y = A^T x (warp per row, scatter with FP64 atomics),
// deterministic dot products (fixed-order two-stage reduction), vector updates, and a 2x2 block-Jacobi
// preconditioner built from the diagonal blocks of a 2-dof CSR matrix.
//
// Cahn-Hilliard (rows 2i = c, 2i+1 = mu; the conservative element of CahnHilliardElement.cpp:178-292):
//   * ghost rows: the reference's zero-Neumann row replacement (NeumannBC.cpp:127-150): row g becomes
//     s (dU_g - dU_b) = s (U_b - U_g), s = |K_gg| (1 when zero);
//   * the mobility term the Picard iteration leaves out of K: dF/dU = -K + J_M with
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

__global__ void __launch_bounds__(256) spmv_kernel(int rows, const int *rowptr, const int *cols, const double *val,
                                                    const double *x, double *y) {
    const int lane = threadIdx.x & 31;
    for (int r = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; r < rows; r += (gridDim.x * blockDim.x) >> 5) {
        double s = 0.0;
        for (int k = rowptr[r] + lane; k < rowptr[r + 1]; k += kWarp) s += val[k] * x[cols[k]];
        s = group_sum<kWarp>(s);
        if (lane == 0) y[r] = s;
    }
}

__global__ void __launch_bounds__(256) spmv_t_kernel(int rows, const int *rowptr, const int *cols, const double *val,
                                                      const double *x, double *y) {
    const int lane = threadIdx.x & 31;
    for (int r = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; r < rows; r += (gridDim.x * blockDim.x) >> 5) {
        const double xr = x[r];
        if (xr == 0.0) continue;
        for (int k = rowptr[r] + lane; k < rowptr[r + 1]; k += kWarp) atomicAdd(y + cols[k], val[k] * xr);
    }
}

cudaError_t launch_spmv(int rows, const int *rowptr, const int *cols, const double *val, const double *x, double *y,
                        bool transpose, cudaStream_t s) {
    const int g = (rows + 7) / 8;
    const int grid = g < 148 * 16 ? (g > 0 ? g : 1) : 148 * 16;
    if (transpose) {
        cudaError_t e = cudaMemsetAsync(y, 0, sizeof(double) * (size_t)rows, s);
        if (e != cudaSuccess) return e;
        spmv_t_kernel<<<grid, 256, 0, s>>>(rows, rowptr, cols, val, x, y);
    } else {
        spmv_kernel<<<grid, 256, 0, s>>>(rows, rowptr, cols, val, x, y);
    }
    return cudaGetLastError();
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

// p = r + beta (p - omega v)  (BiCGStab direction update)
__global__ void bicg_p_kernel(long long n, const double *r, double beta, double omega, const double *v, double *p) {
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x)
        p[k] = r[k] + beta * (p[k] - omega * v[k]);
}

cudaError_t launch_bicg_p(long long n, const double *r, double beta, double omega, const double *v, double *p,
                          cudaStream_t s) {
    bicg_p_kernel<<<148 * 8, 256, 0, s>>>(n, r, beta, omega, v, p);
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

__global__ void block_apply_kernel(int n, const double *binv, const double *x, double *y) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const double *b = binv + (size_t)i * 4;
        const double x0 = x[2 * (size_t)i], x1 = x[2 * (size_t)i + 1];
        y[2 * (size_t)i] = b[0] * x0 + b[1] * x1;
        y[2 * (size_t)i + 1] = b[2] * x0 + b[3] * x1;
    }
}

cudaError_t launch_block_apply(int n, const double *binv, const double *x, double *y, cudaStream_t s) {
    block_apply_kernel<<<(n + 255) / 256 > 0 ? (n + 255) / 256 : 1, 256, 0, s>>>(n, binv, x, y);
    return cudaGetLastError();
}

// ---- Cahn-Hilliard pieces ------------------------------------------------------------------------------------
__device__ __forceinline__ int slot_of(const int *cols, int lo, int hi, int target) {
    int l = lo, h = hi - 1;
    while (l <= h) {
        const int mid = l + ((h - l) >> 1);
        const int c = cols[mid];
        if (c == target) return mid;
        if (c < target) l = mid + 1; else h = mid - 1;
    }
    return -1;
}

// Neumann row replacement on the ghost rows of (K, rhs) at state U; rows must hold the mirror column
__global__ void ch_ghost_rows_kernel(int n, const int *mirror, const int *rowptr, const int *cols, const double *u,
                                     double *kv, double *rhs) {
    for (int g = blockIdx.x * blockDim.x + threadIdx.x; g < n; g += gridDim.x * blockDim.x) {
        const int b = mirror[g] - 1;
        if (b < 0) continue;
        for (int a = 0; a < 2; ++a) {
            const int row = 2 * g + a;
            const int lo = rowptr[row], hi = rowptr[row + 1];
            const int sd = slot_of(cols, lo, hi, row), sb = slot_of(cols, lo, hi, 2 * b + a);
            double sc = sd >= 0 ? fabs(kv[sd]) : 0.0;
            if (!(sc > 0.0)) sc = 1.0;
            for (int k = lo; k < hi; ++k) kv[k] = 0.0;
            if (sd >= 0) kv[sd] = sc;
            if (sb >= 0) kv[sb] = -sc;
            rhs[row] = sc * (u[2 * (size_t)b + a] - u[2 * (size_t)g + a]);
        }
    }
}

cudaError_t launch_ch_ghost_rows(int n, const int *mirror, const int *rowptr, const int *cols, const double *u,
                                 double *kv, double *rhs, cudaStream_t s) {
    ch_ghost_rows_kernel<<<(n + 255) / 256 > 0 ? (n + 255) / 256 : 1, 256, 0, s>>>(n, mirror, rowptr, cols, u, kv, rhs);
    return cudaGetLastError();
}

__device__ __forceinline__ double mob_prime(double c, double M0) {
    return (c > 1.0e-8 && c < 1.0 - 1.0e-8) ? M0 * (1.0 - 2.0 * c) : 0.0;
}

// y[c rows] -= J_M^T x  (y already holds K^T x; the adjoint operator is K^T - J_M^T).  Bulk rows i only.
// J_M^T x at column c_i: M'(c_i) (A_i x_{c_i} + sum over bonds t = i -> j with i -> j paired-reverse... ) is
// gathered per column node k from its own family: the row i of a bond i -> k is reached through the reverse bond.
__global__ void __launch_bounds__(256) ch_mob_adj_kernel(ChAdjArgs a) {
    constexpr int WPB = 256 / kWarp;
    const int lane = threadIdx.x & 31;
    const int wib = threadIdx.x >> 5;
    for (int k = blockIdx.x * WPB + wib; k < a.n; k += gridDim.x * WPB) {
        // (1) diagonal term of row k (if k is bulk): A_k = sum_t -(paired ? g2/2 : g2) (mu_j - mu_k)
        // (2) terms of rows i (bulk) whose bond i -> k is paired and k non-ghost: -(1/2) (V_k / V_i) g2_rev (mu_k - mu_i)
        //     reached from k's family: t = k -> i, its reverse r = rev[t] is the bond i -> k, g2_rev(i->k) = lap[t]
        const bool bulk_k = a.mirror == nullptr || a.mirror[k] == 0;
        const bool ghost_k = a.ghost && a.ghost[k];
        const double mu_k = a.u[2 * (size_t)k + 1], Vk = a.vol[k];
        double acc = 0.0;
        for (int t = a.off[k] + lane; t < a.off[k + 1]; t += kWarp) {
            const int j = __ldg(a.nbr + t);
            const double mu_j = a.u[2 * (size_t)j + 1];
            const int r = a.rev[t];
            if (bulk_k && !(a.ghost && a.ghost[j])) {
                const bool paired = r >= 0 && Vk > 0.0;
                acc += a.x[2 * (size_t)k] * (-(paired ? 0.5 : 1.0) * a.lap[t] * (mu_j - mu_k));
            }
            // row j (as "i") with its bond j -> k = r: needs j bulk, k non-ghost, that bond paired (rev(r) = t >= 0)
            if (r >= 0 && !ghost_k && (a.mirror == nullptr || a.mirror[j] == 0)) {
                const double Vj = a.vol[j];
                if (Vj > 0.0) acc += a.x[2 * (size_t)j] * (-0.5 * (Vk / Vj) * a.lap[t] * (mu_k - mu_j));
            }
        }
        acc = group_sum<kWarp>(acc);
        if (lane == 0) a.y[2 * (size_t)k] -= mob_prime(a.u[2 * (size_t)k], a.M0) * acc;
    }
}

cudaError_t launch_ch_mob_adj(const ChAdjArgs &a, cudaStream_t s) {
    const int g = (a.n + 7) / 8;
    ch_mob_adj_kernel<<<g > 0 ? g : 1, 256, 0, s>>>(a);
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
