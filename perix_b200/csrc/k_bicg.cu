// Device-resident BiCGStab for the 2-dof systems of the implicit Cahn-Hilliard run (ch_solver.cpp).
//
// Right-preconditioned BiCGStab (van der Vorst 1992) with the 2x2 block-Jacobi inverse M (rows 2i, 2i+1 of a node),
// run as ONE cooperative persistent kernel per solve: every block takes part in every phase and the phases are
// separated by grid barriers, so the matrix (61 MB of values at 256^2) and the work vectors stay in L2 across the
// iterations and no scalar goes back to the host.  Each dot product is a per-block partial sum followed by a barrier,
// after which every block adds the partials in the same fixed order, so all blocks take the same decisions and the
// result is deterministic.  The partial sums alternate between two buffers, so a block that runs ahead into the next
// reduction never overwrites partials another block is still reading.
//
// The iteration keeps rh = M r and vh = M v per node, so both preconditioned vectors are formed where the products
// gather them (ph_j = rh_j + beta (ph_j - omega vh_j), sh_j = rh_j - alpha vh_j) and an iteration needs three
// barriers (x0 = 0, r = r0 = b, rh = M b, ph = vh = 0, rho = alpha = omega = 1, rho1 = r0.r):
//   A  ph' = rh + beta (ph - omega vh),  v = A ph',  vh' = M v,  r0.v         | barrier   alpha = rho1 / r0.v
//   B  s = r - alpha v,  sh = rh - alpha vh',  t = A sh,  t.t, t.s, s.s        | barrier   omega = t.s / t.t
//      |s| <= tol |b|: x += alpha ph', done
//   C  x += alpha ph' + omega sh,  r = s - omega t,  rh = M r,  r.r, r0.r     | barrier   |r| <= tol |b|: done
//      rho = rho1, rho1 = r0.r, beta = (rho1 / rho)(alpha / omega)
// ph and vh are double-buffered: phase A reads one copy while it writes the other.  The gathered and the stored
// values come from one helper with explicit rounding, so both are bitwise the same.
// The matrix must consist of dense 2x2 node blocks (rows 2i and 2i+1 share one column list of pairs (2j, 2j+1), as
// every pattern the reference builds does, SparseMatrix.cpp:73-185).  The product reads it through a block view: bptr
// (node -> first block) and bcol (block -> column node), with the CSR values of node i's two rows at 4 bptr[i] and
// 4 bptr[i] + 2 nblk_i.  Adjoint solves run the same kernel on an explicit transpose (block_transpose below and a
// value gather).
//
// The grid barrier waits are bounded: a block that waits longer than kSpinLimit polls sets the abort word and
// returns, and every other block leaves at its next barrier; the host reports the timeout.  The cooperative launch
// makes every block resident at once, so the waits end in normal operation.
#include <vector>

#include "k_kernels.h"
#include "pxb_common.cuh"

namespace pxb {

namespace {

constexpr int kThreads = 256;
constexpr int kBlocksPerSM = 3;  // 80 registers a thread
constexpr int kWarps = kThreads / kWarp;
constexpr int kMaxGrid = 512;  // most blocks of the solve kernel
static_assert(kMaxGrid <= kBicgParts && kMaxGrid % kWarp == 0, "partial sum slots");
constexpr int kSpmvLanes = 8;  // lanes per node (its two rows)
constexpr int kUnroll = 2;     // blocks per lane and pass
constexpr unsigned kSpinLimit = 1u << 22;  // barrier polls (a few seconds at most)

// Vector loads are ordinary (L1-cached) loads: within a phase no vector is both written and read by different
// threads, and the fences of the grid barrier order every write of one phase before the reads of the next.
__device__ __forceinline__ double2 ld2(const double *p, int i) { return reinterpret_cast<const double2 *>(p)[i]; }
__device__ __forceinline__ void st2(double *p, int i, double a, double b) {
    reinterpret_cast<double2 *>(p)[i] = make_double2(a, b);
}
__device__ __forceinline__ void block2(const double *binv, int i, double x0, double x1, double &y0, double &y1) {
    const double2 b0 = __ldg(reinterpret_cast<const double2 *>(binv) + 2 * i);
    const double2 b1 = __ldg(reinterpret_cast<const double2 *>(binv) + 2 * i + 1);
    y0 = b0.x * x0 + b0.y * x1;
    y1 = b1.x * x0 + b1.y * x1;
}

// Grid barrier on a monotonic arrival counter: barrier number e (1, 2, ...) ends when e * gridDim.x blocks have
// arrived.  Returns false when the wait gave up or another block aborted.
__device__ bool grid_sync(BicgScalars *sc, unsigned int &epoch) {
    __shared__ int ok;
    __syncthreads();
    ++epoch;
    if (threadIdx.x == 0) {
        const unsigned int target = epoch * gridDim.x;
        volatile unsigned int *count = &sc->bar_count;
        volatile int *abort = &sc->abort;
        __threadfence();
        atomicAdd(&sc->bar_count, 1u);
        int good = 1;
        unsigned int polls = 0;
        while ((int)(*count - target) < 0) {
            if (*abort || ++polls > kSpinLimit) {
                *abort = 1;
                good = 0;
                break;
            }
            __nanosleep(32);
        }
        __threadfence();
        ok = good;
    }
    __syncthreads();
    return ok != 0;
}

// Grid totals of NV per-thread values: block sums into part, a barrier, then every block adds the partials in the
// same order.  Every thread receives the totals.
template <int NV>
__device__ bool grid_total(const double (&val)[NV], double *part, BicgScalars *sc, unsigned int &epoch,
                           double (&tot)[NV]) {
    static_assert(NV <= kWarps, "one warp per total");
    __shared__ double sh[NV][kWarps];
    __shared__ double res[NV];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
    for (int q = 0; q < NV; ++q) {
        const double s = group_sum<kWarp>(val[q]);
        if (lane == 0) sh[q][w] = s;
    }
    __syncthreads();
    if (threadIdx.x == 0)
#pragma unroll
        for (int q = 0; q < NV; ++q) {
            double t = 0.0;
            for (int k = 0; k < kWarps; ++k) t += sh[q][k];
            part[q * kBicgParts + blockIdx.x] = t;
        }
    if (!grid_sync(sc, epoch)) return false;
    if (w < NV) {  // warp q adds the partials of value q, all loads in flight at once
        constexpr int M = kMaxGrid / kWarp;
        double v[M];
#pragma unroll
        for (int m = 0; m < M; ++m) {
            const int k = lane + kWarp * m;
            v[m] = k < (int)gridDim.x ? __ldcg(part + w * kBicgParts + k) : 0.0;
        }
        double s = 0.0;
#pragma unroll
        for (int m = 0; m < M; ++m) s += v[m];
        s = group_sum<kWarp>(s);
        if (lane == 0) res[w] = s;
    }
    __syncthreads();
#pragma unroll
    for (int q = 0; q < NV; ++q) tot[q] = res[q];
    __syncthreads();
    return true;
}

// the preconditioned vectors of phases A and B, with explicit rounding (gathered and stored copies agree bitwise)
__device__ __forceinline__ double2 new_ph(double2 rh, double2 ph, double2 vh, double beta, double omega) {
    return make_double2(__fma_rn(beta, __fma_rn(-omega, vh.x, ph.x), rh.x),
                        __fma_rn(beta, __fma_rn(-omega, vh.y, ph.y), rh.y));
}
__device__ __forceinline__ double2 new_sh(double2 rh, double2 vh, double alpha) {
    return make_double2(__fma_rn(-alpha, vh.x, rh.x), __fma_rn(-alpha, vh.y, rh.y));
}

struct Scal {
    double alpha, beta, omega;
};

// Phase A (STAGE 0) or B (STAGE 1) over node blocks: the product of A with the preconditioned vector formed at the
// gather, each lane keeping up to kUnroll blocks in flight; the group leader of node i then does node i's vector work
// and accumulates its share of the phase's dot products into d[].
template <int STAGE>
__device__ void product_phase(const BicgArgs &a, const Scal &c, const double *pho, const double *vho, double *phn,
                              double *vhn, double (&d)[3]) {
    constexpr int G = kSpmvLanes, GPW = kWarp / G, U = kUnroll;
    const int lane = threadIdx.x & 31, gl = lane % G;
    const int warp = (blockIdx.x * kThreads + threadIdx.x) >> 5, nwarps = (gridDim.x * kThreads) >> 5;
    for (int base = warp * GPW; base < a.n; base += nwarps * GPW) {
        const int i = base + lane / G;
        double y0 = 0.0, y1 = 0.0;
        if (i < a.n) {
            const int b0 = __ldg(a.bptr + i), nblk = __ldg(a.bptr + i + 1) - b0;
            const double2 *v0 = reinterpret_cast<const double2 *>(a.val + 4 * (size_t)b0), *v1 = v0 + nblk;
            for (int b = gl; b < nblk; b += U * G) {
                int j[U];
                double2 e0[U], e1[U];
#pragma unroll
                for (int q = 0; q < U; ++q) {
                    const int bb = b + q * G;
                    j[q] = bb < nblk ? __ldg(a.bcol + b0 + bb) : -1;
                    if (bb < nblk) {
                        e0[q] = __ldg(v0 + bb);
                        e1[q] = __ldg(v1 + bb);
                    }
                }
#pragma unroll
                for (int q = 0; q < U; ++q)
                    if (j[q] >= 0) {
                        const double2 xj = STAGE == 0
                                               ? new_ph(ld2(a.rh, j[q]), ld2(pho, j[q]), ld2(vho, j[q]), c.beta, c.omega)
                                               : new_sh(ld2(a.rh, j[q]), ld2(vhn, j[q]), c.alpha);
                        y0 += e0[q].x * xj.x + e0[q].y * xj.y;
                        y1 += e1[q].x * xj.x + e1[q].y * xj.y;
                    }
            }
        }
        y0 = group_sum<G>(y0);
        y1 = group_sum<G>(y1);
        if (i < a.n && gl == 0) {
            if (STAGE == 0) {
                const double2 ph = new_ph(ld2(a.rh, i), ld2(pho, i), ld2(vho, i), c.beta, c.omega);
                st2(phn, i, ph.x, ph.y);
                st2(a.v, i, y0, y1);
                double h0, h1;
                block2(a.binv, i, y0, y1, h0, h1);
                st2(vhn, i, h0, h1);
                const double2 r0 = ld2(a.r0, i);
                d[0] += r0.x * y0 + r0.y * y1;
            } else {
                const double2 r = ld2(a.r, i), v = ld2(a.v, i);
                const double s0 = r.x - c.alpha * v.x, s1 = r.y - c.alpha * v.y;
                const double2 sh = new_sh(ld2(a.rh, i), ld2(vhn, i), c.alpha);
                st2(a.s, i, s0, s1);
                st2(a.sh, i, sh.x, sh.y);
                st2(a.t, i, y0, y1);
                d[0] += y0 * y0 + y1 * y1;
                d[1] += y0 * s0 + y1 * s1;
                d[2] += s0 * s0 + s1 * s1;
            }
        }
    }
}

__device__ __forceinline__ void finish(BicgScalars *sc, int status, int its, double relres) {
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        sc->status = status;
        sc->its = its;
        sc->relres = relres;
    }
}

__global__ void __launch_bounds__(kThreads, kBlocksPerSM) bicg_solve_kernel(BicgArgs a, double tol, int max_its) {
    BicgScalars *sc = a.sc;
    unsigned int epoch = 0;
    int set = 0;
    auto part = [&]() {
        double *p = a.part + (size_t)set * 3 * kBicgParts;
        set ^= 1;
        return p;
    };
    const int tid = blockIdx.x * kThreads + threadIdx.x, nth = gridDim.x * kThreads;
    double bb = 0.0;
    for (int i = tid; i < a.n; i += nth) {
        const double2 b = ld2(a.b, i);
        st2(a.x, i, 0.0, 0.0);
        st2(a.r, i, b.x, b.y);
        st2(a.r0, i, b.x, b.y);
        double h0, h1;
        block2(a.binv, i, b.x, b.y, h0, h1);
        st2(a.rh, i, h0, h1);
        st2(a.ph[0], i, 0.0, 0.0);
        st2(a.vh[0], i, 0.0, 0.0);
        bb += b.x * b.x + b.y * b.y;
    }
    double t1[1], t3[3];
    if (!grid_total<1>({bb}, part(), sc, epoch, t1)) return;
    const double bnorm = sqrt(t1[0]);
    if (!(bnorm > 0.0)) return finish(sc, kBicgDone, 0, 0.0);
    double rho = 1.0, rho1 = t1[0];
    Scal c{1.0, t1[0], 1.0};
    for (int k = 1;; ++k) {
        const double *pho = a.ph[(k - 1) & 1], *vho = a.vh[(k - 1) & 1];
        double *phn = a.ph[k & 1], *vhn = a.vh[k & 1];
        double d[3] = {0.0, 0.0, 0.0};
        product_phase<0>(a, c, pho, vho, phn, vhn, d);
        if (!grid_total<1>({d[0]}, part(), sc, epoch, t1)) return;
        if (t1[0] == 0.0 || !isfinite(t1[0])) return finish(sc, kBicgBreakdown, k - 1, 0.0);
        c.alpha = rho1 / t1[0];
        d[0] = d[1] = d[2] = 0.0;
        product_phase<1>(a, c, pho, vho, phn, vhn, d);
        if (!grid_total<3>({d[0], d[1], d[2]}, part(), sc, epoch, t3)) return;
        const double sn = sqrt(t3[2]);
        if (sn <= tol * bnorm) {
            for (int i = tid; i < a.n; i += nth) {
                const double2 x = ld2(a.x, i), ph = ld2(phn, i);
                st2(a.x, i, x.x + c.alpha * ph.x, x.y + c.alpha * ph.y);
            }
            return finish(sc, kBicgDone, k, sn / bnorm);
        }
        c.omega = t3[0] > 0.0 ? t3[1] / t3[0] : 0.0;
        double rr = 0.0, r0r = 0.0;
        for (int i = tid; i < a.n; i += nth) {
            const double2 x = ld2(a.x, i), ph = ld2(phn, i), sh = ld2(a.sh, i), s = ld2(a.s, i), t = ld2(a.t, i);
            const double2 r0 = ld2(a.r0, i);
            st2(a.x, i, (x.x + c.alpha * ph.x) + c.omega * sh.x, (x.y + c.alpha * ph.y) + c.omega * sh.y);
            const double q0 = s.x - c.omega * t.x, q1 = s.y - c.omega * t.y;
            st2(a.r, i, q0, q1);
            double h0, h1;
            block2(a.binv, i, q0, q1, h0, h1);
            st2(a.rh, i, h0, h1);
            rr += q0 * q0 + q1 * q1;
            r0r += r0.x * q0 + r0.y * q1;
        }
        if (!grid_total<3>({rr, r0r, 0.0}, part(), sc, epoch, t3)) return;
        const double relres = sqrt(t3[0]) / bnorm;
        if (relres <= tol) return finish(sc, kBicgDone, k, relres);
        if (k >= max_its) return finish(sc, kBicgMaxIts, k, relres);
        rho = rho1;
        rho1 = t3[1];
        if (rho1 == 0.0 || !isfinite(rho1) || c.omega == 0.0) return finish(sc, kBicgBreakdown, k, relres);
        c.beta = (rho1 / rho) * (c.alpha / c.omega);
    }
}

// vt[q] = v[perm[q]]: the values of the transposed matrix
__global__ void gather_values_kernel(long long nnz, const int *perm, const double *v, double *vt) {
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < nnz; q += (long long)gridDim.x * blockDim.x)
        vt[q] = v[__ldg(perm + q)];
}

}  // namespace

bool block_view(int n, const int *rowptr, const int *cols, std::vector<int> &bptr, std::vector<int> &bcol) {
    bptr.assign((size_t)n + 1, 0);
    bcol.clear();
    bcol.reserve((size_t)(rowptr[2 * (size_t)n] / 4));
    for (int i = 0; i < n; ++i) {
        const int lo0 = rowptr[2 * i], lo1 = rowptr[2 * i + 1], hi1 = rowptr[2 * i + 2];
        const int len = lo1 - lo0;
        if (len != hi1 - lo1 || (len & 1) || lo0 != 4 * (int)bcol.size()) return false;
        for (int k = 0; k < len; k += 2) {
            const int c = cols[lo0 + k];
            if ((c & 1) || cols[lo0 + k + 1] != c + 1 || cols[lo1 + k] != c || cols[lo1 + k + 1] != c + 1) return false;
            bcol.push_back(c >> 1);
        }
        bptr[(size_t)i + 1] = (int)bcol.size();
    }
    return true;
}

void block_transpose(int n, const std::vector<int> &bptr, const std::vector<int> &bcol, std::vector<int> &tbptr,
                     std::vector<int> &tbcol, std::vector<int> &perm) {
    const size_t nblk = bcol.size();
    tbptr.assign((size_t)n + 1, 0);
    for (int j : bcol) tbptr[(size_t)j + 1]++;
    for (int j = 0; j < n; ++j) tbptr[(size_t)j + 1] += tbptr[(size_t)j];
    tbcol.assign(nblk, 0);
    std::vector<int> fill(tbptr.begin(), tbptr.end() - 1), pos(nblk);
    for (int i = 0; i < n; ++i)  // rows in ascending order: each transposed row's columns come out sorted
        for (int p = bptr[(size_t)i]; p < bptr[(size_t)i + 1]; ++p) {
            const int q = fill[(size_t)bcol[(size_t)p]]++;
            tbcol[(size_t)q] = i;
            pos[(size_t)p] = q;
        }
    // entry (2j+a, 2i+b) of the transpose is entry (2i+b, 2j+a) of the matrix
    perm.assign(4 * nblk, 0);
    for (int i = 0; i < n; ++i) {
        const int b0 = bptr[(size_t)i], ni = bptr[(size_t)i + 1] - b0;
        for (int p = 0; p < ni; ++p) {
            const int q = pos[(size_t)(b0 + p)], j = bcol[(size_t)(b0 + p)];
            const int t0 = tbptr[(size_t)j], nj = tbptr[(size_t)j + 1] - t0, qq = q - t0;
            for (int ra = 0; ra < 2; ++ra)
                for (int rb = 0; rb < 2; ++rb)
                    perm[4 * (size_t)t0 + (size_t)ra * 2 * nj + 2 * (size_t)qq + rb] =
                        4 * b0 + rb * 2 * ni + 2 * p + ra;
        }
    }
}

cudaError_t launch_gather_values(long long nnz, const int *perm, const double *v, double *vt, cudaStream_t s) {
    const long long g = (nnz + 255) / 256;
    gather_values_kernel<<<(int)(g < 148 * 16 ? (g > 0 ? g : 1) : 148 * 16), 256, 0, s>>>(nnz, perm, v, vt);
    return cudaGetLastError();
}

cudaError_t launch_bicg_solve(const BicgArgs &a, double tol, int max_its, cudaStream_t s) {
    static int grid = 0;  // resident blocks of the device: at most kBicgParts
    if (grid == 0) {
        int dev = 0, sms = 0, per_sm = 0;
        cudaError_t e = cudaGetDevice(&dev);
        if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, bicg_solve_kernel, kThreads, 0);
        if (e != cudaSuccess) return e;
        const int g = sms * per_sm;
        if (g < 1) return cudaErrorCooperativeLaunchTooLarge;
        grid = g < kMaxGrid ? g : kMaxGrid;
    }
    cudaError_t e = cudaMemsetAsync(a.sc, 0, sizeof(BicgScalars), s);
    if (e != cudaSuccess) return e;
    BicgArgs args = a;
    void *params[] = {&args, &tol, &max_its};
    return cudaLaunchCooperativeKernel(reinterpret_cast<const void *>(bicg_solve_kernel), dim3(grid), dim3(kThreads),
                                       params, 0, s);
}

}  // namespace pxb
