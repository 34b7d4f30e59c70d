// CSR sparsity pattern on the device, the same pattern SparseMatrix::initFromPDMesh builds
// (src/MathUtils/SparseMatrix.cpp:73-185) and pxb_csr_pattern restates on the host: per node i the column nodes
// {i} u family(i) u {mirror(i)}, sorted and unique, each expanded to ndof x ndof dense blocks, 0-based.
//
// One warp per node sorts the node list in shared memory (bitonic, padded to a power of two) and compacts the
// duplicates with a ballot; the count pass and the fill pass run the same code, so the counts match the lists the
// fill writes.  Between them an exclusive scan over the nodes (three kernels: block sums, one block over the sums,
// block scans) gives every node its first block; row (i, a) starts at ndof^2 first(i) + a ndof m_i.  The fill also
// writes the block view (first block per node, column node per block) that the 2-dof solvers read.
#include <climits>

#include "k_kernels.h"
#include "pxb_common.cuh"

namespace pxb {

namespace {

constexpr int kPatCap = kFamMax;  // largest node list (family + self + mirror) a warp sorts
constexpr int kPatWarps = 4;
constexpr int kScanThreads = 512;

// the sorted unique node list of node i in out[0, m); returns m, or -1 when the list exceeds kPatCap
__device__ int node_list(const PatternArgs &a, int i, int *s, int *out) {
    const int lane = threadIdx.x & 31;
    const int b0 = a.off[i], len = a.off[i + 1] - b0;
    const int mir = a.mirror ? a.mirror[i] : 0;
    const bool has_m = mir >= 1 && mir <= a.n;
    const int tot = len + 1 + (has_m ? 1 : 0);
    if (tot > kPatCap) return -1;
    int size = 2;
    while (size < tot) size <<= 1;
    for (int k = lane; k < size; k += 32) {
        int v = INT_MAX;
        if (k < len) v = a.nbr[b0 + k];
        else if (k == len) v = i;
        else if (k == len + 1 && has_m) v = mir - 1;
        s[k] = v;
    }
    __syncwarp();
    for (int k = 2; k <= size; k <<= 1)
        for (int j = k >> 1; j > 0; j >>= 1) {
            for (int x = lane; x < size; x += 32) {
                const int l = x ^ j;
                if (l > x) {
                    const bool up = (x & k) == 0;
                    const int vx = s[x], vl = s[l];
                    if ((vx > vl) == up) {
                        s[x] = vl;
                        s[l] = vx;
                    }
                }
            }
            __syncwarp();
        }
    int m = 0;
    for (int c = 0; c < tot; c += 32) {
        const int k = c + lane;
        const int v = k < tot ? s[k] : INT_MAX;
        const bool keep = k < tot && (k == 0 || s[k - 1] != v);
        const unsigned ball = __ballot_sync(kFull, keep);
        if (keep) out[m + __popc(ball & ((1u << lane) - 1u))] = v;
        m += __popc(ball);
    }
    __syncwarp();
    return m;
}

template <bool FILL>
__global__ void __launch_bounds__(kPatWarps * 32) pattern_kernel(PatternArgs a) {
    __shared__ int s[kPatWarps][kPatCap];
    __shared__ int o[kPatWarps][kPatCap];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (int i = blockIdx.x * kPatWarps + w; i < a.n; i += gridDim.x * kPatWarps) {
        const int m = node_list(a, i, s[w], o[w]);
        if (FILL && i == a.n - 1 && lane == 0) {
            a.rowptr[(size_t)a.n * a.ndof] = (int)((long long)a.ndof * a.ndof * a.first[a.n]);
            if (a.bptr) a.bptr[a.n] = (int)a.first[a.n];
        }
        if (!FILL) {
            if (lane == 0) {
                if (m < 0) atomicAdd(a.overflow, 1);
                a.count[i] = m < 0 ? 0 : m;
            }
            continue;
        }
        if (m < 0) continue;
        const long long first = a.first[i];
        const int nd = a.ndof;
        for (int k = lane; k < m; k += 32) {
            if (a.bcol) a.bcol[first + k] = o[w][k];
            for (int r = 0; r < nd; ++r) {
                const long long row0 = (long long)nd * nd * first + (long long)r * m * nd;
                for (int b = 0; b < nd; ++b) a.cols[row0 + (long long)k * nd + b] = o[w][k] * nd + b;
            }
        }
        if (lane < nd) a.rowptr[(size_t)i * nd + lane] = (int)((long long)nd * nd * first + (long long)lane * m * nd);
        if (a.bptr && lane == 0) a.bptr[i] = (int)first;
        __syncwarp();
    }
}

// exclusive scan of count[0, n) into first[0, n] (first[n] = total), 64-bit sums
__global__ void __launch_bounds__(kScanThreads) scan_blocks_kernel(int n, const int *count, long long *bsum) {
    __shared__ long long sh[kScanThreads / 32];
    const int i = blockIdx.x * kScanThreads + threadIdx.x;
    long long v = i < n ? count[i] : 0;
    v = group_sum<kWarp>(v);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
        long long t = 0;
        for (int k = 0; k < kScanThreads / 32; ++k) t += sh[k];
        bsum[blockIdx.x] = t;
    }
}

__global__ void __launch_bounds__(kScanThreads) scan_sums_kernel(int nblocks, long long *bsum, long long *total) {
    __shared__ long long carry;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (int c = 0; c < nblocks; c += kScanThreads) {
        const int k = c + threadIdx.x;
        const long long v = k < nblocks ? bsum[k] : 0;
        long long incl = v;  // inclusive warp scan, then across warps
        for (int o = 1; o < 32; o <<= 1) {
            const long long t = __shfl_up_sync(kFull, incl, o);
            if ((threadIdx.x & 31) >= o) incl += t;
        }
        __shared__ long long wsum[kScanThreads / 32];
        if ((threadIdx.x & 31) == 31) wsum[threadIdx.x >> 5] = incl;
        __syncthreads();
        long long before = carry;
        for (int q = 0; q < (int)(threadIdx.x >> 5); ++q) before += wsum[q];
        if (k < nblocks) bsum[k] = before + incl - v;
        __syncthreads();
        if (threadIdx.x == kScanThreads - 1) carry = before + incl;
        __syncthreads();
    }
    if (threadIdx.x == 0) *total = carry;
}

__global__ void __launch_bounds__(kScanThreads) scan_apply_kernel(int n, const int *count, const long long *bsum,
                                                                  const long long *total, long long *first) {
    __shared__ long long wsum[kScanThreads / 32];
    const int i = blockIdx.x * kScanThreads + threadIdx.x;
    const long long v = i < n ? count[i] : 0;
    long long incl = v;
    for (int o = 1; o < 32; o <<= 1) {
        const long long t = __shfl_up_sync(kFull, incl, o);
        if ((threadIdx.x & 31) >= o) incl += t;
    }
    if ((threadIdx.x & 31) == 31) wsum[threadIdx.x >> 5] = incl;
    __syncthreads();
    long long before = bsum[blockIdx.x];
    for (int q = 0; q < (int)(threadIdx.x >> 5); ++q) before += wsum[q];
    if (i < n) first[i] = before + incl - v;
    if (i == n - 1 || (n == 0 && i == 0)) first[n] = *total;
}

int pattern_grid(int n) {
    const int g = (n + kPatWarps - 1) / kPatWarps;
    return g < 1 ? 1 : (g < 148 * 16 ? g : 148 * 16);
}

}  // namespace

int pattern_scan_blocks(int n) { return (n + kScanThreads - 1) / kScanThreads > 0 ? (n + kScanThreads - 1) / kScanThreads : 1; }

cudaError_t launch_pattern_count(const PatternArgs &a, long long *bsum, long long *total, cudaStream_t s) {
    pattern_kernel<false><<<pattern_grid(a.n), kPatWarps * 32, 0, s>>>(a);
    const int nb = pattern_scan_blocks(a.n);
    scan_blocks_kernel<<<nb, kScanThreads, 0, s>>>(a.n, a.count, bsum);
    scan_sums_kernel<<<1, kScanThreads, 0, s>>>(nb, bsum, total);
    scan_apply_kernel<<<nb, kScanThreads, 0, s>>>(a.n, a.count, bsum, total, a.first);
    return cudaGetLastError();
}

cudaError_t launch_pattern_fill(const PatternArgs &a, cudaStream_t s) {
    pattern_kernel<true><<<pattern_grid(a.n), kPatWarps * 32, 0, s>>>(a);
    return cudaGetLastError();
}

}  // namespace pxb
