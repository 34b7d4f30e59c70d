// Families on the device, in the reference's order (src/PDMesh/CreatePDMesh.cpp:910-1082; the host restatement is
// pxb_families in host_mesh.cpp, which these kernels reproduce bit for bit).
//
// The reference opens cells of size `radius` in node order and, cell by cell, pairs the cell's members (a < b)
// and then each member with the members of the forward half of its neighbour cells (4 offsets in 2D, 13 in 3D);
// every accepted pair appends j to fam(i) and i to fam(j).  So every accepted pair has a visit key
//   (rank of the processing cell, phase = 0 intra / 1 + offset index, outer position, inner position)
// and fam(x) lists the partners of x in increasing key.  A cell's rank is the order in which it was opened, i.e.
// the order of its smallest node id, so that id stands in for the rank.
//
// Steps: cell coordinates and a hash table of cells (min node id, member count); members per cell, sorted by node
// id (position = insertion order); per node, the candidates of the 3^dim surrounding cells with the reference's
// distance test, counted, then written with their keys; finally each family is sorted by key (one warp per node,
// bitonic in shared memory).
#include <cstdint>

#include "k_kernels.h"
#include "pxb_common.cuh"

namespace pxb {

namespace {

constexpr unsigned long long kEmpty = ~0ULL;

__device__ __forceinline__ unsigned long long cell_key(long ix, long iy, long iz) {
    const long b = 1L << 20;
    return ((unsigned long long)(ix + b) << 42) | ((unsigned long long)(iy + b) << 21) | (unsigned long long)(iz + b);
}

__device__ __forceinline__ unsigned long long hash64(unsigned long long k) {
    k ^= k >> 33;
    k *= 0xff51afd7ed558ccdULL;
    k ^= k >> 33;
    k *= 0xc4ceb9fe1a85ec53ULL;
    k ^= k >> 33;
    return k;
}

__device__ __forceinline__ int find_slot(const unsigned long long *keys, unsigned mask, unsigned long long key) {
    unsigned s = (unsigned)hash64(key) & mask;
    for (unsigned probe = 0; probe <= mask; ++probe) {
        const unsigned long long k = keys[s];
        if (k == key) return (int)s;
        if (k == kEmpty) return -1;
        s = (s + 1) & mask;
    }
    return -1;
}

// forward stencils of the reference (CreatePDMesh.cpp:1001-1010)
__constant__ int c_st2[4][3] = {{1, -1, 0}, {1, 0, 0}, {1, 1, 0}, {0, 1, 0}};
__constant__ int c_st3[13][3] = {{1, -1, -1}, {1, -1, 0}, {1, -1, 1}, {1, 0, -1}, {1, 0, 0}, {1, 0, 1}, {1, 1, -1},
                                 {1, 1, 0},   {1, 1, 1},  {0, 1, -1}, {0, 1, 0},  {0, 1, 1}, {0, 0, 1}};

}  // namespace

// cell coordinates of every node and insertion into the cell table (key, member count, smallest node id)
__global__ void fam_cells_kernel(FamArgs a) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < a.n; i += gridDim.x * blockDim.x) {
        const double *p = a.coords + 3 * (size_t)i;
        const long ix = (int)floor((p[0] - a.lo[0]) / a.radius);
        const long iy = (int)floor((p[1] - a.lo[1]) / a.radius);
        const long iz = a.is3d ? (int)floor((p[2] - a.lo[2]) / a.radius) : 0;
        if (ix < -(1L << 20) || ix >= (1L << 20) || iy < -(1L << 20) || iy >= (1L << 20) || iz < -(1L << 20) ||
            iz >= (1L << 20)) {
            atomicExch(a.err, 1);
            a.cell_of[i] = -1;
            continue;
        }
        a.cxyz[3 * (size_t)i] = (int)ix;
        a.cxyz[3 * (size_t)i + 1] = (int)iy;
        a.cxyz[3 * (size_t)i + 2] = (int)iz;
        const unsigned long long key = cell_key(ix, iy, iz);
        unsigned s = (unsigned)hash64(key) & a.mask;
        int slot = -1;
        for (unsigned probe = 0; probe <= a.mask; ++probe) {
            const unsigned long long prev = atomicCAS(a.keys + s, kEmpty, key);
            if (prev == kEmpty || prev == key) {
                slot = (int)s;
                break;
            }
            s = (s + 1) & a.mask;
        }
        if (slot < 0) {
            atomicExch(a.err, 2);
            a.cell_of[i] = -1;
            continue;
        }
        a.cell_of[i] = slot;
        atomicAdd(a.ccount + slot, 1);
        atomicMin(a.cminid + slot, i);
    }
}

// members of every cell (unordered), then each cell's list sorted by node id and the positions written back
__global__ void fam_members_kernel(FamArgs a) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < a.n; i += gridDim.x * blockDim.x) {
        const int s = a.cell_of[i];
        if (s < 0) continue;
        const int k = atomicAdd(a.cfill + s, 1);
        a.members[a.cstart[s] + k] = i;
    }
}

__global__ void fam_sort_cells_kernel(FamArgs a) {
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s <= (int)a.mask; s += gridDim.x * blockDim.x) {
        const int c = a.ccount[s];
        if (c == 0) continue;
        int *m = a.members + a.cstart[s];
        for (int x = 1; x < c; ++x) {  // insertion sort: cells hold a few tens of nodes
            const int v = m[x];
            int y = x - 1;
            while (y >= 0 && m[y] > v) {
                m[y + 1] = m[y];
                --y;
            }
            m[y + 1] = v;
        }
        for (int x = 0; x < c; ++x) a.pos[m[x]] = x;
    }
}

// per node x: visit the 3^dim cells around its own, test every member, count (pass 0) or write key + partner (1)
template <bool WRITE>
__global__ void fam_candidates_kernel(FamArgs a) {
    const int ns = a.is3d ? 13 : 4;
    for (int x = blockIdx.x * blockDim.x + threadIdx.x; x < a.n; x += gridDim.x * blockDim.x) {
        if (a.cell_of[x] < 0) continue;
        const int cx = a.cxyz[3 * (size_t)x], cy = a.cxyz[3 * (size_t)x + 1], cz = a.cxyz[3 * (size_t)x + 2];
        const double *px = a.coords + 3 * (size_t)x;
        const int mycell = a.cell_of[x];
        const int posx = a.pos[x];
        int cnt = 0;
        long long w = WRITE ? (long long)a.off[x] - a.off_base : 0;
        for (int dz = (a.is3d ? -1 : 0); dz <= (a.is3d ? 1 : 0); ++dz)
            for (int dy = -1; dy <= 1; ++dy)
                for (int dx = -1; dx <= 1; ++dx) {
                    const int s = find_slot(a.keys, a.mask, cell_key(cx + dx, cy + dy, cz + dz));
                    if (s < 0) continue;
                    // which cell processes the pair, and in which phase
                    int phase = -1;
                    bool x_outer = true;
                    if (dx == 0 && dy == 0 && dz == 0) {
                        phase = 0;
                    } else {
                        for (int o = 0; o < ns; ++o) {
                            const int *st = a.is3d ? c_st3[o] : c_st2[o];
                            if (st[0] == dx && st[1] == dy && st[2] == dz) { phase = 1 + o; x_outer = true; }
                            if (st[0] == -dx && st[1] == -dy && st[2] == -dz) { phase = 1 + o; x_outer = false; }
                        }
                    }
                    const int *m = a.members + a.cstart[s];
                    const int c = a.ccount[s];
                    for (int q = 0; q < c; ++q) {
                        const int j = m[q];
                        if (j == x) continue;
                        // the reference's test on (outer - inner); the squared differences do not depend on the order
                        const double *pj = a.coords + 3 * (size_t)j;
                        const double ddx = px[0] - pj[0], ddy = px[1] - pj[1], ddz = a.is3d ? (px[2] - pj[2]) : 0.0;
                        // (dx^2 + dy^2) + dz^2 with separate roundings, as the host computes it (no contraction)
                        const double d2 = __dadd_rn(__dadd_rn(__dmul_rn(ddx, ddx), __dmul_rn(ddy, ddy)), __dmul_rn(ddz, ddz));
                        if (!(d2 <= a.r2 + a.r2tol)) continue;
                        if (WRITE) {
                            unsigned long long rank, outer, inner;
                            if (phase == 0) {
                                rank = (unsigned long long)a.cminid[mycell];
                                outer = (unsigned long long)min(posx, q);
                                inner = (unsigned long long)max(posx, q);
                            } else if (x_outer) {
                                rank = (unsigned long long)a.cminid[mycell];
                                outer = (unsigned long long)posx;
                                inner = (unsigned long long)q;
                            } else {
                                rank = (unsigned long long)a.cminid[s];
                                outer = (unsigned long long)q;
                                inner = (unsigned long long)posx;
                            }
                            a.fkey[w] = (rank << 32) | ((unsigned long long)phase << 24) | (outer << 12) | inner;
                            a.fval[w] = j;
                            ++w;
                        }
                        ++cnt;
                    }
                }
        if (!WRITE) a.fcount[x] = cnt;
    }
}

// one warp per node: bitonic sort of the family's (key, partner) pairs in shared memory, partners written 0-based
__global__ void __launch_bounds__(128) fam_sort_kernel(FamArgs a) {
    constexpr int WPB = 4, CAP = kFamMax;
    __shared__ unsigned long long sk[WPB][CAP];
    __shared__ int sv[WPB][CAP];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (int x = blockIdx.x * WPB + w; x < a.n; x += gridDim.x * WPB) {
        const long long b0 = a.off[x];
        const int len = a.off[x + 1] - a.off[x];
        for (int k = lane; k < CAP; k += 32) {
            sk[w][k] = k < len ? a.fkey[b0 - a.off_base + k] : kEmpty;
            sv[w][k] = k < len ? a.fval[b0 - a.off_base + k] : 0;
        }
        __syncwarp();
        int size = 2;
        while (size < len) size <<= 1;
        for (int k = 2; k <= size; k <<= 1)
            for (int j = k >> 1; j > 0; j >>= 1) {
                for (int i = lane; i < size; i += 32) {
                    const int l = i ^ j;
                    if (l > i) {
                        const bool up = (i & k) == 0;
                        const unsigned long long ki = sk[w][i], kl = sk[w][l];
                        if ((ki > kl) == up) {
                            sk[w][i] = kl;
                            sk[w][l] = ki;
                            const int t = sv[w][i];
                            sv[w][i] = sv[w][l];
                            sv[w][l] = t;
                        }
                    }
                }
                __syncwarp();
            }
        for (int k = lane; k < len; k += 32) a.nbr[b0 + k] = sv[w][k] + a.id_base;
        __syncwarp();
    }
}

cudaError_t launch_fam_cells(const FamArgs &a, cudaStream_t s) {
    const int g = (int)((a.n + 255) / 256 < 148 * 16 ? (a.n + 255) / 256 : 148 * 16);
    fam_cells_kernel<<<g > 0 ? g : 1, 256, 0, s>>>(a);
    return cudaGetLastError();
}
cudaError_t launch_fam_members(const FamArgs &a, cudaStream_t s) {
    const int g = (int)((a.n + 255) / 256 < 148 * 16 ? (a.n + 255) / 256 : 148 * 16);
    fam_members_kernel<<<g > 0 ? g : 1, 256, 0, s>>>(a);
    return cudaGetLastError();
}
cudaError_t launch_fam_sort_cells(const FamArgs &a, cudaStream_t s) {
    const long long slots = (long long)a.mask + 1;
    const int g = (int)((slots + 255) / 256 < 148 * 16 ? (slots + 255) / 256 : 148 * 16);
    fam_sort_cells_kernel<<<g > 0 ? g : 1, 256, 0, s>>>(a);
    return cudaGetLastError();
}
cudaError_t launch_fam_candidates(const FamArgs &a, bool write, cudaStream_t s) {
    const int g = (int)((a.n + 127) / 128 < 148 * 32 ? (a.n + 127) / 128 : 148 * 32);
    if (write) fam_candidates_kernel<true><<<g > 0 ? g : 1, 128, 0, s>>>(a);
    else fam_candidates_kernel<false><<<g > 0 ? g : 1, 128, 0, s>>>(a);
    return cudaGetLastError();
}
cudaError_t launch_fam_sort(const FamArgs &a, cudaStream_t s) {
    const int g = (int)((a.n + 3) / 4 < 148 * 16 ? (a.n + 3) / 4 : 148 * 16);
    fam_sort_kernel<<<g > 0 ? g : 1, 128, 0, s>>>(a);
    return cudaGetLastError();
}

}  // namespace pxb
