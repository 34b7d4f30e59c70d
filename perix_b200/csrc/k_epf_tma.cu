// explicit_pddo_frac step with the bond streams staged through shared memory by TMA bulk copies.
//
// Each block cycles through tiles of NT consecutive nodes (grid-stride).  A tile's families form one
// contiguous bond range, so its per-bond streams (health byte, neighbour id, the c Navier operator streams)
// and its per-node rows (offsets, positions, u^n, u^{n-1}) are each one contiguous span of global memory.
// One thread fetches them with cp.async.bulk 1D copies (16-byte aligned starts and sizes: the bond range is
// widened to multiples of 16 bonds, the allocations carry the padding) into an S-stage ring, completing on a
// per-stage "full" mbarrier.  Consumers wait on that mbarrier, so DRAM streaming for the next S-1 tiles runs
// while the current tile computes; only the neighbour gathers (mostly L2 hits) remain ordinary loads.
// There is no block-wide barrier per tile: each warp, when done with a stage, counts itself in a shared
// counter; the warp that completes the count refills the stage with the block's tile k+S.  Warps therefore
// drift up to S tiles apart, which hides the gather latency of one warp behind the arithmetic of another.
// The compute is the lanes-per-node schedule of k_epf.cu (LPN lanes per node, UNR bonds per lane per pass,
// NT = 8 warps * 32/LPN nodes per tile).
//
// Every wait is bounded: a warp that gives up raises a shared flag and leaves the tile loop, the others leave
// at their next tile, the block's copies still in flight are waited for (bounded), and the kernel records
// the failure in err[0].  No TMA multicast is used.
// The same pipeline serves the device adjoint's reverse sweep (epf_adjoint_tma_kernel, below): the tile's ids,
// reverse health bytes and node rows staged, the reverse operators prefetched into L2.
#include <type_traits>

#include "k_kernels.h"
#include "pxb_common.cuh"

namespace pxb {

namespace {

__device__ __forceinline__ unsigned smem_u32(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(unsigned long long *bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(unsigned long long *bar, unsigned bytes) {
    asm volatile(
        "{\n\t.reg .b64 st;\n\t"
        "mbarrier.arrive.expect_tx.shared::cta.b64 st, [%0], %1;\n\t}" ::"r"(smem_u32(bar)),
        "r"(bytes)
        : "memory");
}

constexpr unsigned kSuspendNs = 1000;  // try_wait suspend-time hint
constexpr int kTileDesc = 64;          // bond ranges of its first tiles a block loads up front

__device__ __forceinline__ bool mbar_try_wait(unsigned long long *bar, unsigned parity) {
    unsigned ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity), "r"(kSuspendNs)
        : "memory");
    return ok != 0;
}

// bounded wait: false if the phase did not complete within the iteration budget.  Each try_wait may suspend
// the thread for up to kSuspendNs (it resumes as soon as the phase completes), so a waiting warp issues few
// instructions; the default budget is 2^19 tries (about half a second).
constexpr int kWaitTries = 1 << 19;
__device__ __forceinline__ bool mbar_wait(unsigned long long *bar, unsigned parity, int tries = kWaitTries) {
    for (int it = 0; it < tries; ++it)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}

__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, unsigned bytes, unsigned long long *bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}

// the same copy with an L2 cache-policy operand (createpolicy): bond streams larger than the L2 are read once per
// step, so they go in as evict-first and leave the node rows the neighbour gathers reuse resident in L2
__device__ __forceinline__ void bulk_g2s_hint(void *dst, const void *src, unsigned bytes, unsigned long long *bar,
                                              unsigned long long policy) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint [%0], [%1], %2, [%3], %4;" ::
            "r"(smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(bar)), "l"(policy)
        : "memory");
}

// bulk prefetch of [src, src + bytes) into L2 (no shared memory, no barrier); src 16-byte aligned, bytes % 16 == 0
__device__ __forceinline__ void bulk_prefetch_l2(const void *src, unsigned bytes) {
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(src), "r"(bytes) : "memory");
}

// per-thread asynchronous copy of one element (4 or 8 bytes, both addresses aligned to it) global -> shared, and
// its group fences
template <typename T>
__device__ __forceinline__ void cp_async_elem(T *dst, const T *src) {
    static_assert(sizeof(T) == 4 || sizeof(T) == 8, "4- or 8-byte elements");
    if constexpr (sizeof(T) == 8)
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(smem_u32(dst)), "l"(src) : "memory");
    else
        asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(smem_u32(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

__device__ __forceinline__ unsigned long long policy_evict_first() {
    unsigned long long p;
    asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
    return p;
}

__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }

__device__ __forceinline__ unsigned up16(unsigned b) { return (b + 15u) & ~15u; }

__device__ __forceinline__ double ref_stretch_t(double y2, double r2) {
    const double r = sqrt(r2);
    return __ddiv_rn(__dsub_rn(sqrt(y2), r), r);
}

template <int DIM>
__device__ __forceinline__ double dot_rn_t(const double *a, const double *b) {
    double s = __dmul_rn(a[0], b[0]);
    s = __dadd_rn(s, __dmul_rn(a[1], b[1]));
    if constexpr (DIM == 3) s = __dadd_rn(s, __dmul_rn(a[2], b[2]));
    return s;
}

// P = packed Navier coefficients of the bond (navier_pack_kernel): 2D (p11, p22, pxy), 3D (p11, p22, p33,
// p12, p13, p23), symmetric; L += P e as a chain of FMAs per component
template <int DIM>
__device__ __forceinline__ void navier_acc_t(const double *p, const double *e, double *L) {
    if constexpr (DIM == 3) {
        L[0] = fma(p[0], e[0], fma(p[3], e[1], fma(p[4], e[2], L[0])));
        L[1] = fma(p[3], e[0], fma(p[1], e[1], fma(p[5], e[2], L[1])));
        L[2] = fma(p[4], e[0], fma(p[5], e[1], fma(p[2], e[2], L[2])));
    } else {
        L[0] = fma(p[0], e[0], fma(p[2], e[1], L[0]));
        L[1] = fma(p[2], e[0], fma(p[1], e[1], L[1]));
    }
}

template <int DIM>
__device__ __forceinline__ double pick_t(const double *v, int d) {
    double r = v[0];
#pragma unroll
    for (int k = 1; k < DIM; ++k)
        if (d == k) r = v[k];
    return r;
}

// stage layout (bytes, all sections 16-aligned): G[NC][maxb] (not with PL2) | nbr[maxb] | health[maxb] |
// off[NT+16] | pos[NT] | u[NT*DIM + 2] | uprev[NT*DIM + 2] | (XI) xi[DIM][maxb] FP32 bond vectors
template <int DIM, bool MIXED, int NT, bool XI = false, bool PL2 = false>
struct StageLayout {
    static constexpr int NC = (DIM == 3) ? 6 : 3;
    static constexpr int ES = MIXED ? 4 : 8;
    static constexpr int PS = (DIM == 3) ? 32 : 16;
    __host__ __device__ static unsigned g_off(int) { return 0; }
    // PL2: the coefficients are not staged (prefetched into L2 and loaded per lane)
    __host__ __device__ static unsigned nbr_off(int maxb) { return PL2 ? 0u : (unsigned)(NC * maxb * ES); }
    __host__ __device__ static unsigned h_off(int maxb) { return nbr_off(maxb) + (unsigned)maxb * 4u; }
    __host__ __device__ static unsigned off_off(int maxb) { return h_off(maxb) + (unsigned)maxb; }
    __host__ __device__ static unsigned pos_off(int maxb) { return off_off(maxb) + (unsigned)(NT + 16) * 4u; }
    __host__ __device__ static unsigned u_off(int maxb) { return pos_off(maxb) + (unsigned)NT * PS; }
    __host__ __device__ static unsigned up_off(int maxb) {
        return u_off(maxb) + (((unsigned)(NT * DIM + 2) * 8u + 15u) & ~15u);
    }
    __host__ __device__ static unsigned xi_off(int maxb) {
        return up_off(maxb) + (((unsigned)(NT * DIM + 2) * 8u + 15u) & ~15u);
    }
    __host__ __device__ static unsigned bytes(int maxb) {
        return xi_off(maxb) + (XI ? (unsigned)(DIM * maxb) * 4u : 0u);
    }
};

// Stretch test of one bond in the reference's FP64 arithmetic (ExplicitPDDOFracElement.cpp:239-299): a squared
// comparison decides bonds clearly away from the threshold, (sqrt(y2) - r)/r > s_c with rounded ops decides the
// rest.  Returns 1 (breaks), 0 (holds), or 0 for a zero-length bond (never tested).
template <int DIM, typename PosT>
__device__ __forceinline__ int break_fp64(const PosT &xj, const PosT &xi, const double *e, const EpfArgs &a) {
    double xv[DIM], yv[DIM];
    xv[0] = __dsub_rn(xj.x, xi.x);
    xv[1] = __dsub_rn(xj.y, xi.y);
    if constexpr (DIM == 3) xv[2] = __dsub_rn(xj.z, xi.z);
#pragma unroll
    for (int d = 0; d < DIM; ++d) yv[d] = __dadd_rn(xv[d], e[d]);
    const double r2 = dot_rn_t<DIM>(xv, xv);
    if (!(r2 > 0.0)) return 0;
    const double y2 = dot_rn_t<DIM>(yv, yv);
    const double band = 1.0e-6 * r2;
    const double qh = y2 - a.sc_hi2 * r2;
    if (a.tension_only) {
        if (qh > band) return 1;
        if (qh < -band) return 0;
        return ref_stretch_t(y2, r2) > a.sc ? 1 : 0;
    }
    const double ql = a.sc_lo2 * r2 - y2;
    if (qh > band || ql > band) return 1;
    if (qh < -band && ql < -band) return 0;
    return fabs(ref_stretch_t(y2, r2)) > a.sc ? 1 : 0;
}

}  // namespace

// FLAGS bit 0 (XI): stage FP32 bond vectors for an FP32 stretch pre-test (both precisions); bit 1 (PL2): do not stage
// the packed coefficients but prefetch each tile's coefficient ranges into L2 with bulk prefetches as its copies are
// issued, and load them per lane at the start of each pass (the stage then holds ids, health and node rows only, so
// shared memory no longer limits the resident warps)
template <int DIM, bool MIXED, int LPN, int UNR, int S, int MINB, int WPB, int FLAGS>
__global__ void __launch_bounds__(WPB * 32, MINB) epf_tma_kernel(EpfArgs a) {
    constexpr bool XI = (FLAGS & 1) != 0;
    constexpr bool PL2 = (FLAGS & 2) != 0;
    // CPA (bit 2, with PL2): each lane copies its next pass's coefficients from L2 into a private double buffer in
    // shared memory (cp.async) while it computes the current pass, instead of holding them in registers
    constexpr bool CPA = PL2 && (FLAGS & 4) != 0;
    // EF (bit 3): the displacement-first clear-hold test |e|^2 < e2_hold, which needs no positions; only the bonds
    // that fail it gather x_j for the reference test
    constexpr bool EF = (FLAGS & 8) != 0 && !XI;
    constexpr bool XS = XI;
    using PosT = typename Vec<DIM>::T;
    using GT = typename std::conditional<MIXED, float, double>::type;
    constexpr int GPW = kWarp / LPN;
    constexpr int NT = WPB * GPW;
    using SL = StageLayout<DIM, MIXED, NT, XI, PL2>;
    constexpr int NC = SL::NC;

    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ unsigned long long bar[S];
    __shared__ int s_t0a[S];
    __shared__ unsigned s_done[S];  // warps finished with the stage's current tile
    __shared__ int s_last[S];       // block-local sequence number of the last copy issued into the stage
    __shared__ int s_fail;
    __shared__ int s_d0[kTileDesc], s_d1[kTileDesc];  // bond range of the block's first tiles
    __shared__ unsigned long long s_umax[WPB];
    __shared__ unsigned long long s_broken[WPB];

    const int tid = threadIdx.x;
    const int lane = tid & 31;
    const int wib = tid >> 5;
    const int gl = lane & (LPN - 1);
    const int grp = lane / LPN;
    const int maxb = a.maxb;
    const unsigned stage_bytes = SL::bytes(maxb);
    const PosT *pos = static_cast<const PosT *>(a.pos);
    const GT *Pg = static_cast<const GT *>(a.P);
    const bool rate = a.rate != 0;  // RATE: the acceleration out, no u^{n-1} stream, no BC pass
    const float sc_hi2f = (float)a.sc_hi2, sc_lo2f = (float)a.sc_lo2;
    // FP64 clear-hold test with the rounding band folded into the thresholds: y2 < ((1+sc)^2 - 1e-6) r2 and
    // y2 > ((1-sc)^2 + 1e-6) r2 (the rounding of these two constants is far inside the band)
    const double hi_band = a.sc_hi2 - 1.0e-6, lo_band = a.sc_lo2 + 1.0e-6;

    const int ntiles = (a.n - a.node0 + NT - 1) / NT;
    const int mycount = blockIdx.x < ntiles ? (ntiles - 1 - (int)blockIdx.x) / (int)gridDim.x + 1 : 0;

    // one thread: fetch the block's k-th tile into stage k % S
    auto issue = [&](int k) {
        const int st = k % S;
        const int tile = (int)blockIdx.x + k * (int)gridDim.x;
        const int n0 = a.node0 + tile * NT;
        const int cnt = min(NT, a.n - n0);
        const int t0 = k < kTileDesc ? s_d0[k] : __ldg(a.off + n0);
        const int t1 = k < kTileDesc ? s_d1[k] : __ldg(a.off + n0 + cnt);
        const int t0a = t0 & ~15;
        const unsigned nbond = up16((unsigned)(t1 - t0a));
        unsigned char *base = smem + (size_t)st * stage_bytes;
        const unsigned bytes_g = nbond * SL::ES, bytes_n = nbond * 4u, bytes_h = nbond;
        const unsigned bytes_off = up16((unsigned)(cnt + 1) * 4u);
        const unsigned bytes_pos = (unsigned)cnt * SL::PS;
        const unsigned bytes_u = up16((unsigned)cnt * DIM * 8u);
        const unsigned bytes_up = rate ? 0u : bytes_u;
        const unsigned total = (PL2 ? 0u : NC * bytes_g) + bytes_n + bytes_h + bytes_off + bytes_pos + bytes_u +
                               bytes_up + (XS ? (unsigned)DIM * bytes_n : 0u);
        s_t0a[st] = t0a;
        s_last[st] = k;
        fence_proxy_async();
        mbar_arrive_expect_tx(&bar[st], total);
        if (a.evict_first) {
            const unsigned long long ef = policy_evict_first();
#pragma unroll
            for (int c = 0; c < NC; ++c) {
                // the prefetch keeps the normal priority (the streaming loads that consume it mark it evict-first);
                // prefetched as evict-first, lines were evicted before use
                if constexpr (PL2) bulk_prefetch_l2(Pg + (size_t)c * a.nb + t0a, bytes_g);
                else bulk_g2s_hint(base + (size_t)c * maxb * SL::ES, Pg + (size_t)c * a.nb + t0a, bytes_g, &bar[st], ef);
            }
            bulk_g2s_hint(base + SL::nbr_off(maxb), a.nbr + t0a, bytes_n, &bar[st], ef);
            bulk_g2s_hint(base + SL::h_off(maxb), a.health + t0a, bytes_h, &bar[st], ef);
        } else {
#pragma unroll
            for (int c = 0; c < NC; ++c) {
                if constexpr (PL2) bulk_prefetch_l2(Pg + (size_t)c * a.nb + t0a, bytes_g);
                else bulk_g2s(base + (size_t)c * maxb * SL::ES, Pg + (size_t)c * a.nb + t0a, bytes_g, &bar[st]);
            }
            bulk_g2s(base + SL::nbr_off(maxb), a.nbr + t0a, bytes_n, &bar[st]);
            bulk_g2s(base + SL::h_off(maxb), a.health + t0a, bytes_h, &bar[st]);
        }
        bulk_g2s(base + SL::off_off(maxb), a.off + n0, bytes_off, &bar[st]);
        bulk_g2s(base + SL::pos_off(maxb), pos + n0, bytes_pos, &bar[st]);
        bulk_g2s(base + SL::u_off(maxb), a.u + (size_t)n0 * DIM, bytes_u, &bar[st]);
        if (!rate) bulk_g2s(base + SL::up_off(maxb), a.u_other + (size_t)n0 * DIM, bytes_up, &bar[st]);
        if constexpr (XS) {
#pragma unroll
            for (int d = 0; d < DIM; ++d)
                if (a.evict_first)
                    bulk_g2s_hint(base + SL::xi_off(maxb) + (size_t)d * maxb * 4u, a.xib + (size_t)d * a.nb + t0a,
                                  bytes_n, &bar[st], policy_evict_first());
                else
                    bulk_g2s(base + SL::xi_off(maxb) + (size_t)d * maxb * 4u, a.xib + (size_t)d * a.nb + t0a,
                             bytes_n, &bar[st]);
        }
    };

    if (tid == 0) {
        for (int s = 0; s < S; ++s) {
            mbar_init(&bar[s], 1);
            s_done[s] = 0;
            s_last[s] = -1;
        }
        s_fail = 0;
        fence_mbar_init();
    }
    // launched with programmatic serialisation (a captured loop of steps), the next step may start its blocks now:
    // they only run the set-up above their wait while this grid's blocks finish
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    // the bond ranges of the block's first tiles, all loaded at once: a refill then issues its copies without
    // first waiting on a global load (family offsets never change during a run)
    for (int k = tid; k < mycount && k < kTileDesc; k += WPB * kWarp) {
        const int n0 = a.node0 + ((int)blockIdx.x + k * (int)gridDim.x) * NT;
        s_d0[k] = __ldg(a.off + n0);
        s_d1[k] = __ldg(a.off + min(n0 + NT, a.n));
    }
    __syncthreads();
    // nothing a previous step writes (u, health, counters) is read before this point: wait for the previous grid
    // to complete and its writes to be visible (returns at once when the launch had no programmatic dependency)
    asm volatile("griddepcontrol.wait;" ::: "memory");
    const double t_new = a.t_sched ? a.t_sched[a.step_in_chunk] : 0.0;
    if (tid == 0)
        for (int k = 0; k < S && k < mycount; ++k) issue(k);

    unsigned long long broken = 0;
    double umax = 0.0;

    for (int k = 0; k < mycount; ++k) {
        const int st = k % S;
        if (*(volatile int *)&s_fail) break;
        // the consumers' wait (its budget: EpfArgs::wait_tries, the default unless a test shortens it); the drain
        // of the copies in flight after a failure below always keeps the default budget
        const bool ok_wait = __all_sync(kFull, mbar_wait(&bar[st], (unsigned)((k / S) & 1), a.wait_tries));
        if (!ok_wait) {
            if (lane == 0) atomicExch(&s_fail, 1);
            break;
        }
        unsigned char *base = smem + (size_t)st * stage_bytes;
        const GT *sP = reinterpret_cast<const GT *>(base);
        const int *sN = reinterpret_cast<const int *>(base + SL::nbr_off(maxb));
        unsigned char *sH = base + SL::h_off(maxb);
        const int *sOff = reinterpret_cast<const int *>(base + SL::off_off(maxb));
        const PosT *sPos = reinterpret_cast<const PosT *>(base + SL::pos_off(maxb));
        const double *sU = reinterpret_cast<const double *>(base + SL::u_off(maxb));
        const double *sUp = reinterpret_cast<const double *>(base + SL::up_off(maxb));
        const float *sXi = reinterpret_cast<const float *>(base + SL::xi_off(maxb));
        const int t0a = s_t0a[st];
        const int n0 = a.node0 + ((int)blockIdx.x + k * (int)gridDim.x) * NT;
        const int cnt = min(NT, a.n - n0);
        const int li = wib * GPW + grp;  // tile-local node of this group
        const bool act = li < cnt;
        const int i = n0 + li;
        int b0 = 0, b1 = 0;
        PosT xi{};
        double ui[DIM];
#pragma unroll
        for (int d = 0; d < DIM; ++d) ui[d] = 0.0;
        // the node's BC words, loaded before the bond passes so that their latency overlaps them
        unsigned own_bits = 0;
        int bce0 = 0, bce1 = 0;
        if (act) {
            b0 = sOff[li] - t0a;
            b1 = sOff[li + 1] - t0a;
            xi = sPos[li];
#pragma unroll
            for (int d = 0; d < DIM; ++d) ui[d] = sU[li * DIM + d];
            if (!rate) {
                if (a.bc_own) own_bits = __ldg(a.bc_own + i);
                if (a.bc_off) {
                    bce0 = __ldg(a.bc_off + i);
                    bce1 = __ldg(a.bc_off + i + 1);
                }
            }
        }
        double L[DIM];
#pragma unroll
        for (int d = 0; d < DIM; ++d) L[d] = 0.0;
        // UNR bonds per lane per pass: staged reads, then all neighbour gathers, then the arithmetic
        // CPA: this lane's double buffer, [buf][q][c] with the lane index innermost (conflict-free)
        GT *cbuf = nullptr;
        auto cpa_issue = [&](int tb, int buf) {
            const GT *Pt = Pg + t0a;
#pragma unroll
            for (int q = 0; q < UNR; ++q) {
                const int t = tb + q * LPN;
                if (t < b1) {
#pragma unroll
                    for (int c = 0; c < NC; ++c)
                        cp_async_elem(cbuf + ((size_t)(buf * UNR + q) * NC + c) * kWarp, Pt + (size_t)c * a.nb + t);
                }
            }
            cp_async_commit();
        };
        if constexpr (CPA) {
            cbuf = reinterpret_cast<GT *>(smem + (size_t)S * stage_bytes) + (size_t)wib * 2 * UNR * NC * kWarp + lane;
            cpa_issue(b0 + gl, 0);
        }
        int pass = 0;
        for (int t0 = b0 + gl; t0 < b1; t0 += LPN * UNR, ++pass) {
            if constexpr (CPA) {  // the next pass's copies go out, this pass's must have landed
                cpa_issue(t0 + LPN * UNR, (pass + 1) & 1);
                cp_async_wait<1>();
            }
            uint8_t h[UNR];
            int j[UNR];
#pragma unroll
            for (int q = 0; q < UNR; ++q) {
                const int t = t0 + q * LPN;
                const bool ok = t < b1;
                h[q] = ok ? sH[t] : (uint8_t)0;
                j[q] = ok ? sN[t] : i;  // past the family: the node itself (a valid gather, masked by h = 0)
            }
            // PL2: the pass's coefficients from L2 (prefetched with the tile), issued before the gathers
            GT pv[PL2 ? UNR : 1][NC];
            if constexpr (PL2 && !CPA) {
                const GT *Pt = Pg + t0a;
#pragma unroll
                for (int q = 0; q < UNR; ++q) {
                    const int t = t0 + q * LPN;
#pragma unroll
                    for (int c = 0; c < NC; ++c) pv[q][c] = t < b1 ? __ldcs(Pt + (size_t)c * a.nb + t) : GT(0);
                }
            }
            // the gathers are unconditional (broken bonds and the tail read valid rows and are masked below)
            PosT xj[UNR];
            double uj[UNR][DIM];
#pragma unroll
            for (int q = 0; q < UNR; ++q) {
                if constexpr (!XS && !EF) xj[q] = ldg_vec(pos + j[q]);
                if constexpr (DIM == 2) {
                    const double2 v = __ldg(reinterpret_cast<const double2 *>(a.u) + j[q]);
                    uj[q][0] = v.x;
                    uj[q][1] = v.y;
                } else {
#pragma unroll
                    for (int d = 0; d < DIM; ++d) uj[q][d] = __ldg(a.u + (size_t)j[q] * DIM + d);
                }
            }
            // every bond of the pass as an independent stream: a squared comparison accepts the bonds that clearly
            // hold (nearly all of them); the others (breaking, or within the rounding band of the threshold) take
            // the reference test in a rarely entered branch; then the forces of the held bonds
            bool hold[UNR], slow[UNR];
            double e[UNR][DIM];
            bool any_slow = false;
#pragma unroll
            for (int q = 0; q < UNR; ++q) {
                const int t = t0 + q * LPN;
#pragma unroll
                for (int d = 0; d < DIM; ++d) e[q][d] = __dsub_rn(uj[q][d], ui[d]);
                bool fast = true;  // clearly holds
                if (a.damage) {
                    if constexpr (EF) {
                        // |s| = ||xi + e| - |xi|| / |xi| <= |e| / r_min: below the bound the bond holds under either
                        // criterion, whatever its direction (the bound keeps a 1e-6 relative margin for rounding)
                        double e2 = e[q][0] * e[q][0] + e[q][1] * e[q][1];
                        if constexpr (DIM == 3) e2 = fma(e[q][2], e[q][2], e2);
                        fast = e2 < a.e2_hold;
                    } else if constexpr (XS) {
                        // FP32 squared test on the staged FP32 bond vector.  Its error (ξ rounded to FP32, e
                        // rounded, FP32 sums: < 1e-6 r^2 wherever |y|^2 is near (1 +- s_c)^2 r^2) stays well inside
                        // the 4e-6 r^2 band; outside the clear-hold region the reference arithmetic decides on the
                        // exact positions (gathered only then), so decisions equal the FP64 path's.
                        const bool ok = t < b1;
                        float xf[DIM], yf[DIM];
#pragma unroll
                        for (int d = 0; d < DIM; ++d) {
                            xf[d] = ok ? sXi[(size_t)d * maxb + t] : 0.f;
                            yf[d] = xf[d] + (float)e[q][d];
                        }
                        float r2f = xf[0] * xf[0] + xf[1] * xf[1];
                        float y2f = yf[0] * yf[0] + yf[1] * yf[1];
                        if constexpr (DIM == 3) {
                            r2f += xf[2] * xf[2];
                            y2f += yf[2] * yf[2];
                        }
                        const float bandf = 4.0e-6f * r2f;
                        fast = (y2f - sc_hi2f * r2f < -bandf) && (a.tension_only || sc_lo2f * r2f - y2f < -bandf);
                        fast = fast || !(r2f > 0.f);
                    } else {
                        // contracted FP64 (a few ulps of r2 and y2, far inside the 1e-6 r2 band)
                        double xv[DIM], yv[DIM];
                        xv[0] = xj[q].x - xi.x;
                        xv[1] = xj[q].y - xi.y;
                        if constexpr (DIM == 3) xv[2] = xj[q].z - xi.z;
#pragma unroll
                        for (int d = 0; d < DIM; ++d) yv[d] = xv[d] + e[q][d];
                        double r2 = xv[0] * xv[0] + xv[1] * xv[1];
                        double y2 = yv[0] * yv[0] + yv[1] * yv[1];
                        if constexpr (DIM == 3) {
                            r2 = fma(xv[2], xv[2], r2);
                            y2 = fma(yv[2], yv[2], y2);
                        }
                        fast = (y2 < hi_band * r2) && (a.tension_only || y2 > lo_band * r2);
                        fast = fast || !(r2 > 0.0);
                    }
                }
                hold[q] = h[q] && fast;
                slow[q] = h[q] && !fast;
                any_slow = any_slow || slow[q];
            }
            if (any_slow) {
#pragma unroll
                for (int q = 0; q < UNR; ++q) {
                    if (!slow[q]) continue;
                    int brk;
                    if constexpr (XS || EF) brk = break_fp64<DIM>(ldg_vec(pos + j[q]), xi, e[q], a);
                    else brk = break_fp64<DIM>(xj[q], xi, e[q], a);
                    if (brk) {
                        a.health[t0a + t0 + q * LPN] = 0;
                        ++broken;
                    } else {
                        hold[q] = true;
                    }
                }
            }
#pragma unroll
            for (int q = 0; q < UNR; ++q) {
                if (!hold[q]) continue;
                const int t = t0 + q * LPN;
                double pd[NC];
#pragma unroll
                for (int c = 0; c < NC; ++c) {
                    if constexpr (CPA) pd[c] = (double)cbuf[((size_t)((pass & 1) * UNR + q) * NC + c) * kWarp];
                    else if constexpr (PL2) pd[c] = (double)pv[q < (PL2 ? UNR : 1) ? q : 0][c];
                    else pd[c] = (double)sP[(size_t)c * maxb + t];
                }
                navier_acc_t<DIM>(pd, e[q], L);
            }
        }
        if constexpr (CPA) cp_async_wait<0>();  // nothing of this lane's may still land in its buffer
#pragma unroll
        for (int d = 0; d < DIM; ++d) L[d] = group_sum<LPN>(L[d]);

        double unew = 0.0;
        if (act && gl < DIM) {
            const int d = gl;
            // the body force by selects (a runtime index into the parameter array would go through local memory)
            const double bd = d == 0 ? a.b[0] : (d == 1 ? a.b[1] : a.b[DIM - 1]);
            const double acc = __ddiv_rn(__dadd_rn(pick_t<DIM>(L, d), bd), a.rho);
            const size_t kk = (size_t)i * DIM + d;
            if (rate) {
                a.accel[kk] = acc;
            } else {
                unew = cd_next(pick_t<DIM>(ui, d), sUp[li * DIM + d], acc, a.dt2, a.var_step, a.cv_rho, a.cv_w);
                const bool owned = (own_bits >> d) & 1u;
                if (!owned) {
                    a.u_other[kk] = unew;
                    umax = max_nan(umax, fabs(unew));
                }
            }
        }
        if (a.bc_off && !rate) {
            double un[DIM];
#pragma unroll
            for (int d = 0; d < DIM; ++d) un[d] = __shfl_sync(kFull, unew, grp * LPN + d);
            for (int e = bce0 + gl; e < bce1; e += LPN) {
                const int comp = a.bc_comp[e];
                const int form = a.bc_form[e];
                const double g1 = __dadd_rn(a.bc_val[e], __dmul_rn(a.bc_vel[e], t_new));
                double v;
                if (form == 0) v = pick_t<DIM>(un, comp);
                else if (form == 1) v = g1;
                else if (form == 2) v = __dsub_rn(__dmul_rn(2.0, g1), pick_t<DIM>(un, comp));
                else v = __dsub_rn(__dmul_rn(2.0, g1), __dadd_rn(a.bc_val2[e], __dmul_rn(a.bc_vel2[e], t_new)));
                a.u_other[(size_t)a.bc_tgt[e] * DIM + comp] = v;
                umax = max_nan(umax, fabs(v));
            }
        }
        // stage st consumed by this warp; the warp that completes the count refills it with tile k+S
        __syncwarp();
        if (lane == 0) {
            __threadfence_block();
            if (atomicAdd(&s_done[st], 1u) == (unsigned)(WPB - 1)) {
                atomicExch(&s_done[st], 0u);
                __threadfence_block();
                if (k + S < mycount) issue(k + S);
            }
        }
    }
    __syncthreads();
    if (s_fail && tid == 0) {
        // the last tile issued into each stage may still be in flight: wait (bounded) for its copies
        for (int s = 0; s < S; ++s)
            if (s_last[s] >= 0) mbar_wait(&bar[s], (unsigned)((s_last[s] / S) & 1));
        if (a.err) atomicAdd(a.err, 1u);
    }

    umax = group_max_nan<kWarp>(umax);
    if (lane == 0) s_umax[wib] = dbl_key(umax);
    unsigned long long bsum = broken;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) bsum += __shfl_xor_sync(kFull, bsum, o);
    if (lane == 0) s_broken[wib] = bsum;
    __syncthreads();
    if (tid == 0) {
        unsigned long long bb = 0, mm = 0;
        for (int w = 0; w < WPB; ++w) {
            bb += s_broken[w];
            mm = s_umax[w] > mm ? s_umax[w] : mm;
        }
        if (bb && a.n_broken) atomicAdd(a.n_broken, bb);
        if (a.umax) atomicMax(a.umax + a.step_in_chunk, mm);
    }
}

// ---- the reverse-only adjoint step, staged -------------------------------------------------------------------
// The same per-node sums as epf_adjoint_kernel<..., REV> (k_epf.cu) with the step kernel's pipeline: tiles of NT
// consecutive nodes, one thread copies a tile's neighbour ids, reverse health bytes, family offsets and node rows
// (u, the scaled adjoint's source abar and rin) into an S-stage ring by cp.async.bulk, the reverse operators GR of the
// tile are prefetched into L2 and loaded per lane; LPN lanes per node, UNR reverse bonds a lane per pass.  Per node
//   U = sum_t hrev_t P(GR_t) Lbar_j - P(SG_m) Lbar_m,   Lbar = scale abar / rho,
//   ubar_m = c_r rin_m + c_w abar_m + U,   rout_m = c_o abar_m,   dJ/dC += Lbar_j . dP/dC(GR_t) (u_m - u_j).
// Every wait is bounded; a warp that gives up raises the block's flag, the copies in flight are drained (bounded) and
// err[0] counts the failure.
template <int DIM, int NT>
struct AdjStage {
    static constexpr unsigned ROW = ((unsigned)(NT * DIM + 2) * 8u + 15u) & ~15u;
    __host__ __device__ static unsigned h_off(int maxb) { return (unsigned)maxb * 4u; }
    __host__ __device__ static unsigned off_off(int maxb) { return h_off(maxb) + (unsigned)maxb; }
    __host__ __device__ static unsigned u_off(int maxb) { return off_off(maxb) + (unsigned)(NT + 16) * 4u; }
    __host__ __device__ static unsigned w_off(int maxb) { return u_off(maxb) + ROW; }
    __host__ __device__ static unsigned r_off(int maxb) { return w_off(maxb) + ROW; }
    __host__ __device__ static unsigned bytes(int maxb) { return r_off(maxb) + ROW; }
};

// f = P(g) e, P the Navier coefficients of the operator sums g (2D Gxx, Gyy, Gxy; 3D Gxx, Gyy, Gzz, Gxy, Gxz, Gyz)
template <int DIM>
__device__ __forceinline__ void adj_apply(const double *g, double C11, double C12, double C66, const double *e,
                                          double *f) {
    const double ac = C12 + C66;
    if constexpr (DIM == 3) {
        const double p11 = C11 * g[0] + C66 * (g[1] + g[2]), p22 = C11 * g[1] + C66 * (g[0] + g[2]),
                     p33 = C11 * g[2] + C66 * (g[0] + g[1]);
        const double p12 = ac * g[3], p13 = ac * g[4], p23 = ac * g[5];
        f[0] = p11 * e[0] + p12 * e[1] + p13 * e[2];
        f[1] = p12 * e[0] + p22 * e[1] + p23 * e[2];
        f[2] = p13 * e[0] + p23 * e[1] + p33 * e[2];
    } else {
        const double p11 = C11 * g[0] + C66 * g[1], p22 = C66 * g[0] + C11 * g[1], p12 = ac * g[2];
        f[0] = p11 * e[0] + p12 * e[1];
        f[1] = p12 * e[0] + p22 * e[1];
    }
}

template <int DIM, bool MIXED, int LPN, int UNR, int S, int MINB, int WPB>
__global__ void __launch_bounds__(WPB * 32, MINB) epf_adjoint_tma_kernel(EpfAdjArgs a) {
    using GT = typename std::conditional<MIXED, float, double>::type;
    constexpr int NC = (DIM == 3) ? 6 : 3;
    constexpr int GPW = kWarp / LPN;
    constexpr int NT = WPB * GPW;
    using SL = AdjStage<DIM, NT>;
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ unsigned long long bar[S];
    __shared__ int s_t0a[S];
    __shared__ unsigned s_done[S];
    __shared__ int s_last[S];
    __shared__ int s_fail;
    __shared__ int s_d0[kTileDesc], s_d1[kTileDesc];
    __shared__ double s_dC[WPB][3];

    const int tid = threadIdx.x, lane = tid & 31, wib = tid >> 5;
    const int gl = lane & (LPN - 1), grp = lane / LPN;
    const int maxb = a.maxb;
    const unsigned stage_bytes = SL::bytes(maxb);
    const GT *GR = static_cast<const GT *>(a.GR);
    const double lscale = a.scale * a.inv_rho;
    const int ntiles = (a.n + NT - 1) / NT;
    const int mycount = blockIdx.x < ntiles ? (ntiles - 1 - (int)blockIdx.x) / (int)gridDim.x + 1 : 0;

    auto issue = [&](int k) {
        const int st = k % S;
        const int n0 = ((int)blockIdx.x + k * (int)gridDim.x) * NT;
        const int cnt = min(NT, a.n - n0);
        const int t0 = k < kTileDesc ? s_d0[k] : __ldg(a.off + n0);
        const int t1 = k < kTileDesc ? s_d1[k] : __ldg(a.off + n0 + cnt);
        const int t0a = t0 & ~15;
        const unsigned nbond = up16((unsigned)(t1 - t0a));
        unsigned char *base = smem + (size_t)st * stage_bytes;
        const unsigned bytes_off = up16((unsigned)(cnt + 1) * 4u);
        const unsigned bytes_row = up16((unsigned)cnt * DIM * 8u);
        const unsigned total = nbond * 5u + bytes_off + 2u * bytes_row + (a.rin ? bytes_row : 0u);
        s_t0a[st] = t0a;
        s_last[st] = k;
        fence_proxy_async();
        mbar_arrive_expect_tx(&bar[st], total);
#pragma unroll
        for (int c = 0; c < NC; ++c) bulk_prefetch_l2(GR + (size_t)c * a.nb + t0a, nbond * (unsigned)sizeof(GT));
        if (a.evict_first) {
            const unsigned long long ef = policy_evict_first();
            bulk_g2s_hint(base, a.nbr + t0a, nbond * 4u, &bar[st], ef);
            bulk_g2s_hint(base + SL::h_off(maxb), a.hrev + t0a, nbond, &bar[st], ef);
        } else {
            bulk_g2s(base, a.nbr + t0a, nbond * 4u, &bar[st]);
            bulk_g2s(base + SL::h_off(maxb), a.hrev + t0a, nbond, &bar[st]);
        }
        bulk_g2s(base + SL::off_off(maxb), a.off + n0, bytes_off, &bar[st]);
        bulk_g2s(base + SL::u_off(maxb), a.u + (size_t)n0 * DIM, bytes_row, &bar[st]);
        bulk_g2s(base + SL::w_off(maxb), a.abar + (size_t)n0 * DIM, bytes_row, &bar[st]);
        if (a.rin) bulk_g2s(base + SL::r_off(maxb), a.rin + (size_t)n0 * DIM, bytes_row, &bar[st]);
    };

    if (tid == 0) {
        for (int st = 0; st < S; ++st) {
            mbar_init(&bar[st], 1);
            s_done[st] = 0;
            s_last[st] = -1;
        }
        s_fail = 0;
        fence_mbar_init();
    }
    for (int k = tid; k < mycount && k < kTileDesc; k += WPB * kWarp) {
        const int n0 = ((int)blockIdx.x + k * (int)gridDim.x) * NT;
        s_d0[k] = __ldg(a.off + n0);
        s_d1[k] = __ldg(a.off + min(n0 + NT, a.n));
    }
    __syncthreads();
    if (tid == 0)
        for (int k = 0; k < S && k < mycount; ++k) issue(k);

    double dC[3] = {0.0, 0.0, 0.0};
    for (int k = 0; k < mycount; ++k) {
        const int st = k % S;
        if (*(volatile int *)&s_fail) break;
        const bool ok_wait = __all_sync(kFull, mbar_wait(&bar[st], (unsigned)((k / S) & 1), a.wait_tries));
        if (!ok_wait) {
            if (lane == 0) atomicExch(&s_fail, 1);
            break;
        }
        unsigned char *base = smem + (size_t)st * stage_bytes;
        const int *sN = reinterpret_cast<const int *>(base);
        const unsigned char *sH = base + SL::h_off(maxb);
        const int *sOff = reinterpret_cast<const int *>(base + SL::off_off(maxb));
        const double *sU = reinterpret_cast<const double *>(base + SL::u_off(maxb));
        const double *sW = reinterpret_cast<const double *>(base + SL::w_off(maxb));
        const double *sR = reinterpret_cast<const double *>(base + SL::r_off(maxb));
        const int t0a = s_t0a[st];
        const int n0 = ((int)blockIdx.x + k * (int)gridDim.x) * NT;
        const int cnt = min(NT, a.n - n0);
        const int li = wib * GPW + grp;
        const bool act = li < cnt;
        const int m = n0 + li;
        int b0 = 0, b1 = 0;
        double um[DIM], U[DIM];
#pragma unroll
        for (int d = 0; d < DIM; ++d) {
            um[d] = act ? sU[li * DIM + d] : 0.0;
            U[d] = 0.0;
        }
        if (act) {
            b0 = sOff[li] - t0a;
            b1 = sOff[li + 1] - t0a;
        }
        const GT *Gt = GR + t0a;
        for (int t0 = b0 + gl; t0 < b1; t0 += LPN * UNR) {
            int j[UNR];
            bool h[UNR];
            GT gv[UNR][NC];
#pragma unroll
            for (int q = 0; q < UNR; ++q) {
                const int t = t0 + q * LPN;
                const bool ok = t < b1;
                j[q] = ok ? sN[t] : m;  // past the family: the node itself (a valid gather, masked by h = 0)
                h[q] = ok && sH[t] != 0;
#pragma unroll
                for (int c = 0; c < NC; ++c) gv[q][c] = ok ? __ldcs(Gt + (size_t)c * a.nb + t) : GT(0);
            }
            double Lj[UNR][DIM], uj[UNR][DIM];
            if (a.UW) {  // one interleaved row (u_j, abar_j) a bond: DIM 16-byte loads
#pragma unroll
                for (int q = 0; q < UNR; ++q) {
                    const double2 *row = reinterpret_cast<const double2 *>(a.UW + (size_t)j[q] * 2 * DIM);
                    double r[2 * DIM];
#pragma unroll
                    for (int h2 = 0; h2 < DIM; ++h2) {
                        const double2 v = __ldg(row + h2);
                        r[2 * h2] = v.x;
                        r[2 * h2 + 1] = v.y;
                    }
#pragma unroll
                    for (int d = 0; d < DIM; ++d) {
                        uj[q][d] = r[d];
                        Lj[q][d] = r[DIM + d] * lscale;
                    }
                }
            } else {
#pragma unroll
                for (int q = 0; q < UNR; ++q)
#pragma unroll
                    for (int d = 0; d < DIM; ++d) {
                        Lj[q][d] = __ldg(a.abar + (size_t)j[q] * DIM + d) * lscale;
                        uj[q][d] = __ldg(a.u + (size_t)j[q] * DIM + d);
                    }
            }
#pragma unroll
            for (int q = 0; q < UNR; ++q) {
                if (!h[q]) continue;
                double g[NC], f[DIM], e[DIM];
#pragma unroll
                for (int c = 0; c < NC; ++c) g[c] = (double)gv[q][c];
                adj_apply<DIM>(g, a.C11, a.C12, a.C66, Lj[q], f);
#pragma unroll
                for (int d = 0; d < DIM; ++d) {
                    U[d] += f[d];
                    e[d] = um[d] - uj[q][d];
                }
                const double *L = Lj[q];
                if constexpr (DIM == 3) {
                    dC[0] += L[0] * g[0] * e[0] + L[1] * g[1] * e[1] + L[2] * g[2] * e[2];
                    dC[1] += L[0] * (g[3] * e[1] + g[4] * e[2]) + L[1] * (g[3] * e[0] + g[5] * e[2]) +
                             L[2] * (g[4] * e[0] + g[5] * e[1]);
                    dC[2] += L[0] * ((g[1] + g[2]) * e[0] + g[3] * e[1] + g[4] * e[2]) +
                             L[1] * (g[3] * e[0] + (g[0] + g[2]) * e[1] + g[5] * e[2]) +
                             L[2] * (g[4] * e[0] + g[5] * e[1] + (g[0] + g[1]) * e[2]);
                } else {
                    dC[0] += L[0] * g[0] * e[0] + L[1] * g[1] * e[1];
                    dC[1] += L[0] * g[2] * e[1] + L[1] * g[2] * e[0];
                    dC[2] += L[0] * (g[1] * e[0] + g[2] * e[1]) + L[1] * (g[2] * e[0] + g[0] * e[1]);
                }
            }
        }
#pragma unroll
        for (int d = 0; d < DIM; ++d) U[d] = group_sum<LPN>(U[d]);
        if (act && gl < DIM) {
            // the own bonds' term - P(SG_m) Lbar_m, then the central difference's transpose
            double sg[NC], Lm[DIM], f[DIM];
#pragma unroll
            for (int c = 0; c < NC; ++c) sg[c] = __ldg(a.SG + (size_t)m * NC + c);
#pragma unroll
            for (int d = 0; d < DIM; ++d) Lm[d] = sW[li * DIM + d] * lscale;
            adj_apply<DIM>(sg, a.C11, a.C12, a.C66, Lm, f);
            const int d = gl;
            const double w = sW[li * DIM + d];
            const double r = a.rin ? sR[li * DIM + d] : 0.0;
            const size_t kk = (size_t)m * DIM + d;
            double ud = 0.0, fd = 0.0;
#pragma unroll
            for (int e2 = 0; e2 < DIM; ++e2) {
                if (e2 == d) {
                    ud = U[e2];
                    fd = f[e2];
                }
            }
            a.ubar[kk] = a.c_r * r + a.c_w * w + (ud - fd);
            if (a.rout) a.rout[kk] = a.c_o * w;
        }
        __syncwarp();
        if (lane == 0) {
            __threadfence_block();
            if (atomicAdd(&s_done[st], 1u) == (unsigned)(WPB - 1)) {
                atomicExch(&s_done[st], 0u);
                __threadfence_block();
                if (k + S < mycount) issue(k + S);
            }
        }
    }
    __syncthreads();
    if (s_fail && tid == 0) {
        for (int st = 0; st < S; ++st)
            if (s_last[st] >= 0) mbar_wait(&bar[st], (unsigned)((s_last[st] / S) & 1));
        if (a.err) atomicAdd(a.err, 1u);
    }
#pragma unroll
    for (int c = 0; c < 3; ++c) dC[c] = group_sum<kWarp>(dC[c]);
    if (lane == 0) {
        s_dC[wib][0] = dC[0];
        s_dC[wib][1] = dC[1];
        s_dC[wib][2] = dC[2];
    }
    __syncthreads();
    if (tid < 3 && a.dC) {
        double v = 0.0;
        for (int w = 0; w < WPB; ++w) v += s_dC[w][tid];
        atomicAdd(a.dC + tid, v);
    }
}

static LaunchShape g_last_shape{0, 0, 0};

LaunchShape epf_tma_last_shape() { return g_last_shape; }

// the per-lane coefficient double buffers of the CPA configurations (after the ring)
constexpr size_t cpa_bytes(int dim, bool mixed, int unr, int wpb, int flags) {
    return ((flags & 6) == 6) ? (size_t)wpb * 2 * unr * (dim == 3 ? 6 : 3) * kWarp * (mixed ? 4 : 8) : 0;
}

template <int DIM, bool MIXED, int LPN, int UNR, int S, int MINB, int WPB, int FLAGS>
static cudaError_t launch_tma(const EpfArgs &a, cudaStream_t s) {
    constexpr int NT = WPB * (kWarp / LPN);
    using SL = StageLayout<DIM, MIXED, NT, (FLAGS & 1) != 0, (FLAGS & 2) != 0>;
    auto k = epf_tma_kernel<DIM, MIXED, LPN, UNR, S, MINB, WPB, FLAGS>;
    constexpr size_t cpa = cpa_bytes(DIM, MIXED, UNR, WPB, FLAGS);
    const size_t smem = (size_t)S * SL::bytes(a.maxb) + cpa;
    static size_t configured = 0;
    if (smem > configured) {
        cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        configured = smem;
    }
    // resident blocks for this shared-memory size, queried once per size (the per-step rate call launches
    // outside any graph, where these queries would cost more than the launch)
    static size_t cap_smem = 0;
    static long long cap_blocks = 0;
    if (cap_blocks == 0 || cap_smem != smem) {
        int dev = 0, sms = 148, per_sm = 1;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, WPB * kWarp, smem);
        cap_blocks = (long long)sms * (per_sm > 0 ? per_sm : 1);
        cap_smem = smem;
    }
    const long long ntiles = ((long long)a.n - a.node0 + NT - 1) / NT;
    const long long cap = cap_blocks;
    const int grid = (int)(ntiles < cap ? ntiles : cap);
    g_last_shape = LaunchShape{grid > 0 ? grid : 1, WPB * kWarp, smem};
    if (a.pdl && !a.rate) {
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3((unsigned)(grid > 0 ? grid : 1));
        cfg.blockDim = dim3(WPB * kWarp);
        cfg.dynamicSmemBytes = smem;
        cfg.stream = s;
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
        attr[0].val.programmaticStreamSerializationAllowed = 1;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        const cudaError_t e = cudaLaunchKernelEx(&cfg, k, a);
        if (e != cudaSuccess) return e;
        return cudaGetLastError();
    }
    k<<<grid > 0 ? grid : 1, WPB * kWarp, smem, s>>>(a);
    return cudaGetLastError();
}

// Staged configurations: lanes per node, bonds per lane per pass, stages, minimum resident blocks (launch
// bounds), warps per block, flags (1: staged FP32 bond vectors for the stretch pre-test, 8 (2D) / 12 (3D) more
// staged bytes per bond; 2: coefficients prefetched into L2 and loaded per lane instead of staged; 4 (with 2): those
// loads go through a per-lane double buffer in shared memory filled by cp.async one pass ahead; 8 (without 1): the
// displacement-first clear-hold test, positions gathered only for the bonds it does not clear).  A tile is
// WPB * 32/LPN nodes.
struct TmaCfg {
    int lpn, unr, stages, minb, wpb, xi;
};
#define PXB_TMA2(X)                                                                                               \
    X(0, 4, 2, 2, 6, 4, 8) X(1, 4, 4, 2, 4, 4, 8) X(2, 8, 4, 3, 1, 8, 0) X(3, 8, 2, 2, 3, 8, 0)                  \
    X(4, 8, 1, 2, 4, 8, 0) X(5, 8, 2, 2, 4, 8, 0) X(6, 4, 2, 2, 6, 4, 0) X(7, 4, 4, 2, 4, 4, 0)                  \
    X(8, 8, 2, 2, 8, 4, 0) X(9, 4, 2, 2, 3, 8, 0) X(10, 4, 2, 2, 6, 4, 1) X(11, 4, 4, 2, 4, 4, 1)                \
    X(12, 8, 2, 2, 6, 4, 1) X(13, 8, 2, 3, 3, 8, 2) X(14, 4, 2, 3, 3, 8, 2) X(15, 4, 4, 3, 2, 8, 3)
#define PXB_TMA3(X)                                                                                               \
    X(0, 32, 2, 2, 1, 8, 0) X(1, 16, 2, 3, 2, 8, 2) X(2, 16, 2, 3, 2, 8, 10) X(3, 16, 3, 2, 2, 8, 10)            \
    X(4, 16, 3, 3, 2, 8, 10) X(5, 8, 2, 2, 2, 8, 10) X(6, 32, 2, 2, 2, 4, 1) X(7, 16, 1, 2, 3, 8, 10)            \
    X(8, 16, 2, 2, 2, 8, 10) X(9, 16, 1, 3, 3, 8, 2) X(10, 32, 1, 3, 3, 8, 3) X(11, 32, 2, 3, 2, 8, 10)          \
    X(12, 16, 2, 2, 2, 8, 2) X(13, 16, 2, 3, 3, 8, 6) X(14, 32, 1, 3, 3, 8, 2) X(15, 32, 1, 3, 6, 4, 2)
#define PXB_CFG(i, l, u, st, mb, w, x) {l, u, st, mb, w, x},
static constexpr TmaCfg kTma2[kEpfTmaConfigs] = {PXB_TMA2(PXB_CFG)};
static constexpr TmaCfg kTma3[kEpfTmaConfigs] = {PXB_TMA3(PXB_CFG)};
#undef PXB_CFG

int epf_tma_lanes(int dim, int which) { return dim == 3 ? kTma3[which].lpn : kTma2[which].lpn; }

int epf_tma_tile_nodes(int dim, int which) {
    const TmaCfg c = dim == 3 ? kTma3[which] : kTma2[which];
    return c.wpb * (kWarp / c.lpn);
}

template <int DIM, bool MIXED, bool XI, bool PL2>
static size_t tma_stage_bytes(int nt, int maxb) {
    switch (nt) {
        case 4: return StageLayout<DIM, MIXED, 4, XI, PL2>::bytes(maxb);
        case 8: return StageLayout<DIM, MIXED, 8, XI, PL2>::bytes(maxb);
        case 16: return StageLayout<DIM, MIXED, 16, XI, PL2>::bytes(maxb);
        case 32: return StageLayout<DIM, MIXED, 32, XI, PL2>::bytes(maxb);
        default: return StageLayout<DIM, MIXED, 64, XI, PL2>::bytes(maxb);  // 64 nodes (LPN 4 x 8 warps)
    }
}

template <int DIM, bool MIXED>
static size_t tma_smem_dm(int which, int maxb) {
    const TmaCfg c = DIM == 3 ? kTma3[which] : kTma2[which];
    const int nt = c.wpb * (kWarp / c.lpn);
    size_t per = 0;
    switch (c.xi & 3) {  // the stage layout follows the bond-vector (1) and L2-prefetch (2) bits alone
        case 0: per = tma_stage_bytes<DIM, MIXED, false, false>(nt, maxb); break;
        case 1: per = tma_stage_bytes<DIM, MIXED, true, false>(nt, maxb); break;
        case 2: per = tma_stage_bytes<DIM, MIXED, false, true>(nt, maxb); break;
        default: per = tma_stage_bytes<DIM, MIXED, true, true>(nt, maxb); break;
    }
    return (size_t)c.stages * per + cpa_bytes(DIM, MIXED, c.unr, c.wpb, c.xi);
}

size_t epf_tma_smem(int dim, bool mixed, int which, int maxb) {
    if (dim == 3) return mixed ? tma_smem_dm<3, true>(which, maxb) : tma_smem_dm<3, false>(which, maxb);
    return mixed ? tma_smem_dm<2, true>(which, maxb) : tma_smem_dm<2, false>(which, maxb);
}

#define PXB_CASE2(i, l, u, st, mb, w, x) \
    case i: return launch_tma<2, MIXED, l, u, st, mb, w, x>(a, s);
#define PXB_CASE3(i, l, u, st, mb, w, x) \
    case i: return launch_tma<3, MIXED, l, u, st, mb, w, x>(a, s);
template <int DIM, bool MIXED>
static cudaError_t launch_tma_dm(const EpfArgs &a, int which, cudaStream_t s) {
    if constexpr (DIM == 3) {
        switch (which) { PXB_TMA3(PXB_CASE3) default: return cudaErrorInvalidValue; }
    } else {
        switch (which) { PXB_TMA2(PXB_CASE2) default: return cudaErrorInvalidValue; }
    }
}
#undef PXB_CASE2
#undef PXB_CASE3

// the staged adjoint's configurations per dimension (which = 0, 1, 2): lanes per node, reverse bonds a lane per pass,
// stages, minimum resident blocks, warps per block
template <int DIM, int W>
struct AdjCfg;
template <>
struct AdjCfg<3, 0> {
    static constexpr int LPN = 16, UNR = 2, S = 3, MINB = 2, WPB = 8;
};
template <>
struct AdjCfg<3, 1> {
    static constexpr int LPN = 16, UNR = 1, S = 3, MINB = 3, WPB = 8;
};
template <>
struct AdjCfg<3, 2> {
    static constexpr int LPN = 16, UNR = 3, S = 3, MINB = 2, WPB = 8;
};
template <>
struct AdjCfg<2, 0> {
    static constexpr int LPN = 4, UNR = 2, S = 2, MINB = 4, WPB = 4;
};
template <>
struct AdjCfg<2, 1> {
    static constexpr int LPN = 4, UNR = 1, S = 2, MINB = 6, WPB = 4;
};
template <>
struct AdjCfg<2, 2> {
    static constexpr int LPN = 8, UNR = 2, S = 2, MINB = 4, WPB = 4;
};

int epf_adj_tma_maxb(int dim, int max_family) {
    // the largest tile of the configurations: 16 nodes in 3D, 32 in 2D
    const int nt = dim == 3 ? 16 : 32;
    const long long b = (long long)nt * max_family + 32;
    return (int)((b + 31) / 32 * 32);
}

template <int DIM, bool MIXED, int W>
static cudaError_t launch_adj_tma(const EpfAdjArgs &a, cudaStream_t s) {
    using Cf = AdjCfg<DIM, W>;
    constexpr int NT = Cf::WPB * (kWarp / Cf::LPN);
    static_assert(NT <= (DIM == 3 ? 16 : 32), "epf_adj_tma_maxb sizes the largest tile");
    auto k = epf_adjoint_tma_kernel<DIM, MIXED, Cf::LPN, Cf::UNR, Cf::S, Cf::MINB, Cf::WPB>;
    const size_t smem = (size_t)Cf::S * AdjStage<DIM, NT>::bytes(a.maxb);
    static size_t configured = 0;
    if (smem > configured) {
        const cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        configured = smem;
    }
    static size_t cap_smem = 0;
    static long long cap_blocks = 0;
    if (cap_blocks == 0 || cap_smem != smem) {
        int dev = 0, sms = 148, per_sm = 1;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, Cf::WPB * kWarp, smem);
        cap_blocks = (long long)sms * (per_sm > 0 ? per_sm : 1);
        cap_smem = smem;
    }
    const long long ntiles = ((long long)a.n + NT - 1) / NT;
    const int grid = (int)(ntiles < cap_blocks ? ntiles : cap_blocks);
    k<<<grid > 0 ? grid : 1, Cf::WPB * kWarp, smem, s>>>(a);
    return cudaGetLastError();
}

template <int DIM, bool MIXED>
static cudaError_t launch_adj_tma_w(const EpfAdjArgs &a, int which, cudaStream_t s) {
    switch (which) {
        case 1: return launch_adj_tma<DIM, MIXED, 1>(a, s);
        case 2: return launch_adj_tma<DIM, MIXED, 2>(a, s);
        default: return launch_adj_tma<DIM, MIXED, 0>(a, s);
    }
}

cudaError_t launch_epf_adjoint_tma(const EpfAdjArgs &a, int dim, bool mixed, int which, cudaStream_t s) {
    if (!a.SG || !a.GR || !a.hrev || a.maxb <= 0) return cudaErrorInvalidValue;
    if (dim == 3) return mixed ? launch_adj_tma_w<3, true>(a, which, s) : launch_adj_tma_w<3, false>(a, which, s);
    return mixed ? launch_adj_tma_w<2, true>(a, which, s) : launch_adj_tma_w<2, false>(a, which, s);
}

cudaError_t launch_epf_tma(const EpfArgs &a, int dim, bool mixed, int which, cudaStream_t s) {
    if (dim == 3) return mixed ? launch_tma_dm<3, true>(a, which, s) : launch_tma_dm<3, false>(a, which, s);
    return mixed ? launch_tma_dm<2, true>(a, which, s) : launch_tma_dm<2, false>(a, which, s);
}

}  // namespace pxb
