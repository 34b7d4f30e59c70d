// g-function build for callers that cannot allocate device memory.
//
// Some callers must not call cudaMalloc: an application whose device memory belongs to another allocator
// (a framework's caching pool, or a solver that reserves the whole GPU up front and hands out slices), or a
// time-stepping loop that cannot afford the implicit device synchronisation cudaMalloc/cudaFree may perform.
// pxb_gbuild_noalloc_d serves them: the caller passes every input and output as device memory it already
// owns, and the build's working memory (the packed node positions the kernel gathers from, the two
// degenerate-family counters and an input-check flag) lives in one file-scope __device__ array of fixed size,
// kNoallocScratchBytes (4 MiB), which every GPU that loads this library holds until the process exits.  The
// first call on a device looks up that array's device address (cudaGetSymbolAddress); make that first call
// before any stream capture begins.  All calls share the one array, so calls that overlap on the GPU
// (different streams or host threads at the same time) race on it and must be serialised by the caller.
#include <climits>
#include <cstdint>
#include <mutex>
#include <string>

#include "k_kernels.h"
#include "pxb_common.cuh"
#include "pxb_context.h"

namespace {

constexpr size_t kNoallocScratchBytes = 4u << 20;  // 4 MiB per device
constexpr size_t kCounterBytes = 256;              // n_degenerate (u32), first_degenerate (i32), input flag (u32)

__device__ __align__(256) unsigned char g_noalloc_scratch[kNoallocScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_setup_mutex;
void *g_scratch_addr[kMaxDevices] = {};

// Resolve the device address of the scratch array on the current device (once per device).  In host code
// `g_noalloc_scratch` is only a host-side stand-in for the symbol, so a kernel must be given this address.
int scratch_address(int device, void **out) {
    if (device < 0 || device >= kMaxDevices) return pxb::fail(PXB_ERR_INVALID, "pxb_gbuild_noalloc_d: device index too large");
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (!g_scratch_addr[device]) {
        void *p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return pxb::cuda_fail(e, "cudaGetSymbolAddress(g_noalloc_scratch)");
        g_scratch_addr[device] = p;
    }
    *out = g_scratch_addr[device];
    return PXB_OK;
}

// The caller's family CSR, checked on the device before the build reads through it: off[0] == 0, offsets
// non-decreasing, off[n] == nb, every id in [0, n).  A violation sets *bad (the build is then not launched), so a
// malformed list is reported instead of turning into reads outside the caller's buffers or the scratch array.
__global__ void noalloc_check_kernel(int n, long long nb, const int *off, const int *ids, unsigned int *bad) {
    const long long total = (long long)n + 1 > nb ? (long long)n + 1 : nb;
    unsigned int b = 0;
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < total;
         k += (long long)gridDim.x * blockDim.x) {
        if (k <= n) {
            const int o = off[k];
            if (k == 0 && o != 0) b = 1;
            if (k > 0 && o < off[k - 1]) b = 1;
            if (k == n && (long long)o != nb) b = 1;
        }
        if (k < nb) {
            const int j = ids[k];
            if (j < 0 || j >= n) b = 1;
        }
    }
    if (b) atomicOr(bad, 1u);
}

}  // namespace

extern "C" int pxb_gbuild_noalloc_max_nodes(int dim) {
    const size_t per_node = dim == 3 ? 32 : 16;
    return (int)((kNoallocScratchBytes - kCounterBytes) / per_node);
}

extern "C" int pxb_gbuild_noalloc_d(int dim, int order, int precision, int n, long long nbtot, const int *neigh_off_d,
                                    const int *neigh_id0_d, const double *coords3_d, const double *vols_d,
                                    const int *layer_d, double delta, double dx_char, void *ops_d, float *defect_d,
                                    uint8_t *degenerate_d, int *n_degenerate, int *first_degenerate, void *stream) {
    using namespace pxb;
    if ((dim != 2 && dim != 3) || n <= 0 || nbtot < 0 || !neigh_off_d || !neigh_id0_d || !coords3_d || !vols_d ||
        !ops_d || !(delta > 0.0) || (precision != PXB_FP64 && precision != PXB_MIXED))
        return fail(PXB_ERR_INVALID, "pxb_gbuild_noalloc_d: bad arguments");
    if (!gbuild_supported(dim, order) && !gbuild_warp_supported(dim, order))
        return fail(PXB_ERR_UNSUPPORTED, "pxb_gbuild_noalloc_d: order not built for this dimension");
    if (n > pxb_gbuild_noalloc_max_nodes(dim))
        return fail(PXB_ERR_INVALID, "pxb_gbuild_noalloc_d: " + std::to_string(n) + " nodes exceed the " +
                                         std::to_string(pxb_gbuild_noalloc_max_nodes(dim)) + "-node limit of the " +
                                         std::to_string(kNoallocScratchBytes >> 20) + " MiB scratch array (" +
                                         std::to_string(dim) + "D)");
    int device = 0;
    PXB_CUDA_TRY(cudaGetDevice(&device));
    void *base = nullptr;
    PXB_TRY(scratch_address(device, &base));
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    unsigned char *scr = static_cast<unsigned char *>(base);
    unsigned int *nd = reinterpret_cast<unsigned int *>(scr);
    int *first = reinterpret_cast<int *>(scr + 8);
    unsigned int *bad = reinterpret_cast<unsigned int *>(scr + 16);
    void *pos = scr + kCounterBytes;
    int sms = 148;
    PXB_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
    // the array keeps the previous call's contents: reset the counters (first_degenerate to 0x7f7f7f7f, above
    // any node index) and the input flag; the packed positions are fully rewritten below
    PXB_CUDA_TRY(cudaMemsetAsync(nd, 0, sizeof(unsigned int), s));
    PXB_CUDA_TRY(cudaMemsetAsync(first, 0x7f, sizeof(int), s));
    PXB_CUDA_TRY(cudaMemsetAsync(bad, 0, sizeof(unsigned int), s));
    noalloc_check_kernel<<<sms * 4, 256, 0, s>>>(n, nbtot, neigh_off_d, neigh_id0_d, bad);
    PXB_CUDA_TRY(cudaGetLastError());
    unsigned int hbad = 0;
    PXB_CUDA_TRY(cudaMemcpyAsync(&hbad, bad, sizeof(hbad), cudaMemcpyDeviceToHost, s));
    PXB_CUDA_TRY(cudaStreamSynchronize(s));
    if (hbad)
        return fail(PXB_ERR_INVALID, "pxb_gbuild_noalloc_d: malformed families (need neigh_off[0] == 0, "
                                     "non-decreasing offsets, neigh_off[n] == nbtot and 0-based ids in [0, n))");
    const bool with_defect = precision == PXB_MIXED && order == 2 && defect_d != nullptr;
    if (with_defect)
        PXB_CUDA_TRY(cudaMemsetAsync(defect_d, 0, sizeof(float) * (size_t)n * (size_t)((nop_of(dim, 2) - dim) * dim), s));
    PXB_CUDA_TRY(launch_pos_pack(n, dim, coords3_d, pos, s));
    GBuildArgs a;
    a.n = n;
    a.nb = nbtot;
    a.off = neigh_off_d;
    a.nbr = neigh_id0_d;
    a.pos = pos;
    a.vol = vols_d;
    a.layer = layer_d;
    a.delta = delta;
    a.dx_char = dx_char;
    a.ops = ops_d;
    a.degenerate = degenerate_d;
    a.n_degenerate = nd;
    a.first_degenerate = first;
    a.defect = with_defect ? defect_d : nullptr;
    // the schedule pxb_gbuild picks by default: one warp per node in 3D and above order 2, lane groups otherwise
    const bool warp = !gbuild_supported(dim, order) || dim == 3 || order > 2;
    if (warp) PXB_CUDA_TRY(launch_gbuild_warp(a, dim, order, precision == PXB_MIXED, false, s));
    else PXB_CUDA_TRY(launch_gbuild(a, dim, order, precision == PXB_MIXED, sms * 16, s));
    unsigned int hnd = 0;
    int hfirst = 0;
    PXB_CUDA_TRY(cudaMemcpyAsync(&hnd, nd, sizeof(hnd), cudaMemcpyDeviceToHost, s));
    PXB_CUDA_TRY(cudaMemcpyAsync(&hfirst, first, sizeof(hfirst), cudaMemcpyDeviceToHost, s));
    PXB_CUDA_TRY(cudaStreamSynchronize(s));
    if (n_degenerate) *n_degenerate = (int)hnd;
    if (first_degenerate) *first_degenerate = hnd ? hfirst + 1 : 0;
    if (hnd)
        return fail(PXB_ERR_DEGENERATE, "degenerate moment matrix at node " + std::to_string(hfirst + 1) + " (" +
                                            std::to_string(hnd) + " non-ghost node(s))");
    return PXB_OK;
}
