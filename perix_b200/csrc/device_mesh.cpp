// Host side of the device family build (see k_families.cu and fam_builder.h).
#include <algorithm>
#include <limits>
#include <string>
#include <vector>

#include "fam_builder.h"

namespace pxb {

int FamBuilder::count(pxb_ctx *c, int n, bool is3d, const double *coords_host, double radius, std::vector<int> &hoff,
                      int &maxf, long long &tot) {
    FamArgs &a = a_;
    a = FamArgs{};
    a.n = n;
    a.is3d = is3d ? 1 : 0;
    for (int d = 0; d < 3; ++d) a.lo[d] = std::numeric_limits<double>::max();
    for (int i = 0; i < n; ++i)
        for (int d = 0; d < 3; ++d) a.lo[d] = std::min(a.lo[d], coords_host[3 * (size_t)i + d]);
    if (!is3d) a.lo[2] = 0.0;
    a.radius = radius;
    a.r2 = radius * radius;
    a.r2tol = 64.0 * std::numeric_limits<double>::epsilon() * a.r2;
    unsigned slots = 1024;
    while (slots < 2u * (unsigned)n && slots < (1u << 31)) slots <<= 1;
    a.mask = slots - 1;
    cudaStream_t s = c->stream;
    PXB_TRY(dev_upload(c, coords_, coords_host, sizeof(double) * 3 * (size_t)n));
    PXB_TRY(dev_alloc(c, keys_, sizeof(unsigned long long) * slots));
    PXB_CUDA_TRY(cudaMemsetAsync(keys_.p, 0xff, keys_.bytes, s));
    PXB_TRY(dev_alloc(c, ccount_, sizeof(int) * slots));
    PXB_CUDA_TRY(cudaMemsetAsync(ccount_.p, 0, ccount_.bytes, s));
    PXB_TRY(dev_alloc(c, cminid_, sizeof(int) * slots));
    PXB_CUDA_TRY(cudaMemsetAsync(cminid_.p, 0x7f, cminid_.bytes, s));
    PXB_TRY(dev_alloc(c, cfill_, sizeof(int) * slots));
    PXB_CUDA_TRY(cudaMemsetAsync(cfill_.p, 0, cfill_.bytes, s));
    PXB_TRY(dev_alloc(c, cstart_, sizeof(int) * slots));
    PXB_TRY(dev_alloc(c, members_, sizeof(int) * (size_t)n));
    PXB_TRY(dev_alloc(c, cell_of_, sizeof(int) * (size_t)n));
    PXB_TRY(dev_alloc(c, cxyz_, sizeof(int) * 3 * (size_t)n));
    PXB_TRY(dev_alloc(c, pos_, sizeof(int) * (size_t)n));
    PXB_TRY(dev_alloc(c, fcount_, sizeof(int) * (size_t)n));
    PXB_TRY(dev_alloc(c, err_, sizeof(int)));
    PXB_CUDA_TRY(cudaMemsetAsync(err_.p, 0, sizeof(int), s));
    a.coords = coords_.as<double>();
    a.keys = keys_.as<unsigned long long>();
    a.ccount = ccount_.as<int>();
    a.cminid = cminid_.as<int>();
    a.cstart = cstart_.as<int>();
    a.cfill = cfill_.as<int>();
    a.members = members_.as<int>();
    a.cell_of = cell_of_.as<int>();
    a.cxyz = cxyz_.as<int>();
    a.pos = pos_.as<int>();
    a.fcount = fcount_.as<int>();
    a.err = err_.as<int>();
    PXB_CUDA_TRY(launch_fam_cells(a, s));
    int herr = 0;
    std::vector<int> hcount(slots), hstart(slots);
    PXB_TRY(d2h(c, &herr, err_.p, sizeof(int)));
    PXB_TRY(d2h(c, hcount.data(), ccount_.p, sizeof(int) * slots));
    PXB_TRY(sync(c));
    if (herr) return fail(PXB_ERR_INVALID, "device families: cell index out of range or cell table full");
    long long acc = 0;
    int maxcell = 0;
    for (unsigned k = 0; k < slots; ++k) {
        hstart[k] = (int)acc;
        acc += hcount[k];
        maxcell = std::max(maxcell, hcount[k]);
    }
    if (maxcell >= kFamCell)
        return fail(PXB_ERR_UNSUPPORTED, "device families: more than " + std::to_string(kFamCell - 1) +
                                             " nodes in one cell of size radius (use pxb_families on the host)");
    PXB_TRY(h2d(c, cstart_.p, hstart.data(), sizeof(int) * slots));
    PXB_CUDA_TRY(launch_fam_members(a, s));
    PXB_CUDA_TRY(launch_fam_sort_cells(a, s));
    PXB_CUDA_TRY(launch_fam_candidates(a, false, s));
    std::vector<int> hfc((size_t)n);
    PXB_TRY(d2h(c, hfc.data(), fcount_.p, sizeof(int) * (size_t)n));
    PXB_TRY(sync(c));
    hoff.assign((size_t)n + 1, 0);
    tot = 0;
    maxf = 0;
    for (int i = 0; i < n; ++i) {
        tot += hfc[(size_t)i];
        if (tot > std::numeric_limits<int>::max()) return fail(PXB_ERR_INVALID, "device families: more than 2^31-1 bonds");
        hoff[(size_t)i + 1] = (int)tot;
        maxf = std::max(maxf, hfc[(size_t)i]);
    }
    if (maxf > kFamMax)
        return fail(PXB_ERR_UNSUPPORTED, "device families: a family exceeds " + std::to_string(kFamMax) +
                                             " members (use pxb_families on the host)");
    return PXB_OK;
}

int FamBuilder::fill(pxb_ctx *c, const int *off_d, int *nbr_d, int id_base) {
    FamArgs &a = a_;
    int first = 0, last = 0;
    PXB_TRY(d2h(c, &first, off_d, sizeof(int)));
    PXB_TRY(d2h(c, &last, off_d + a.n, sizeof(int)));
    PXB_TRY(sync(c));
    const long long tot = (long long)last - first;
    PXB_TRY(dev_alloc(c, fkey_, sizeof(unsigned long long) * (size_t)std::max(1LL, tot)));
    PXB_TRY(dev_alloc(c, fval_, sizeof(int) * (size_t)std::max(1LL, tot)));
    a.off = off_d;
    a.off_base = first;
    a.fkey = fkey_.as<unsigned long long>();
    a.fval = fval_.as<int>();
    a.nbr = nbr_d;
    a.id_base = id_base;
    PXB_CUDA_TRY(launch_fam_candidates(a, true, c->stream));
    PXB_CUDA_TRY(launch_fam_sort(a, c->stream));
    return check_launch(c, "device families");
}

}  // namespace pxb
