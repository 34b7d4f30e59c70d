// Device family build (k_families.cu) in two phases, shared by pxb_set_geometry_points and pxb_batch_set_points.
#pragma once

#include <vector>

#include "k_kernels.h"
#include "pxb_context.h"

namespace pxb {

// count(): cells, members, candidate counts -> host offsets hoff[n+1], largest family, bond total.
// fill(): keyed candidates and the per-family sort, written 0-based (+ id_base) at nbr_d[off_d[x] + k].
// The device temporaries live until the builder is destroyed; fill() needs the count() of the same builder.
class FamBuilder {
public:
    int count(pxb_ctx *c, int n, bool is3d, const double *coords_host, double radius, std::vector<int> &hoff,
              int &maxf, long long &tot);
    int fill(pxb_ctx *c, const int *off_d, int *nbr_d, int id_base);
    const double *coords_d() const { return coords_.as<double>(); }

private:
    FamArgs a_;
    DevBuf coords_, keys_, ccount_, cminid_, cstart_, cfill_, members_, cell_of_, cxyz_, pos_, fcount_, fkey_, fval_, err_;
};

}  // namespace pxb
