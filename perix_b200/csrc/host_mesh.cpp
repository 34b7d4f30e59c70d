// Host-side (C++20) mesh inputs of the hot path: structured PD lattice with mirror ghosts, family lists in
// the reference's visit order, initial-crack bond test and the CSR sparsity pattern.  These feed the
// device path when the library is driven standalone (bench, tests); a PeriX caller passes its own.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <limits>
#include <unordered_map>
#include <vector>

#include "pxb_context.h"

namespace {

// ---- structured lattice (reference src/PDMesh/CreatePDMesh.cpp:451-800 on the meshes of
//      src/Mesh/Lagrange2DQuad4MeshGenerator.cpp / Lagrange3DHex8MeshGenerator.cpp) ---------------------------
struct Lattice {
    int dim, nx, ny, nz;
    double x0, y0, z0, hx, hy, hz;
    // mesh-node coordinate along an axis (node index 1-based), as the generators compute it
    double nodex(int i) const { return x0 + (i - 1) * hx; }
    double nodey(int j) const { return y0 + (j - 1) * hy; }
    double nodez(int k) const { return z0 + (k - 1) * hz; }
};

// Average of a face's corner coordinates in the generator's corner order (sum from 0, then divide).
double avg(std::initializer_list<double> v) {
    double s = 0.0;
    for (double x : v) s += x;
    return s / static_cast<double>(v.size());
}

}  // namespace

extern "C" int pxb_lattice(int dim, int nx, int ny, int nz, const double *box, int *n_nodes, double *coords3,
                           double *vols, int *mirror, int *ghost_group, double *dxyz) {
    if ((dim != 2 && dim != 3) || nx < 1 || ny < 1 || (dim == 3 && nz < 1) || !box || !n_nodes)
        return pxb::fail(PXB_ERR_INVALID, "pxb_lattice: bad arguments");
    Lattice L{dim, nx, ny, dim == 3 ? nz : 0, box[0], box[2], dim == 3 ? box[4] : 0.0, 0, 0, 0};
    L.hx = (box[1] - box[0]) / nx;
    L.hy = (box[3] - box[2]) / ny;
    L.hz = dim == 3 ? (box[5] - box[4]) / nz : 0.0;
    const long long nbulk = (long long)nx * ny * (dim == 3 ? nz : 1);
    const long long nghost = (dim == 3) ? 2LL * ny * nz + 2LL * nx * nz + 2LL * nx * ny : 2LL * ny + 2LL * nx;
    if (nbulk + nghost > std::numeric_limits<int>::max()) return pxb::fail(PXB_ERR_INVALID, "pxb_lattice: too many nodes");
    *n_nodes = (int)(nbulk + nghost);
    // cell sizes from the first element, like createPDMesh (CreatePDMesh.cpp:495-506)
    const double DX = std::abs(L.nodex(2) - L.nodex(1));
    const double DY = std::abs(L.nodey(2) - L.nodey(1));
    const double DZ = dim == 3 ? std::abs(L.nodez(2) - L.nodez(1)) : 0.0;
    if (dxyz) { dxyz[0] = DX; dxyz[1] = DY; dxyz[2] = DZ; }
    if (!coords3) return PXB_OK;
    const double cellV = dim == 3 ? DX * DY * DZ : DX * DY;
    int id = 0;
    auto put = [&](double x, double y, double z, int mir, int grp) {
        coords3[3 * (size_t)id] = x;
        coords3[3 * (size_t)id + 1] = y;
        coords3[3 * (size_t)id + 2] = z;
        if (vols) vols[id] = cellV;
        if (mirror) mirror[id] = mir;
        if (ghost_group) ghost_group[id] = grp;
        ++id;
    };
    if (dim == 2) {
        // bulk cell centres, element e=(j-1)*nx+i: midpoint of corners 1 and 3
        for (int j = 1; j <= ny; ++j)
            for (int i = 1; i <= nx; ++i)
                put(0.5 * (L.nodex(i) + L.nodex(i + 1)), 0.5 * (L.nodey(j) + L.nodey(j + 1)), 0.0, 0, -1);
        auto eid = [&](int i, int j) { return (j - 1) * nx + i; };
        const double hxh = 0.5 * DX, hyh = 0.5 * DY;
        // left: edge (i4,i1) of element (1,j), ghost at -x
        for (int j = 1; j <= ny; ++j) {
            const double cx = avg({L.nodex(1), L.nodex(1)}), cy = avg({L.nodey(j + 1), L.nodey(j)});
            put(cx - hxh, cy, 0.0, eid(1, j), 0);
        }
        // right: edge (i2,i3) of element (nx,j)
        for (int j = 1; j <= ny; ++j) {
            const double cx = avg({L.nodex(nx + 1), L.nodex(nx + 1)}), cy = avg({L.nodey(j), L.nodey(j + 1)});
            put(cx + hxh, cy, 0.0, eid(nx, j), 1);
        }
        // bottom: edge (i1,i2) of element (i,1)
        for (int i = 1; i <= nx; ++i) {
            const double cx = avg({L.nodex(i), L.nodex(i + 1)}), cy = avg({L.nodey(1), L.nodey(1)});
            put(cx, cy - hyh, 0.0, eid(i, 1), 2);
        }
        // top: edge (i3,i4) of element (i,ny)
        for (int i = 1; i <= nx; ++i) {
            const double cx = avg({L.nodex(i + 1), L.nodex(i)}), cy = avg({L.nodey(ny + 1), L.nodey(ny + 1)});
            put(cx, cy + hyh, 0.0, eid(i, ny), 3);
        }
    } else {
        for (int k = 1; k <= nz; ++k)
            for (int j = 1; j <= ny; ++j)
                for (int i = 1; i <= nx; ++i)
                    put(0.5 * (L.nodex(i) + L.nodex(i + 1)), 0.5 * (L.nodey(j) + L.nodey(j + 1)),
                        0.5 * (L.nodez(k) + L.nodez(k + 1)), 0, -1);
        auto eid = [&](int i, int j, int k) { return (j - 1) * nx + i + (k - 1) * nx * ny; };
        const double hxh = 0.5 * DX, hyh = 0.5 * DY, hzh = 0.5 * DZ;
        // corner coordinates of element (i,j,k): corner c in {1..8} as in the hex8 generator
        auto cxy = [&](int i, int j, int k, int c, int axis) -> double {
            const int di = (c == 2 || c == 3 || c == 6 || c == 7) ? 1 : 0;
            const int dj = (c == 3 || c == 4 || c == 7 || c == 8) ? 1 : 0;
            const int dk = (c >= 5) ? 1 : 0;
            return axis == 0 ? L.nodex(i + di) : (axis == 1 ? L.nodey(j + dj) : L.nodez(k + dk));
        };
        auto face = [&](int i, int j, int k, const int (&c)[4], int axis) {
            return avg({cxy(i, j, k, c[0], axis), cxy(i, j, k, c[1], axis), cxy(i, j, k, c[2], axis),
                        cxy(i, j, k, c[3], axis)});
        };
        static const int fl[4] = {1, 5, 8, 4}, fr[4] = {2, 3, 7, 6}, fb[4] = {1, 2, 6, 5}, ft[4] = {4, 8, 7, 3},
                         fk[4] = {1, 4, 3, 2}, ff[4] = {5, 6, 7, 8};
        for (int k = 1; k <= nz; ++k)
            for (int j = 1; j <= ny; ++j)
                put(face(1, j, k, fl, 0) - hxh, face(1, j, k, fl, 1), face(1, j, k, fl, 2), eid(1, j, k), 0);
        for (int k = 1; k <= nz; ++k)
            for (int j = 1; j <= ny; ++j)
                put(face(nx, j, k, fr, 0) + hxh, face(nx, j, k, fr, 1), face(nx, j, k, fr, 2), eid(nx, j, k), 1);
        for (int k = 1; k <= nz; ++k)
            for (int i = 1; i <= nx; ++i)
                put(face(i, 1, k, fb, 0), face(i, 1, k, fb, 1) - hyh, face(i, 1, k, fb, 2), eid(i, 1, k), 2);
        for (int k = 1; k <= nz; ++k)
            for (int i = 1; i <= nx; ++i)
                put(face(i, ny, k, ft, 0), face(i, ny, k, ft, 1) + hyh, face(i, ny, k, ft, 2), eid(i, ny, k), 3);
        for (int j = 1; j <= ny; ++j)
            for (int i = 1; i <= nx; ++i)
                put(face(i, j, 1, fk, 0), face(i, j, 1, fk, 1), face(i, j, 1, fk, 2) - hzh, eid(i, j, 1), 4);
        for (int j = 1; j <= ny; ++j)
            for (int i = 1; i <= nx; ++i)
                put(face(i, j, nz, ff, 0), face(i, j, nz, ff, 1), face(i, j, nz, ff, 2) + hzh, eid(i, j, nz), 5);
    }
    return PXB_OK;
}

// ---- initial-crack bond test (reference src/PDMesh/PDMesh.cpp:19-159) ----------------------------------------
namespace {

int side2(double ux, double uy, double vx, double vy) {
    const double det = ux * vy - uy * vx;
    const double tol = 1.0e-12 * (std::fabs(ux) * std::fabs(vy) + std::fabs(uy) * std::fabs(vx));
    return det > tol ? 1 : (det < -tol ? -1 : 0);
}

int side_plane(const double *p, const double *c0, const double *nrm) {
    const double w[3] = {p[0] - c0[0], p[1] - c0[1], p[2] - c0[2]};
    const double d = w[0] * nrm[0] + w[1] * nrm[1] + w[2] * nrm[2];
    const double tol = 1.0e-12 * (std::fabs(w[0] * nrm[0]) + std::fabs(w[1] * nrm[1]) + std::fabs(w[2] * nrm[2]));
    return d > tol ? 1 : (d < -tol ? -1 : 0);
}

bool pierces(const double *A, const double *B, const double *q) {
    const double *c[4] = {q, q + 3, q + 6, q + 9};
    const double u[3] = {c[1][0] - c[0][0], c[1][1] - c[0][1], c[1][2] - c[0][2]};
    const double v[3] = {c[3][0] - c[0][0], c[3][1] - c[0][1], c[3][2] - c[0][2]};
    const double nrm[3] = {u[1] * v[2] - u[2] * v[1], u[2] * v[0] - u[0] * v[2], u[0] * v[1] - u[1] * v[0]};
    const double nl = std::sqrt(nrm[0] * nrm[0] + nrm[1] * nrm[1] + nrm[2] * nrm[2]);
    if (nl <= 0.0) return false;
    if (side_plane(A, c[0], nrm) * side_plane(B, c[0], nrm) >= 0) return false;
    const double dA = (A[0] - c[0][0]) * nrm[0] + (A[1] - c[0][1]) * nrm[1] + (A[2] - c[0][2]) * nrm[2];
    const double dB = (B[0] - c[0][0]) * nrm[0] + (B[1] - c[0][1]) * nrm[1] + (B[2] - c[0][2]) * nrm[2];
    const double s = dA / (dA - dB);
    const double Q[3] = {A[0] + s * (B[0] - A[0]), A[1] + s * (B[1] - A[1]), A[2] + s * (B[2] - A[2])};
    const double un[3] = {nrm[0] / nl, nrm[1] / nl, nrm[2] / nl};
    for (int k = 0; k < 4; ++k) {
        const double *p0 = c[k], *p1 = c[(k + 1) % 4];
        const double e[3] = {p1[0] - p0[0], p1[1] - p0[1], p1[2] - p0[2]};
        const double g[3] = {Q[0] - p0[0], Q[1] - p0[1], Q[2] - p0[2]};
        const double w[3] = {e[1] * g[2] - e[2] * g[1], e[2] * g[0] - e[0] * g[2], e[0] * g[1] - e[1] * g[0]};
        if (w[0] * un[0] + w[1] * un[1] + w[2] * un[2] <= 1.0e-9 * nl) return false;
    }
    return true;
}

struct CrackSet {
    int n;
    const double *x;
    const int *mirror;
    int ncr, npl;
    const double *cr, *pl;
    bool any() const { return ncr > 0 || npl > 0; }
    bool cuts(int i1, int j1) const {
        auto res = [&](int id) {
            if (mirror && id >= 1 && id <= n) {
                const int b = mirror[id - 1];
                if (b >= 1 && b <= n) return b;
            }
            return id;
        };
        const int a = res(i1), b = res(j1);
        if (a == b) return false;
        const double *A = x + 3 * (size_t)(a - 1), *B = x + 3 * (size_t)(b - 1);
        for (int c = 0; c < ncr; ++c) {
            const double *s = cr + 4 * c;
            if (side2(s[2] - s[0], s[3] - s[1], A[0] - s[0], A[1] - s[1]) *
                    side2(s[2] - s[0], s[3] - s[1], B[0] - s[0], B[1] - s[1]) >= 0)
                continue;
            if (side2(B[0] - A[0], B[1] - A[1], s[0] - A[0], s[1] - A[1]) *
                    side2(B[0] - A[0], B[1] - A[1], s[2] - A[0], s[3] - A[1]) < 0)
                return true;
        }
        for (int c = 0; c < npl; ++c)
            if (pierces(A, B, pl + 12 * c)) return true;
        return false;
    }
};

}  // namespace

// ---- families (reference src/PDMesh/CreatePDMesh.cpp:910-1082) ------------------------------------------------
// Cells of size `radius` are opened in node order; each cell pairs its own members (a<b) and then the
// members of the forward half of its neighbour cells (4 offsets in 2D, 13 in 3D); every accepted pair
// appends j to i and i to j.  This reproduces the reference family order exactly.  With per-node horizons
// (node_h, the reference's VariableHorizon) the cells take the largest horizon and a pair is kept when
// |x_i - x_j|^2 <= cut^2 (1 + 64 eps) with cut = max(delta_i, delta_j) (CreatePDMesh.cpp:932-938, 1043-1057).
static int families_impl(int n, const double *coords3, double radius, const double *node_h, int is3d, int ncracks,
                         const double *cracks, int nplanes, const double *planes, const int *mirror, int force_only,
                         int *neigh_off, int *neigh_id, long long *nbtot) {
    if (node_h) {
        radius = 0.0;
        for (int i = 0; i < n; ++i) radius = std::max(radius, node_h[i]);
    }
    if (n < 0 || !coords3 || !neigh_off || !(radius > 0.0)) return pxb::fail(PXB_ERR_INVALID, "pxb_families: bad arguments");
    neigh_off[0] = 0;
    if (n == 0) { if (nbtot) *nbtot = 0; return PXB_OK; }
    double lo[3] = {std::numeric_limits<double>::max(), std::numeric_limits<double>::max(),
                    std::numeric_limits<double>::max()};
    for (int i = 0; i < n; ++i)
        for (int a = 0; a < 3; ++a) lo[a] = std::min(lo[a], coords3[3 * (size_t)i + a]);
    if (!is3d) lo[2] = 0.0;
    struct Cell { long ix, iy, iz; std::vector<int> members; };
    std::vector<Cell> cells;
    std::unordered_map<uint64_t, int> index;
    index.reserve((size_t)n);
    auto key = [](long ix, long iy, long iz) -> uint64_t {
        const long b = 1L << 20;
        return ((uint64_t)(ix + b) << 42) | ((uint64_t)(iy + b) << 21) | (uint64_t)(iz + b);
    };
    for (int i = 0; i < n; ++i) {
        const double *p = coords3 + 3 * (size_t)i;
        const long ix = (int)std::floor((p[0] - lo[0]) / radius);
        const long iy = (int)std::floor((p[1] - lo[1]) / radius);
        const long iz = is3d ? (int)std::floor((p[2] - lo[2]) / radius) : 0;
        auto [it, fresh] = index.emplace(key(ix, iy, iz), (int)cells.size());
        if (fresh) cells.push_back(Cell{ix, iy, iz, {}});
        cells[(size_t)it->second].members.push_back(i);
    }
    static const int st2[4][3] = {{1, -1, 0}, {1, 0, 0}, {1, 1, 0}, {0, 1, 0}};
    static const int st3[13][3] = {{1, -1, -1}, {1, -1, 0}, {1, -1, 1}, {1, 0, -1}, {1, 0, 0}, {1, 0, 1}, {1, 1, -1},
                                   {1, 1, 0},   {1, 1, 1},  {0, 1, -1}, {0, 1, 0},  {0, 1, 1}, {0, 0, 1}};
    const CrackSet cs{n, coords3, mirror, ncracks, nplanes, cracks, planes};
    const bool cut = !force_only && cs.any();
    const double r2 = radius * radius;
    const double r2tol = 64.0 * std::numeric_limits<double>::epsilon() * r2;
    std::vector<int> cnt((size_t)n, 0);
    auto visit = [&](auto &&emit) {
        auto pair = [&](int i, int j) {
            const double *a = coords3 + 3 * (size_t)i, *b = coords3 + 3 * (size_t)j;
            const double dx = a[0] - b[0], dy = a[1] - b[1], dz = is3d ? (a[2] - b[2]) : 0.0;
            const double d2 = dx * dx + dy * dy + dz * dz;
            if (node_h) {
                const double cut = std::max(node_h[i], node_h[j]);
                const double cut2 = cut * cut;
                if (d2 > cut2 + 64.0 * std::numeric_limits<double>::epsilon() * cut2) return;
            } else if (!(d2 <= r2 + r2tol)) {
                return;
            }
            if (cut && cs.cuts(i + 1, j + 1)) return;
            emit(i, j);
        };
        for (const Cell &c : cells) {
            const auto &m = c.members;
            for (size_t a = 0; a < m.size(); ++a)
                for (size_t b = a + 1; b < m.size(); ++b) pair(m[a], m[b]);
            const int ns = is3d ? 13 : 4;
            for (int o = 0; o < ns; ++o) {
                const int *d = is3d ? st3[o] : st2[o];
                auto f = index.find(key(c.ix + d[0], c.iy + d[1], c.iz + d[2]));
                if (f == index.end()) continue;
                const auto &m2 = cells[(size_t)f->second].members;
                for (int i : m) for (int j : m2) pair(i, j);
            }
        }
    };
    visit([&](int i, int j) { ++cnt[(size_t)i]; ++cnt[(size_t)j]; });
    long long tot = 0;
    for (int i = 0; i < n; ++i) {
        tot += cnt[(size_t)i];
        if (tot > std::numeric_limits<int>::max()) return pxb::fail(PXB_ERR_INVALID, "pxb_families: more than 2^31-1 bonds");
        neigh_off[i + 1] = (int)tot;
    }
    if (nbtot) *nbtot = tot;
    if (!neigh_id) return PXB_OK;
    std::fill(cnt.begin(), cnt.end(), 0);
    visit([&](int i, int j) {
        neigh_id[neigh_off[i] + cnt[(size_t)i]++] = j + 1;
        neigh_id[neigh_off[j] + cnt[(size_t)j]++] = i + 1;
    });
    return PXB_OK;
}

extern "C" int pxb_families(int n, const double *coords3, double radius, int is3d, int ncracks,
                            const double *cracks, int nplanes, const double *planes, const int *mirror,
                            int force_only, int *neigh_off, int *neigh_id, long long *nbtot) {
    return families_impl(n, coords3, radius, nullptr, is3d, ncracks, cracks, nplanes, planes, mirror, force_only,
                         neigh_off, neigh_id, nbtot);
}

extern "C" int pxb_families_vh(int n, const double *coords3, const double *node_horizon, int is3d, int ncracks,
                               const double *cracks, int nplanes, const double *planes, const int *mirror,
                               int force_only, int *neigh_off, int *neigh_id, long long *nbtot) {
    if (!node_horizon) return pxb::fail(PXB_ERR_INVALID, "pxb_families_vh: node_horizon is NULL");
    return families_impl(n, coords3, 0.0, node_horizon, is3d, ncracks, cracks, nplanes, planes, mirror, force_only,
                         neigh_off, neigh_id, nbtot);
}

// Per-node horizon and spacing (reference PDMesh::computeVariableHorizon, src/PDMesh/CreatePDMesh.cpp:828-905):
// s_i = V_i^(1/dim); s_ref = the median (upper middle) of s_i over the bulk nodes with V_i > 0 (all such nodes when
// no bulk node has one); delta_i = horizon (s_i / s_ref) and spacing_i = dx_char (s_i / s_ref), or the global
// values where V_i <= 0.
extern "C" int pxb_variable_horizon(int n, int dim, const double *vols, const int *mirror, double horizon,
                                    double dx_char, double *node_delta, double *node_spacing) {
    if (n <= 0 || (dim != 2 && dim != 3) || !vols || !node_delta || !(horizon > 0.0))
        return pxb::fail(PXB_ERR_INVALID, "pxb_variable_horizon: bad arguments");
    const double inv_dim = dim == 3 ? (1.0 / 3.0) : 0.5;
    std::vector<double> s((size_t)n, 0.0), sb;
    for (int i = 0; i < n; ++i) s[(size_t)i] = vols[i] > 0.0 ? std::pow(vols[i], inv_dim) : 0.0;
    for (int i = 0; i < n; ++i)
        if ((!mirror || mirror[i] == 0) && s[(size_t)i] > 0.0) sb.push_back(s[(size_t)i]);
    if (sb.empty())
        for (int i = 0; i < n; ++i)
            if (s[(size_t)i] > 0.0) sb.push_back(s[(size_t)i]);
    if (sb.empty()) return pxb::fail(PXB_ERR_INVALID, "pxb_variable_horizon: no positive node volume");
    std::sort(sb.begin(), sb.end());
    const double s_ref = sb[sb.size() / 2];
    const double inv_ref = 1.0 / s_ref;
    for (int i = 0; i < n; ++i) {
        const double ratio = s[(size_t)i] > 0.0 ? s[(size_t)i] * inv_ref : 1.0;
        node_delta[i] = horizon * ratio;
        if (node_spacing) node_spacing[i] = dx_char * ratio;
    }
    return PXB_OK;
}

extern "C" int pxb_crack_cut_mask(int n, const double *coords3, const int *mirror, const int *neigh_off,
                                  const int *neigh_id, int ncracks, const double *cracks, int nplanes,
                                  const double *planes, uint8_t *out) {
    if (n < 0 || !coords3 || !neigh_off || !neigh_id || !out) return pxb::fail(PXB_ERR_INVALID, "pxb_crack_cut_mask: bad arguments");
    const CrackSet cs{n, coords3, mirror, ncracks, nplanes, cracks, planes};
    for (int i = 0; i < n; ++i)
        for (int t = neigh_off[i]; t < neigh_off[i + 1]; ++t) out[t] = cs.any() && cs.cuts(i + 1, neigh_id[t]) ? 1 : 0;
    return PXB_OK;
}

// ---- CSR pattern (reference src/MathUtils/SparseMatrix.cpp:73-185) --------------------------------------------
extern "C" int pxb_csr_pattern(int n, int ndof, const int *neigh_off, const int *neigh_id, const int *mirror,
                               int *rowptr, int *cols, long long *nnz) {
    if (n < 0 || ndof < 1 || !neigh_off || !neigh_id || !rowptr) return pxb::fail(PXB_ERR_INVALID, "pxb_csr_pattern: bad arguments");
    std::vector<int> nodes;
    long long acc = 0;
    rowptr[0] = 0;
    for (int i = 0; i < n; ++i) {
        nodes.assign(neigh_id + neigh_off[i], neigh_id + neigh_off[i + 1]);
        nodes.push_back(i + 1);
        if (mirror && mirror[i] >= 1 && mirror[i] <= n) nodes.push_back(mirror[i]);
        std::sort(nodes.begin(), nodes.end());
        nodes.erase(std::unique(nodes.begin(), nodes.end()), nodes.end());
        for (int a = 0; a < ndof; ++a) {
            if (cols)
                for (size_t k = 0; k < nodes.size(); ++k)
                    for (int b = 0; b < ndof; ++b) cols[acc + (long long)k * ndof + b] = (nodes[k] - 1) * ndof + b;
            acc += (long long)nodes.size() * ndof;
            if (acc > std::numeric_limits<int>::max()) return pxb::fail(PXB_ERR_INVALID, "pxb_csr_pattern: nnz exceeds 2^31-1");
            rowptr[(size_t)i * ndof + a + 1] = (int)acc;
        }
    }
    if (nnz) *nnz = acc;
    return PXB_OK;
}
