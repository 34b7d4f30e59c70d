/* Test infrastructure only (the oracle): a plain-C CPU restatement of PeriX's PDDO hot path.
 * Used by tests/, the smoke check and bench.py's cpu_baseline leg as the checker; the product never links
 * it.  Pinned against the reference's own code (oracle/_ref/libperix_ref.so) and the committed golden
 * fixtures under tests/golden/.  Reference citations are file:line within the PeriX project. */
#define _GNU_SOURCE
#include "pddo_oracle.h"

#include <float.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif
#define ORC_MAX_NOP 32

/* ---- multi-index table: PDOperators.cpp:51-75 (order ascending, p descending, q descending) ---------- */
static int fact_i(int n) {
    int r = 1;
    for (int k = 2; k <= n; ++k) r *= k;
    return r;
}

int orc_qindices(int dim, int order, int *pqr, int *fact) {
    int nop = 0;
    for (int o = 1; o <= order; ++o) {
        if (dim == 3) {
            for (int p = o; p >= 0; --p)
                for (int q = o - p; q >= 0; --q) {
                    if (pqr) { pqr[3 * nop] = p; pqr[3 * nop + 1] = q; pqr[3 * nop + 2] = o - p - q; }
                    if (fact) fact[nop] = fact_i(p) * fact_i(q) * fact_i(o - p - q);
                    ++nop;
                }
        } else {
            for (int p = o; p >= 0; --p) {
                if (pqr) { pqr[3 * nop] = p; pqr[3 * nop + 1] = o - p; pqr[3 * nop + 2] = 0; }
                if (fact) fact[nop] = fact_i(p) * fact_i(o - p);
                ++nop;
            }
        }
    }
    return nop;
}

/* ---- initial-crack test: PDMesh.cpp:19-159 ------------------------------------------------------------ */
static int orient_side(double ux, double uy, double vx, double vy) {
    const double det = ux * vy - uy * vx;
    const double scale = fabs(ux) * fabs(vy) + fabs(uy) * fabs(vx);
    if (det > 1.0e-12 * scale) return 1;
    if (det < -1.0e-12 * scale) return -1;
    return 0;
}

static int plane_side(double px, double py, double pz, double c0x, double c0y, double c0z, double nx, double ny,
                      double nz) {
    const double wx = px - c0x, wy = py - c0y, wz = pz - c0z;
    const double d = wx * nx + wy * ny + wz * nz;
    const double scale = fabs(wx * nx) + fabs(wy * ny) + fabs(wz * nz);
    if (d > 1.0e-12 * scale) return 1;
    if (d < -1.0e-12 * scale) return -1;
    return 0;
}

static int bond_pierces_quad(double ax, double ay, double az, double bx, double by, double bz, const double *q) {
    const double cx[4] = {q[0], q[3], q[6], q[9]};
    const double cy[4] = {q[1], q[4], q[7], q[10]};
    const double cz[4] = {q[2], q[5], q[8], q[11]};
    const double ux = cx[1] - cx[0], uy = cy[1] - cy[0], uz = cz[1] - cz[0];
    const double vx = cx[3] - cx[0], vy = cy[3] - cy[0], vz = cz[3] - cz[0];
    const double nx = uy * vz - uz * vy, ny = uz * vx - ux * vz, nz = ux * vy - uy * vx;
    const double nlen = sqrt(nx * nx + ny * ny + nz * nz);
    if (nlen <= 0.0) return 0;
    const int sA = plane_side(ax, ay, az, cx[0], cy[0], cz[0], nx, ny, nz);
    const int sB = plane_side(bx, by, bz, cx[0], cy[0], cz[0], nx, ny, nz);
    if (sA * sB >= 0) return 0;
    const double dA = (ax - cx[0]) * nx + (ay - cy[0]) * ny + (az - cz[0]) * nz;
    const double dB = (bx - cx[0]) * nx + (by - cy[0]) * ny + (bz - cz[0]) * nz;
    const double t = dA / (dA - dB);
    const double Qx = ax + t * (bx - ax), Qy = ay + t * (by - ay), Qz = az + t * (bz - az);
    const double unx = nx / nlen, uny = ny / nlen, unz = nz / nlen;
    const double tol = 1.0e-9 * nlen;
    for (int k = 0; k < 4; k++) {
        const int m = (k + 1) % 4;
        const double ex = cx[m] - cx[k], ey = cy[m] - cy[k], ez = cz[m] - cz[k];
        const double gx = Qx - cx[k], gy = Qy - cy[k], gz = Qz - cz[k];
        const double wx = ey * gz - ez * gy, wy = ez * gx - ex * gz, wz = ex * gy - ey * gx;
        if (wx * unx + wy * uny + wz * unz <= tol) return 0;
    }
    return 1;
}

int orc_crack_cuts(int n, const double *coords3, const int *mirror, int ncracks, const double *cracks, int nplanes,
                   const double *planes, int i1, int j1) {
    if (ncracks <= 0 && nplanes <= 0) return 0;
    int a = i1, b = j1;
    if (mirror) {
        if (i1 >= 1 && i1 <= n && mirror[i1 - 1] >= 1 && mirror[i1 - 1] <= n) a = mirror[i1 - 1];
        if (j1 >= 1 && j1 <= n && mirror[j1 - 1] >= 1 && mirror[j1 - 1] <= n) b = mirror[j1 - 1];
    }
    if (a == b) return 0;
    const double ax = coords3[3 * (a - 1)], ay = coords3[3 * (a - 1) + 1], az = coords3[3 * (a - 1) + 2];
    const double bx = coords3[3 * (b - 1)], by = coords3[3 * (b - 1) + 1], bz = coords3[3 * (b - 1) + 2];
    for (int c = 0; c < ncracks; ++c) {
        const double cx = cracks[4 * c], cy = cracks[4 * c + 1], dx = cracks[4 * c + 2], dy = cracks[4 * c + 3];
        const int s1 = orient_side(dx - cx, dy - cy, ax - cx, ay - cy);
        const int s2 = orient_side(dx - cx, dy - cy, bx - cx, by - cy);
        if (s1 * s2 >= 0) continue;
        const int s3 = orient_side(bx - ax, by - ay, cx - ax, cy - ay);
        const int s4 = orient_side(bx - ax, by - ay, dx - ax, dy - ay);
        if (s3 * s4 < 0) return 1;
    }
    for (int c = 0; c < nplanes; ++c)
        if (bond_pierces_quad(ax, ay, az, bx, by, bz, planes + 12 * c)) return 1;
    return 0;
}

/* ---- families: CreatePDMesh.cpp:910-1082 ----------------------------------------------------------------
 * Buckets are created in node-id order (:987-995); each bucket visits its intra pairs (a<b, insertion
 * order) and then the forward half-stencil (:1001-1010, :1059-1082); tryAddPair pushes j to i and i to j
 * (:1018-1057).  A small open-addressing table stands in for the unordered_map: only key->bucket lookup
 * matters for the visit order, never the hash order. */
typedef struct {
    uint64_t *keys;
    int *vals;
    size_t cap;
} orc_map;

static uint64_t mix64(uint64_t x) {
    x ^= x >> 33; x *= 0xff51afd7ed558ccdULL; x ^= x >> 33; x *= 0xc4ceb9fe1a85ec53ULL; x ^= x >> 33;
    return x;
}

static int map_find(const orc_map *m, uint64_t key) {
    size_t h = mix64(key) & (m->cap - 1);
    while (m->vals[h] >= 0) {
        if (m->keys[h] == key) return m->vals[h];
        h = (h + 1) & (m->cap - 1);
    }
    return -1;
}

static int map_insert(orc_map *m, uint64_t key, int val) {
    size_t h = mix64(key) & (m->cap - 1);
    while (m->vals[h] >= 0) {
        if (m->keys[h] == key) return m->vals[h];
        h = (h + 1) & (m->cap - 1);
    }
    m->keys[h] = key;
    m->vals[h] = val;
    return -1;
}

static uint64_t encode_cell(long ix, long iy, long iz) {
    const long bias = 1L << 20;
    return ((uint64_t)(ix + bias) << 42) | ((uint64_t)(iy + bias) << 21) | (uint64_t)(iz + bias);
}

typedef struct {
    int n, is3d, ncr, npl, cut, fill;
    const double *x, *cr, *pl;
    const int *mirror;
    double r2, r2tol;
    int *cnt, *ids;
    const int *off;
} orc_fam_ctx;

static void try_add_pair(orc_fam_ctx *c, int i, int j) {
    const double *xi = c->x + 3 * (size_t)i, *xj = c->x + 3 * (size_t)j;
    const double dx = xi[0] - xj[0], dy = xi[1] - xj[1], dz = c->is3d ? (xi[2] - xj[2]) : 0.0;
    const double d2 = dx * dx + dy * dy + dz * dz;
    if (!(d2 <= c->r2 + c->r2tol)) return;
    if (c->cut && orc_crack_cuts(c->n, c->x, c->mirror, c->ncr, c->cr, c->npl, c->pl, i + 1, j + 1)) return;
    if (c->fill) {
        c->ids[c->off[i] + c->cnt[i]] = j + 1;
        c->ids[c->off[j] + c->cnt[j]] = i + 1;
    }
    c->cnt[i]++;
    c->cnt[j]++;
}

long long orc_families(int n, const double *coords3, double radius, int is3d, int ncracks, const double *cracks,
                       int nplanes, const double *planes, const int *mirror, int force_only, int *off, int *ids) {
    if (n <= 0) { off[0] = 0; return 0; }
    double minx = DBL_MAX, miny = DBL_MAX, minz = DBL_MAX;
    for (int i = 0; i < n; ++i) {
        if (coords3[3 * i] < minx) minx = coords3[3 * i];
        if (coords3[3 * i + 1] < miny) miny = coords3[3 * i + 1];
        if (coords3[3 * i + 2] < minz) minz = coords3[3 * i + 2];
    }
    if (!is3d) minz = 0.0;
    const double cs = radius;
    long *cell = (long *)malloc(sizeof(long) * 3 * (size_t)n);
    int *bucket_of = (int *)malloc(sizeof(int) * (size_t)n);
    orc_map map;
    map.cap = 16;
    while (map.cap < 2 * (size_t)n + 16) map.cap <<= 1;
    map.keys = (uint64_t *)malloc(sizeof(uint64_t) * map.cap);
    map.vals = (int *)malloc(sizeof(int) * map.cap);
    for (size_t h = 0; h < map.cap; ++h) map.vals[h] = -1;
    int nb = 0;
    for (int i = 0; i < n; ++i) {
        cell[3 * i] = (long)(int)floor((coords3[3 * i] - minx) / cs);
        cell[3 * i + 1] = (long)(int)floor((coords3[3 * i + 1] - miny) / cs);
        cell[3 * i + 2] = is3d ? (long)(int)floor((coords3[3 * i + 2] - minz) / cs) : 0;
        const uint64_t key = encode_cell(cell[3 * i], cell[3 * i + 1], cell[3 * i + 2]);
        const int found = map_insert(&map, key, nb);
        bucket_of[i] = (found >= 0) ? found : nb++;
    }
    /* bucket member lists in node order */
    int *bstart = (int *)calloc((size_t)nb + 1, sizeof(int));
    int *bnodes = (int *)malloc(sizeof(int) * (size_t)n);
    long *bcell = (long *)malloc(sizeof(long) * 3 * (size_t)nb);
    for (int i = 0; i < n; ++i) bstart[bucket_of[i] + 1]++;
    for (int b = 0; b < nb; ++b) bstart[b + 1] += bstart[b];
    int *bfill = (int *)calloc((size_t)nb, sizeof(int));
    for (int i = 0; i < n; ++i) {
        const int b = bucket_of[i];
        if (bfill[b] == 0) { bcell[3 * b] = cell[3 * i]; bcell[3 * b + 1] = cell[3 * i + 1]; bcell[3 * b + 2] = cell[3 * i + 2]; }
        bnodes[bstart[b] + bfill[b]++] = i;
    }
    static const int st2[4][3] = {{1, -1, 0}, {1, 0, 0}, {1, 1, 0}, {0, 1, 0}};
    static const int st3[13][3] = {{1, -1, -1}, {1, -1, 0}, {1, -1, 1}, {1, 0, -1}, {1, 0, 0}, {1, 0, 1}, {1, 1, -1},
                                   {1, 1, 0},   {1, 1, 1},  {0, 1, -1}, {0, 1, 0},  {0, 1, 1}, {0, 0, 1}};
    orc_fam_ctx c;
    c.n = n; c.is3d = is3d; c.ncr = ncracks; c.npl = nplanes; c.cr = cracks; c.pl = planes; c.x = coords3;
    c.mirror = mirror;
    c.cut = (!force_only) && (ncracks > 0 || nplanes > 0);
    c.r2 = radius * radius;
    c.r2tol = 64.0 * DBL_EPSILON * c.r2;
    c.cnt = (int *)calloc((size_t)n, sizeof(int));
    c.ids = ids;
    c.off = off;
    for (int pass = 0; pass < (ids ? 2 : 1); ++pass) {
        c.fill = pass == 1;
        if (pass == 1) memset(c.cnt, 0, sizeof(int) * (size_t)n);
        for (int b = 0; b < nb; ++b) {
            const int s = bstart[b], e = bstart[b + 1];
            for (int a = s; a < e; ++a)
                for (int q = a + 1; q < e; ++q) try_add_pair(&c, bnodes[a], bnodes[q]);
            const int ns = is3d ? 13 : 4;
            for (int o = 0; o < ns; ++o) {
                const int *d = is3d ? st3[o] : st2[o];
                const int nbk = map_find(&map, encode_cell(bcell[3 * b] + d[0], bcell[3 * b + 1] + d[1], bcell[3 * b + 2] + d[2]));
                if (nbk < 0) continue;
                for (int a = s; a < e; ++a)
                    for (int q = bstart[nbk]; q < bstart[nbk + 1]; ++q) try_add_pair(&c, bnodes[a], bnodes[q]);
            }
        }
        if (pass == 0) {
            off[0] = 0;
            for (int i = 0; i < n; ++i) off[i + 1] = off[i] + c.cnt[i];
        }
    }
    const long long total = off[n];
    free(cell); free(bucket_of); free(map.keys); free(map.vals); free(bstart); free(bnodes); free(bcell);
    free(bfill); free(c.cnt);
    return total;
}

/* ---- g-functions: CalcPDOperators.cpp:48-60 (weight, vc), 108-226 (moment + solve), 307-354 (ops) ----- */
static double orc_weight(double xn, double delta) {
    const double r = 2.0 * xn / delta;
    return exp(-r * r);
}

static double orc_vc(double xn, double delta, double dxc) {
    if (dxc <= 0.0) return 1.0;
    if (xn <= delta - 0.5 * dxc) return 1.0;
    double v = (delta - xn + 0.5 * dxc) / dxc;
    if (v < 0.0) v = 0.0;
    if (v > 1.0) v = 1.0;
    return v;
}

static void orc_monomials(int nop, const int *pqr, double ex, double ey, double ez, double *m) {
    for (int k = 0; k < nop; ++k) {
        double v = 1.0;
        for (int t = 0; t < pqr[3 * k]; ++t) v *= ex;
        for (int t = 0; t < pqr[3 * k + 1]; ++t) v *= ey;
        for (int t = 0; t < pqr[3 * k + 2]; ++t) v *= ez;
        m[k] = v;
    }
}

/* Complete-pivoting LU solve of A X = B (n x n, row-major, B diagonal given as diag[]), the published
 * algorithm behind the reference's Eigen FullPivLU call (MatrixXd.cpp:26-48): pivots below
 * eps*n*|max pivot| are treated as zero (rank-deficient particular solution with free unknowns 0), then
 * the max-norm consistency test of MatrixXd.cpp:40-47 with relTol.  Returns 1 when consistent. */
static int orc_fullpiv_solve(int n, const double *A0, const double *diag, double *X, double relTol) {
    double LU[ORC_MAX_NOP * ORC_MAX_NOP];
    int rp[ORC_MAX_NOP], cp[ORC_MAX_NOP];
    memcpy(LU, A0, sizeof(double) * n * n);
    for (int i = 0; i < n; ++i) { rp[i] = i; cp[i] = i; }
    double maxpiv = 0.0;
    int nz = n;
    for (int k = 0; k < n; ++k) {
        int br = k, bc = k;
        double big = 0.0;
        for (int c = k; c < n; ++c)
            for (int r = k; r < n; ++r) {
                const double v = fabs(LU[r * n + c]);
                if (v > big) { big = v; br = r; bc = c; }
            }
        if (big == 0.0) { nz = k; break; }
        if (big > maxpiv) maxpiv = big;
        if (br != k) {
            for (int c = 0; c < n; ++c) { double t = LU[k * n + c]; LU[k * n + c] = LU[br * n + c]; LU[br * n + c] = t; }
            int t = rp[k]; rp[k] = rp[br]; rp[br] = t;
        }
        if (bc != k) {
            for (int r = 0; r < n; ++r) { double t = LU[r * n + k]; LU[r * n + k] = LU[r * n + bc]; LU[r * n + bc] = t; }
            int t = cp[k]; cp[k] = cp[bc]; cp[bc] = t;
        }
        const double p = LU[k * n + k];
        for (int r = k + 1; r < n; ++r) {
            LU[r * n + k] /= p;
            const double f = LU[r * n + k];
            for (int c = k + 1; c < n; ++c) LU[r * n + c] -= f * LU[k * n + c];
        }
    }
    int rank = 0;
    const double thr = DBL_EPSILON * n * maxpiv;
    for (int k = 0; k < nz; ++k)
        if (fabs(LU[k * n + k]) > thr) ++rank;
    for (int col = 0; col < n; ++col) {
        double y[ORC_MAX_NOP], z[ORC_MAX_NOP];
        for (int i = 0; i < n; ++i) y[i] = (rp[i] == col) ? diag[col] : 0.0; /* P*B */
        for (int i = 0; i < n; ++i)
            for (int j = 0; j < i; ++j) y[i] -= LU[i * n + j] * y[j];
        for (int i = n - 1; i >= 0; --i) {
            if (i >= rank) { z[i] = 0.0; continue; }
            double s = y[i];
            for (int j = i + 1; j < rank; ++j) s -= LU[i * n + j] * z[j];
            z[i] = s / LU[i * n + i];
        }
        for (int i = 0; i < n; ++i) X[cp[i] * n + col] = z[i];
    }
    double resid = 0.0, maxB = 0.0, maxA = 0.0, maxX = 0.0;
    for (int r = 0; r < n; ++r)
        for (int c = 0; c < n; ++c) {
            double s = 0.0;
            for (int k = 0; k < n; ++k) s += A0[r * n + k] * X[k * n + c];
            const double e = fabs(s - (r == c ? diag[r] : 0.0));
            if (e > resid) resid = e;
            if (fabs(A0[r * n + c]) > maxA) maxA = fabs(A0[r * n + c]);
            if (fabs(X[r * n + c]) > maxX) maxX = fabs(X[r * n + c]);
        }
    for (int r = 0; r < n; ++r) if (fabs(diag[r]) > maxB) maxB = fabs(diag[r]);
    double scale = maxB > maxA * maxX ? maxB : maxA * maxX;
    if (scale < DBL_MIN) scale = DBL_MIN;
    return resid <= relTol * scale;
}

int orc_gbuild(int n, int dim, int order, const double *coords3, const double *vols, const int *off,
               const int *ids, double delta, double dx_char, int volume_correction, double *ops,
               unsigned char *degenerate) {
    int pqr[3 * ORC_MAX_NOP], fct[ORC_MAX_NOP];
    const int nop = orc_qindices(dim, order, pqr, fct);
    if (nop > ORC_MAX_NOP) return -1;
    const double inv_delta = 1.0 / delta;
    double idpow[ORC_MAX_NOP], diag[ORC_MAX_NOP];
    for (int k = 0; k < nop; ++k) {
        double v = 1.0;
        const int tot = pqr[3 * k] + pqr[3 * k + 1] + pqr[3 * k + 2];
        for (int t = 0; t < tot; ++t) v *= inv_delta;
        idpow[k] = v;
        diag[k] = (double)fct[k];
    }
    int ndeg = 0;
#pragma omp parallel for schedule(guided) reduction(+ : ndeg)
    for (int i = 0; i < n; ++i) {
        double A[ORC_MAX_NOP * ORC_MAX_NOP], X[ORC_MAX_NOP * ORC_MAX_NOP], m[ORC_MAX_NOP];
        memset(A, 0, sizeof(double) * nop * nop);
        const double x1 = coords3[3 * i], y1 = coords3[3 * i + 1], z1 = coords3[3 * i + 2];
        int usable = 0;
        for (int t = off[i]; t < off[i + 1]; ++t) {
            const int j = ids[t] - 1;
            const double xx = coords3[3 * j] - x1, xy = coords3[3 * j + 1] - y1, xz = coords3[3 * j + 2] - z1;
            const double xn = sqrt(xx * xx + xy * xy + xz * xz);
            if (xn <= 0.0) continue;
            const double w = orc_weight(xn, delta);
            const double vc = volume_correction ? orc_vc(xn, delta, dx_char) : 1.0;
            const double bw = w * vc * vols[j];
            if (bw <= 0.0) continue;
            ++usable;
            orc_monomials(nop, pqr, xx * inv_delta, xy * inv_delta, xz * inv_delta, m);
            for (int a = 0; a < nop; ++a)
                for (int b = 0; b < nop; ++b) A[a * nop + b] += bw * m[a] * m[b];
        }
        const int consistent = orc_fullpiv_solve(nop, A, diag, X, 1.0e-8);
        const int deg = (usable < nop) || !consistent;
        if (degenerate) degenerate[i] = (unsigned char)deg;
        ndeg += deg;
        for (int t = off[i]; t < off[i + 1]; ++t) {
            const int j = ids[t] - 1;
            double *o = ops + (size_t)t * nop;
            const double xx = coords3[3 * j] - x1, xy = coords3[3 * j + 1] - y1, xz = coords3[3 * j + 2] - z1;
            const double xn = sqrt(xx * xx + xy * xy + xz * xz);
            for (int k = 0; k < nop; ++k) o[k] = 0.0;
            if (xn <= 0.0) continue;
            const double w = orc_weight(xn, delta);
            const double vc = volume_correction ? orc_vc(xn, delta, dx_char) : 1.0;
            const double bw = w * vc * vols[j];
            if (bw <= 0.0) continue;
            orc_monomials(nop, pqr, xx * inv_delta, xy * inv_delta, xz * inv_delta, m);
            for (int k = 0; k < nop; ++k) {
                double s = 0.0;
                for (int a = 0; a < nop; ++a) s += X[a * nop + k] * m[a];
                o[k] = s * bw * idpow[k];
            }
        }
    }
    return ndeg;
}

void orc_apply(int n, int nop, const int *off, const int *ids, const double *ops, const double *u, double *out) {
#pragma omp parallel for schedule(guided)
    for (int i = 0; i < n; ++i) {
        double acc[ORC_MAX_NOP];
        for (int k = 0; k < nop; ++k) acc[k] = 0.0;
        for (int t = off[i]; t < off[i + 1]; ++t) {
            const double du = u[ids[t] - 1] - u[i];
            for (int k = 0; k < nop; ++k) acc[k] += ops[(size_t)t * nop + k] * du;
        }
        for (int k = 0; k < nop; ++k) out[(size_t)i * nop + k] = acc[k];
    }
}

/* ---- CSR pattern: SparseMatrix.cpp:73-185 -------------------------------------------------------------- */
static int cmp_int(const void *a, const void *b) {
    const int x = *(const int *)a, y = *(const int *)b;
    return (x > y) - (x < y);
}

long long orc_csr_pattern(int n, int ndof, const int *off, const int *ids, const int *mirror, int *rowptr,
                          int *cols) {
    int maxf = 0;
    for (int i = 0; i < n; ++i) if (off[i + 1] - off[i] > maxf) maxf = off[i + 1] - off[i];
    int *cn = (int *)malloc(sizeof(int) * (size_t)(maxf + 2));
    long long nnz = 0;
    rowptr[0] = 0;
    for (int i = 0; i < n; ++i) {
        int m = 0;
        cn[m++] = i + 1;
        for (int t = off[i]; t < off[i + 1]; ++t) cn[m++] = ids[t];
        if (mirror && mirror[i] >= 1 && mirror[i] <= n) cn[m++] = mirror[i];
        qsort(cn, (size_t)m, sizeof(int), cmp_int);
        int u = 0;
        for (int k = 0; k < m; ++k) if (u == 0 || cn[k] != cn[u - 1]) cn[u++] = cn[k];
        for (int a = 0; a < ndof; ++a) {
            const int row = i * ndof + a;
            if (cols)
                for (int k = 0; k < u; ++k)
                    for (int b = 0; b < ndof; ++b) cols[nnz + (long long)k * ndof + b] = (cn[k] - 1) * ndof + b;
            nnz += (long long)u * ndof;
            rowptr[row + 1] = (int)nnz;
        }
    }
    free(cn);
    return nnz;
}

static int find_slot(const int *rowptr, const int *cols, int row, int col) {
    int lo = rowptr[row], hi = rowptr[row + 1] - 1;
    while (lo <= hi) {
        const int mid = lo + ((hi - lo) >> 1);
        if (cols[mid] == col) return mid;
        if (cols[mid] < col) lo = mid + 1; else hi = mid - 1;
    }
    return -1;
}

void orc_poisson_assemble(int n, int dim, int nop, const int *lapslots, const int *off, const int *ids,
                          const double *ops, double sigma, const double *f, const double *u, const int *rowptr,
                          const int *cols, double *kvals, double *rhs) {
    memset(kvals, 0, sizeof(double) * (size_t)rowptr[n]);
#pragma omp parallel for schedule(guided)
    for (int i = 0; i < n; ++i) {
        double r = 0.0 + (f ? f[i] : 0.0);
        const int sd = find_slot(rowptr, cols, i, i);
        kvals[sd] += -0.0;
        for (int t = off[i]; t < off[i + 1]; ++t) {
            const int j = ids[t] - 1;
            const double *o = ops + (size_t)t * nop;
            double lap = o[lapslots[0]] + o[lapslots[1]];
            if (dim >= 3) lap += o[lapslots[2]];
            const double coeff = sigma * lap;
            r += coeff * (u[j] - u[i]);
            kvals[sd] += -(-coeff);
            kvals[find_slot(rowptr, cols, i, j)] += -coeff;
        }
        rhs[i] = r;
    }
}

/* ---- explicit_pddo_frac: ExplicitPDDOFracElement.cpp:38-53, 239-299; FractureCriterion.h:30-43 ------- */
void orc_elastic_constants(int dim, int plane_stress, double E, double nu, double *C) {
    if (dim >= 3 || !plane_stress) {
        const double d = (1.0 + nu) * (1.0 - 2.0 * nu);
        C[0] = E * (1.0 - nu) / d; C[1] = E * nu / d; C[2] = E / (2.0 * (1.0 + nu));
    } else {
        const double d = 1.0 - nu * nu;
        C[0] = E / d; C[1] = E * nu / d; C[2] = E / (2.0 * (1.0 + nu));
    }
}

double orc_critical_stretch(int dim, int plane_stress, double G0, double E, double delta) {
    if (G0 <= 0.0 || E <= 0.0 || delta <= 0.0) return 0.0;
    double s2;
    if (dim >= 3) s2 = 5.0 * G0 / (6.0 * E * delta);
    else if (plane_stress) s2 = 4.0 * M_PI * G0 / (9.0 * E * delta);
    else s2 = 5.0 * M_PI * G0 / (12.0 * E * delta);
    return sqrt(s2);
}

void orc_epf_rate(int n, int dim, const double *coords3, const int *off, const int *ids, const double *navier,
                  double C11, double C12, double C66, double rho, const double *b, double sc, int tension_only,
                  int damage_on, const double *u, double *health, double *accel) {
    const int damage = damage_on && sc > 0.0;
    const int c = (dim >= 3) ? 6 : 3;
#pragma omp parallel for schedule(guided)
    for (int i = 0; i < n; ++i) {
        const int ri = i * dim;
        const double x0 = coords3[3 * i], y0 = coords3[3 * i + 1], z0 = (dim >= 3) ? coords3[3 * i + 2] : 0.0;
        if (damage) {
            for (int t = off[i]; t < off[i + 1]; ++t) {
                if (health[t] <= 0.0) continue;
                const int j = ids[t] - 1, rj = j * dim;
                const double xi0 = coords3[3 * j] - x0, xi1 = coords3[3 * j + 1] - y0,
                             xi2 = (dim >= 3) ? coords3[3 * j + 2] - z0 : 0.0;
                const double e0 = u[rj] - u[ri], e1 = u[rj + 1] - u[ri + 1], e2 = (dim >= 3) ? u[rj + 2] - u[ri + 2] : 0.0;
                const double r = sqrt(xi0 * xi0 + xi1 * xi1 + xi2 * xi2);
                if (r <= 0.0) continue;
                const double yx = xi0 + e0, yy = xi1 + e1, yz = xi2 + e2;
                const double s = (sqrt(yx * yx + yy * yy + yz * yz) - r) / r;
                if (sc > 0.0 && (tension_only ? (s > sc) : (fabs(s) > sc))) health[t] = 0.0;
            }
        }
        double L[3] = {0.0, 0.0, 0.0};
        for (int t = off[i]; t < off[i + 1]; ++t) {
            const double mu = health[t];
            if (mu <= 0.0) continue;
            const int j = ids[t] - 1, rj = j * dim;
            const double *G = navier + (size_t)t * c;
            const double dux = u[rj] - u[ri], duy = u[rj + 1] - u[ri + 1];
            if (dim >= 3) {
                const double duz = u[rj + 2] - u[ri + 2];
                const double Gxx = G[0], Gyy = G[1], Gzz = G[2], Gxy = G[3], Gxz = G[4], Gyz = G[5];
                const double p11 = C11 * Gxx + C66 * (Gyy + Gzz);
                const double p22 = C11 * Gyy + C66 * (Gxx + Gzz);
                const double p33 = C11 * Gzz + C66 * (Gxx + Gyy);
                const double a = C12 + C66;
                const double p12 = a * Gxy, p13 = a * Gxz, p23 = a * Gyz;
                L[0] += mu * (p11 * dux + p12 * duy + p13 * duz);
                L[1] += mu * (p12 * dux + p22 * duy + p23 * duz);
                L[2] += mu * (p13 * dux + p23 * duy + p33 * duz);
            } else {
                const double Gxx = G[0], Gyy = G[1], Gxy = G[2];
                const double p11 = C11 * Gxx + C66 * Gyy;
                const double p22 = C66 * Gxx + C11 * Gyy;
                const double pxy = (C12 + C66) * Gxy;
                L[0] += mu * (p11 * dux + pxy * duy);
                L[1] += mu * (pxy * dux + p22 * duy);
            }
        }
        for (int a = 0; a < dim; ++a) accel[ri + a] = (L[a] + b[a]) / rho;
    }
}

/* ---- ghost BC preset: DirichletBC.cpp:107-147, NeumannBC.cpp:88-105, BCSystem.cpp:114-129 ------------- */
void orc_bc_preset(int n, int dim, const double *coords3, const int *mirror, int nbc, const int *kind,
                   const int *comp_mask, const int *direct, const double *val, const double *vel,
                   const int *has_box, const double *box, const int *node_off, const int *nodes, double t,
                   double *u) {
    for (int e = 0; e < nbc; ++e) {
        for (int p = node_off[e]; p < node_off[e + 1]; ++p) {
            const int id = nodes[p];
            const int mb = (mirror && id >= 1 && id <= n) ? mirror[id - 1] : 0;
            if (kind[e] == 0) {
                if (has_box[e]) {
                    /* DirichletBC::insideBox (DirichletBC.cpp:89-98): all three axes on the xyz coordinates, an
                       axis with min > max is unconstrained */
                    int inside = 1;
                    for (int a = 0; a < 3; ++a) {
                        const double lo = box[6 * e + 2 * a], hi = box[6 * e + 2 * a + 1];
                        if (lo > hi) continue;
                        const double x = coords3[(size_t)(id - 1) * 3 + a];
                        if (x < lo || x > hi) inside = 0;
                    }
                    if (!inside) continue;
                }
                for (int a = 0; a < dim; ++a) {
                    if (!(comp_mask[e] & (1 << a))) continue;
                    const double g = val[e * dim + a] + vel[e * dim + a] * t;
                    u[(size_t)(id - 1) * dim + a] =
                        (mb >= 1 && !direct[e]) ? 2.0 * g - u[(size_t)(mb - 1) * dim + a] : g;
                }
            } else {
                if (mb < 1) continue;
                for (int a = 0; a < dim; ++a)
                    if (comp_mask[e] & (1 << a)) u[(size_t)(id - 1) * dim + a] = u[(size_t)(mb - 1) * dim + a];
            }
        }
    }
}

void orc_epf_run(int n, int dim, const double *coords3, const int *mirror, const int *off, const int *ids,
                 const double *navier, double C11, double C12, double C66, double rho, const double *b,
                 double sc, int tension_only, int damage_on, const double *u0, const double *v0, double dt,
                 int nsteps, int nbc, const int *kind, const int *comp_mask, const int *direct, const double *val,
                 const double *vel, const int *has_box, const double *box, const int *node_off, const int *nodes,
                 double *u, double *uold, double *health) {
    const size_t nd = (size_t)n * dim;
    double *a = (double *)malloc(sizeof(double) * nd);
    memcpy(u, u0, sizeof(double) * nd);
    orc_epf_rate(n, dim, coords3, off, ids, navier, C11, C12, C66, rho, b, sc, tension_only, damage_on, u, health, a);
    for (size_t k = 0; k < nd; ++k) uold[k] = u[k] - dt * (v0 ? v0[k] : 0.0) + 0.5 * dt * dt * a[k];
    double t = 0.0;
    const double dt2 = dt * dt;
    for (int s = 0; s < nsteps; ++s) {
        const double tn = t + dt;
        orc_epf_rate(n, dim, coords3, off, ids, navier, C11, C12, C66, rho, b, sc, tension_only, damage_on, u, health, a);
        for (size_t k = 0; k < nd; ++k) {
            const double un = 2.0 * u[k] - uold[k] + dt2 * a[k];
            uold[k] = u[k];
            u[k] = un;
        }
        orc_bc_preset(n, dim, coords3, mirror, nbc, kind, comp_mask, direct, val, vel, has_box, box, node_off, nodes,
                      tn, u);
        t = tn;
    }
    free(a);
}
