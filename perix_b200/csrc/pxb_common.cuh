// Device-side building blocks shared by the perix_b200 kernels (sm_100a).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace pxb {

constexpr int kWarp = 32;
constexpr unsigned kFull = 0xffffffffu;

// ---- PDDO multi-index tables at compile time --------------------------------------------------------------
// Reference ordering (src/PDOperators/PDOperators.cpp:51-75): total order ascending, within an order p
// descending, then q descending (r = order-p-q); 2D has r = 0.
__host__ __device__ constexpr int nop_of(int dim, int order) {
    int n = 0;
    for (int o = 1; o <= order; ++o) n += (dim == 3) ? (o + 1) * (o + 2) / 2 : (o + 1);
    return n;
}

template <int DIM, int ORDER>
struct QTable {
    static constexpr int NOP = nop_of(DIM, ORDER);
    int p[NOP], q[NOP], r[NOP];
    double fact[NOP];
    __host__ __device__ constexpr QTable() : p{}, q{}, r{}, fact{} {
        int k = 0;
        for (int o = 1; o <= ORDER; ++o) {
            for (int pp = o; pp >= 0; --pp) {
                if (DIM == 3) {
                    for (int qq = o - pp; qq >= 0; --qq) {
                        p[k] = pp; q[k] = qq; r[k] = o - pp - qq;
                        fact[k] = f(pp) * f(qq) * f(o - pp - qq);
                        ++k;
                    }
                } else {
                    p[k] = pp; q[k] = o - pp; r[k] = 0;
                    fact[k] = f(pp) * f(o - pp);
                    ++k;
                }
            }
        }
    }
    __host__ __device__ static constexpr double f(int n) {
        double v = 1.0;
        for (int i = 2; i <= n; ++i) v *= i;
        return v;
    }
    __host__ __device__ constexpr int slot(int pp, int qq, int rr) const {
        for (int k = 0; k < NOP; ++k)
            if (p[k] == pp && q[k] == qq && r[k] == rr) return k;
        return -1;
    }
};

// Monomials eta^{q_k} for all slots, built by repeated multiplication exactly like the reference
// (CalcPDOperators.cpp:74-86): ex^p * ey^q * ez^r as a left-to-right product starting from 1.
template <int DIM, int ORDER, typename T>
__device__ __forceinline__ void monomials(T ex, T ey, T ez, T *m) {
    constexpr QTable<DIM, ORDER> Q{};
#pragma unroll
    for (int k = 0; k < Q.NOP; ++k) {
        T v = T(1);
#pragma unroll
        for (int t = 0; t < Q.p[k]; ++t) v *= ex;
#pragma unroll
        for (int t = 0; t < Q.q[k]; ++t) v *= ey;
#pragma unroll
        for (int t = 0; t < Q.r[k]; ++t) v *= ez;
        m[k] = v;
    }
}

// ---- weight and rim volume correction (CalcPDOperators.cpp:48-60) -----------------------------------------
__device__ __forceinline__ double bond_weight(double xn, double delta) {
    const double r = 2.0 * xn / delta;
    return exp(-r * r);
}

__device__ __forceinline__ double rim_correction(double xn, double delta, double dxc) {
    if (dxc <= 0.0) return 1.0;
    if (xn <= delta - 0.5 * dxc) return 1.0;
    double v = (delta - xn + 0.5 * dxc) / dxc;
    return fmin(fmax(v, 0.0), 1.0);
}

// ---- warp reductions ---------------------------------------------------------------------------------------
template <int LANES, typename T>
__device__ __forceinline__ T group_sum(T v) {
#pragma unroll
    for (int o = LANES / 2; o > 0; o >>= 1) v += __shfl_xor_sync(kFull, v, o);
    return v;
}

template <int LANES>
__device__ __forceinline__ int group_sum_int(int v) {
#pragma unroll
    for (int o = LANES / 2; o > 0; o >>= 1) v += __shfl_xor_sync(kFull, v, o);
    return v;
}

template <int LANES>
__device__ __forceinline__ double group_max(double v) {
#pragma unroll
    for (int o = LANES / 2; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(kFull, v, o));
    return v;
}

// NaN-propagating maximum of non-negative values (fmax would drop a NaN): the blow-up guard must see a non-finite
// displacement
__device__ __forceinline__ double max_nan(double a, double b) { return (b > a || b != b) ? b : a; }

template <int LANES>
__device__ __forceinline__ double group_max_nan(double v) {
#pragma unroll
    for (int o = LANES / 2; o > 0; o >>= 1) v = max_nan(v, __shfl_xor_sync(kFull, v, o));
    return v;
}

// u^{n+1} of the central difference in the reference's rounding (TimeStepping.cpp:529-545): the uniform step
// 2u - u_prev + dt^2 a, or, for a step whose dt differs from the previous step's (var != 0), the variable-step form
// u + rho (u - u_prev) + w a with rho = dt/dt_prev and w = dt (dt + dt_prev)/2
__device__ __forceinline__ double cd_next(double u, double up, double acc, double dt2, int var, double rho, double w) {
    if (var) return __dadd_rn(__dadd_rn(u, __dmul_rn(rho, __dsub_rn(u, up))), __dmul_rn(w, acc));
    return __dadd_rn(__dsub_rn(__dmul_rn(2.0, u), up), __dmul_rn(dt2, acc));
}

// ---- compensated FP32 accumulation (Knuth two-sum) ---------------------------------------------------------
struct CompF {
    float s, c;
    __device__ __forceinline__ CompF() : s(0.f), c(0.f) {}
    __device__ __forceinline__ void add(float x) {
        const float t = s + x;
        const float bp = t - s;
        const float e = (s - (t - bp)) + (x - bp);
        s = t;
        c += e;
    }
    __device__ __forceinline__ double value() const { return (double)s + (double)c; }
};

// ---- positions ------------------------------------------------------------------------------------------------
// 2D positions are stored as double2, 3D as double4 (x,y,z,0): one aligned vector load per neighbour gather.
template <int DIM>
struct Vec;
template <>
struct Vec<2> {
    using T = double2;
    __device__ __forceinline__ static double c(const double2 &v, int a) { return a == 0 ? v.x : v.y; }
};
template <>
struct Vec<3> {
    using T = double4;
    __device__ __forceinline__ static double c(const double4 &v, int a) { return a == 0 ? v.x : (a == 1 ? v.y : v.z); }
};

// read-only gathers of node positions (the 3D double4 as two 16-byte loads)
__device__ __forceinline__ double2 ldg_vec(const double2 *p) { return __ldg(p); }
__device__ __forceinline__ double4 ldg_vec(const double4 *p) {
    const double2 *q = reinterpret_cast<const double2 *>(p);
    const double2 lo = __ldg(q), hi = __ldg(q + 1);
    return make_double4(lo.x, lo.y, hi.x, hi.y);
}

// order-preserving key for atomicMax on non-negative doubles (NaN sorts above +inf)
__device__ __forceinline__ unsigned long long dbl_key(double v) { return (unsigned long long)__double_as_longlong(v); }

}  // namespace pxb
