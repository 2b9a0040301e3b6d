// Device-side constants and math shared by every kernel of the engine:
// Cartesian index tables, the sparse Cartesian->spherical transform, the
// Boys function and the tabulated Rys roots/weights.  Included once, by
// kernels.cu (one translation unit, so __constant__ data has one copy).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace tlno_gpu {
namespace dev {

constexpr int kMaxL = 4;          // per shell
constexpr int kMaxLSum = 8;       // La + Lb <= 8
constexpr int kNCartCum8 = 165;   // sum_{L<=8} (L+1)(L+2)/2
constexpr int kMaxRoots = 9;

struct DevTables {
    const double* boys;             // [row * 40 + n]
    const double* rys_r[kMaxRoots + 1];
    const double* rys_w[kMaxRoots + 1];
    const float* rys_r32[kMaxRoots + 1];
    const float* rys_w32[kMaxRoots + 1];
    double tmax[kMaxRoots + 1];
    double h2[kMaxRoots + 1][kMaxRoots];
    double hw[kMaxRoots + 1][kMaxRoots];
};

// Cartesian triples for |a| = 0..8 in the reference order
// (for lx = L..0: for ly = L-lx..0), flat index = offset(L) + local.
struct CartTable {
    signed char xyz[kNCartCum8][3];
};

// Sparse Cartesian->spherical transform for L <= 4 with the angular
// normalisation N_ang(cart) folded into each coefficient, the form of the
// reference's final pair projector (rys_engine.ipp:1816-1842).
struct C2STable {
    int count[5];
    int start[5];
    signed char sph[60];
    signed char cart[60];
    double coef[60];      // coefficient * N_ang(cart)
    double coef_raw[60];  // coefficient without N_ang (one-electron path)
    double dense[5][9][15];  // dense form of coef: [L][sph][cart]
};

// Internal linkage: every device translation unit holds its own copy, filled
// by that unit's upload function (upload_constant_tables).
namespace {
__constant__ DevTables c_tabs;
__constant__ CartTable c_cart;
__constant__ C2STable c_c2s;

inline void upload_constant_tables(const DevTables& t, const CartTable& c, const C2STable& s) {
    cudaMemcpyToSymbol(c_tabs, &t, sizeof(t));
    cudaMemcpyToSymbol(c_cart, &c, sizeof(c));
    cudaMemcpyToSymbol(c_c2s, &s, sizeof(s));
}
}  // namespace

__host__ __device__ __forceinline__ int ncart(int L) { return (L + 1) * (L + 2) / 2; }
__host__ __device__ __forceinline__ int nsph(int L) { return 2 * L + 1; }
__host__ __device__ __forceinline__ int cart_offset(int L) { return L * (L + 1) * (L + 2) / 6; }
__host__ __device__ __forceinline__ int ncart_cum(int L) { return (L + 1) * (L + 2) * (L + 3) / 6; }
__host__ __device__ __forceinline__ int cart_flat(int lx, int ly, int lz) {
    const int L = lx + ly + lz;
    const int dx = L - lx;
    return cart_offset(L) + dx * (dx + 1) / 2 + (dx - ly);
}

// ---------------------------------------------------------------------------
// Boys function F_0..F_maxn(x), maxn <= 33.  Below x = 40: F_maxn from a
// 6-term Taylor expansion about the nearest 0.01 grid node (derivatives
// d^k F_n/dx^k = (-1)^k F_{n+k}, remainder below 3e-17), then the stable
// downward recursion F_{n-1} = (2x F_n + e^{-x}) / (2n-1).  At and above 40:
// F_0 = sqrt(pi/x)/2 * erf(sqrt x) and the upward recursion
// F_{n+1} = ((2n+1) F_n - e^{-x}) / (2x), stable there because x > n.
// (Same domains and expansions as the reference's batched evaluator,
// core/math/general_math.cpp:243-309.)
__device__ __forceinline__ void boys_fn(int maxn, double x, double* F) {
    if (x < 40.0) {
        const int k = __double2int_rn(x * 100.0);
        const double d = k * 0.01 - x;
        const double* row = c_tabs.boys + k * 40 + maxn;
        double v = row[5];
        v = fma(v, d * (1.0 / 5.0), row[4]);
        v = fma(v, d * (1.0 / 4.0), row[3]);
        v = fma(v, d * (1.0 / 3.0), row[2]);
        v = fma(v, d * (1.0 / 2.0), row[1]);
        v = fma(v, d, row[0]);
        F[maxn] = v;
        if (maxn > 0) {
            const double ex = exp(-x);
            const double tx = 2.0 * x;
            for (int n = maxn; n >= 1; --n) F[n - 1] = (tx * F[n] + ex) / (2.0 * n - 1.0);
        }
    } else {
        const double sx = sqrt(x);
        double v = 0.5 * sqrt(3.141592653589793238462643383279502884 / x) * erf(sx);
        F[0] = v;
        if (maxn > 0) {
            const double ex = exp(-x);
            const double inv2x = 0.5 / x;
            for (int n = 0; n < maxn; ++n) {
                v = ((2.0 * n + 1.0) * v - ex) * inv2x;
                F[n + 1] = v;
            }
        }
    }
}

// ---------------------------------------------------------------------------
// Rys root t_i^2 and weight w_i (i < N) for argument T.  Below tmax(N) a
// 5-point Newton-forward stencil on the 0.01 grid (the reference's scheme,
// rys_engine.ipp:3784-3812); above it the Hermite asymptotic form.
template <typename R> struct RysTab;
template <> struct RysTab<double> {
    static __device__ __forceinline__ const double* r(int n) { return c_tabs.rys_r[n]; }
    static __device__ __forceinline__ const double* w(int n) { return c_tabs.rys_w[n]; }
};
template <> struct RysTab<float> {
    static __device__ __forceinline__ const float* r(int n) { return c_tabs.rys_r32[n]; }
    static __device__ __forceinline__ const float* w(int n) { return c_tabs.rys_w32[n]; }
};

template <typename R>
__device__ __forceinline__ R newton5(R f0, R f1, R f2, R f3, R f4, R t) {
    const R d1 = f1 - f0;
    const R d2 = (f2 - R(2) * f1 + f0) * R(0.5);
    const R d3 = (f3 - R(3) * f2 + R(3) * f1 - f0) * R(1.0 / 6.0);
    const R d4 = (f4 - R(4) * f3 + R(6) * f2 - R(4) * f1 + f0) * R(1.0 / 24.0);
    return f0 + t * (d1 + (t - R(1)) * (d2 + (t - R(2)) * (d3 + (t - R(3)) * d4)));
}

template <typename R>
__device__ __forceinline__ void rys_root(int N, R T, int i, R& root, R& weight) {
    if (T >= R(c_tabs.tmax[N])) {
        const R inv = R(1) / T;
        root = R(c_tabs.h2[N][i]) * inv;
        weight = R(c_tabs.hw[N][i]) * sqrt(inv);
        return;
    }
    const R fi = T * R(100);
    const int k = static_cast<int>(fi);
    const R t = fi - R(k);
    const R* rb = RysTab<R>::r(N) + k * N + i;
    const R* wb = RysTab<R>::w(N) + k * N + i;
    root = newton5<R>(__ldg(rb), __ldg(rb + N), __ldg(rb + 2 * N), __ldg(rb + 3 * N), __ldg(rb + 4 * N), t);
    weight = newton5<R>(__ldg(wb), __ldg(wb + N), __ldg(wb + 2 * N), __ldg(wb + 3 * N), __ldg(wb + 4 * N), t);
}

// All N roots at once (thread-per-quartet kernels).
template <typename R, int N>
__device__ __forceinline__ void rys_roots_all(R T, R* root, R* weight) {
    if (T >= R(c_tabs.tmax[N])) {
        const R inv = R(1) / T;
        const R sinv = sqrt(inv);
#pragma unroll
        for (int i = 0; i < N; ++i) {
            root[i] = R(c_tabs.h2[N][i]) * inv;
            weight[i] = R(c_tabs.hw[N][i]) * sinv;
        }
        return;
    }
    const R fi = T * R(100);
    const int k = static_cast<int>(fi);
    const R t = fi - R(k);
    const R* rb = RysTab<R>::r(N) + k * N;
    const R* wb = RysTab<R>::w(N) + k * N;
#pragma unroll
    for (int i = 0; i < N; ++i) {
        root[i] = newton5<R>(__ldg(rb + i), __ldg(rb + N + i), __ldg(rb + 2 * N + i),
                             __ldg(rb + 3 * N + i), __ldg(rb + 4 * N + i), t);
        weight[i] = newton5<R>(__ldg(wb + i), __ldg(wb + N + i), __ldg(wb + 2 * N + i),
                               __ldg(wb + 3 * N + i), __ldg(wb + 4 * N + i), t);
    }
}

}  // namespace dev
}  // namespace tlno_gpu
