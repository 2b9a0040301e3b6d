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
    // Rys roots/weights per root count N as local quartic polynomials: grid
    // point k holds 5 coefficient rows of 2N values (N roots, then N
    // weights), record [(k * 5 + j) * 2N + i], so one lookup reads one
    // contiguous 80N-byte record (40N bytes in FP32).
    const double* rys_h[kMaxRoots + 1];
    const float* rys_h32[kMaxRoots + 1];
    double tmax[kMaxRoots + 1];
    double h2[kMaxRoots + 1][kMaxRoots];
    double hw[kMaxRoots + 1][kMaxRoots];
    // FP32 interval polynomials of the mixed-precision kernels (N = 1..3):
    // interval k of width 1/4 holds 6 coefficient rows of 2N floats
    // (lowest power of u = 4T - k - 1/2 first); staged in shared memory.
    const float* rys32[4];
    int rys32_nint[4];
};
constexpr int kRys32PerUnitDev = 4;
constexpr int kRys32CoefDev = 6;

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
// Rys root t_i^2 and weight w_i (i < N) for argument T.  Below tmax(N) the
// 5-point Newton-forward interpolant on the 0.01 grid (the reference's
// scheme, rys_engine.ipp:3784-3812), stored in power form
// c0 + c1 t + ... + c4 t^4 of the offset t in [0, 1) so that one lookup is
// one contiguous record and four FMAs per value; above tmax the Hermite
// asymptotic form.
template <typename R> struct RysTab;
template <> struct RysTab<double> {
    using V2 = double2;
    static __device__ __forceinline__ const double* h(int n) { return c_tabs.rys_h[n]; }
};
template <> struct RysTab<float> {
    using V2 = float2;
    static __device__ __forceinline__ const float* h(int n) { return c_tabs.rys_h32[n]; }
};

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
    const R* rec = RysTab<R>::h(N) + static_cast<long long>(k) * 10 * N;
    R r = __ldg(rec + 8 * N + i), w = __ldg(rec + 9 * N + i);
#pragma unroll
    for (int j = 3; j >= 0; --j) {
        r = r * t + __ldg(rec + 2 * j * N + i);
        w = w * t + __ldg(rec + (2 * j + 1) * N + i);
    }
    root = r;
    weight = w;
}

// All N roots at once (compile-time N).
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
    using V2 = typename RysTab<R>::V2;
    const R fi = T * R(100);
    const int k = static_cast<int>(fi);
    const R t = fi - R(k);
    const V2* rec = reinterpret_cast<const V2*>(RysTab<R>::h(N) + static_cast<long long>(k) * 10 * N);
    R c[5][2 * N];
#pragma unroll
    for (int j = 0; j < 5; ++j)
#pragma unroll
        for (int m = 0; m < N; ++m) {
            const V2 v = __ldg(rec + j * N + m);
            c[j][2 * m] = v.x;
            c[j][2 * m + 1] = v.y;
        }
#pragma unroll
    for (int i = 0; i < 2 * N; ++i) {
        R v = c[4][i];
        v = v * t + c[3][i];
        v = v * t + c[2][i];
        v = v * t + c[1][i];
        v = v * t + c[0][i];
        if (i < N) root[i] = v; else weight[i - N] = v;
    }
}

// FP32 roots and weights for N <= 3 from the shared-memory interval
// polynomials (table = the staged copy of c_tabs.rys32[N]); the Hermite
// asymptotic form above tmax(N).
template <int N>
__device__ __forceinline__ void rys_roots_smem32(float T, const float* __restrict__ table, float* root,
                                                 float* weight) {
    if (T >= float(c_tabs.tmax[N])) {
        const float inv = 1.0f / T;
        const float sinv = sqrtf(inv);
#pragma unroll
        for (int i = 0; i < N; ++i) {
            root[i] = float(c_tabs.h2[N][i]) * inv;
            weight[i] = float(c_tabs.hw[N][i]) * sinv;
        }
        return;
    }
    const float x = T * float(kRys32PerUnitDev);
    const int k = static_cast<int>(x);
    const float u = x - float(k) - 0.5f;
    const float2* rec = reinterpret_cast<const float2*>(table + k * (kRys32CoefDev * 2 * N));
    float c[kRys32CoefDev][2 * N];
#pragma unroll
    for (int j = 0; j < kRys32CoefDev; ++j)
#pragma unroll
        for (int m = 0; m < N; ++m) {
            const float2 v = rec[j * N + m];
            c[j][2 * m] = v.x;
            c[j][2 * m + 1] = v.y;
        }
#pragma unroll
    for (int i = 0; i < 2 * N; ++i) {
        float v = c[kRys32CoefDev - 1][i];
#pragma unroll
        for (int j = kRys32CoefDev - 2; j >= 0; --j) v = fmaf(v, u, c[j][i]);
        if (i < N) root[i] = v; else weight[i - N] = v;
    }
}

}  // namespace dev
}  // namespace tlno_gpu
