// The single device translation unit of the engine: constant tables, the
// ERI kernels, the one-electron kernel and small utility kernels, with their
// host launch wrappers.
#include "kernels.hpp"

#include <algorithm>
#include <cmath>
#include <mutex>
#include <set>
#include <vector>

#include "device_common.cuh"
#include "eri_common.cuh"
#include "fast_classes.hpp"
#include "eri_generic.cuh"
#include "engine.hpp"
#include "onee.cuh"
#include "tables.hpp"

namespace tlno_gpu {

using namespace dev;

namespace {

double binom(int n, int k) {
    if (k < 0 || k > n) return 0.0;
    double r = 1.0;
    for (int i = 1; i <= k; ++i) r = r * (n - k + i) / i;
    return r;
}

double dfact(int n) {  // n!! with (-1)!! = 1
    double r = 1.0;
    for (int k = n; k > 1; k -= 2) r *= k;
    return r;
}

// Real solid harmonics S_lm in Helgaker's closed form (Molecular
// Electronic-Structure Theory, eqs. 6.4.47-6.4.50), expressed over the
// unit-normalised Cartesian monomials of degree l and normalised; PySCF
// ordering (p: x, y, z; l >= 2: m = -l..l).  Produces, for each (sph, cart)
// with a nonzero coefficient, the coefficient on unit-normalised Cartesians.
void build_c2s(C2STable& t) {
    int pos = 0;
    for (int l = 0; l <= 4; ++l) {
        t.start[l] = pos;
        const int nc = (l + 1) * (l + 2) / 2;
        std::vector<int> cx(nc), cy(nc), cz(nc);
        {
            int i = 0;
            for (int x = l; x >= 0; --x)
                for (int y = l - x; y >= 0; --y) { cx[i] = x; cy[i] = y; cz[i] = l - x - y; ++i; }
        }
        auto idx_of = [&](int x, int y, int z) {
            for (int i = 0; i < nc; ++i) if (cx[i] == x && cy[i] == y && cz[i] == z) return i;
            return -1;
        };
        auto gram = [&](int i, int j) {
            const int sx = cx[i] + cx[j], sy = cy[i] + cy[j], sz = cz[i] + cz[j];
            if ((sx & 1) || (sy & 1) || (sz & 1)) return 0.0;
            return dfact(sx - 1) * dfact(sy - 1) * dfact(sz - 1);
        };
        const int ns = 2 * l + 1;
        for (int s = 0; s < ns; ++s) {
            std::vector<double> a(nc, 0.0);  // coefficients on raw monomials
            if (l == 1) {
                a[s] = 1.0;
            } else if (l == 0) {
                a[0] = 1.0;
            } else {
                const int m = s - l, am = std::abs(m);
                const double vm = m < 0 ? 0.5 : 0.0;
                for (int tt = 0; tt <= (l - am) / 2; ++tt)
                    for (int u = 0; u <= tt; ++u) {
                        const int vmax2 = static_cast<int>(std::floor(am / 2.0 - vm)) ;
                        for (int vi = 0; vi <= vmax2; ++vi) {
                            const double v = vi + vm;
                            const int twov = static_cast<int>(std::lround(2 * v));
                            const double sign = ((tt + vi) % 2 == 0) ? 1.0 : -1.0;
                            const double c = sign * std::pow(0.25, tt) * binom(l, tt) * binom(l - tt, am + tt) *
                                             binom(tt, u) * binom(am, twov);
                            const int px = 2 * tt + am - 2 * u - twov;
                            const int py = 2 * u + twov;
                            const int pz = l - 2 * tt - am;
                            const int i = idx_of(px, py, pz);
                            if (i >= 0) a[i] += c;
                        }
                    }
            }
            double n2 = 0.0;
            for (int i = 0; i < nc; ++i)
                for (int j = 0; j < nc; ++j) n2 += a[i] * a[j] * gram(i, j);
            const double inv = 1.0 / std::sqrt(n2);
            for (int i = 0; i < nc; ++i) {
                if (std::fabs(a[i]) < 1e-14) continue;
                const double unit = a[i] * std::sqrt(gram(i, i)) * inv;  // on unit-normalised Cartesians
                const double nang = 1.0 / std::sqrt(dfact(2 * cx[i] - 1) * dfact(2 * cy[i] - 1) * dfact(2 * cz[i] - 1));
                t.sph[pos] = static_cast<signed char>(s);
                t.cart[pos] = static_cast<signed char>(i);
                t.coef_raw[pos] = unit;
                t.coef[pos] = unit * nang;
                t.dense[l][s][i] = unit * nang;
                ++pos;
            }
        }
        t.count[l] = pos - t.start[l];
    }
}

void build_cart(CartTable& t) {
    int i = 0;
    for (int L = 0; L <= kMaxLSum; ++L)
        for (int x = L; x >= 0; --x)
            for (int y = L - x; y >= 0; --y) {
                t.xyz[i][0] = static_cast<signed char>(x);
                t.xyz[i][1] = static_cast<signed char>(y);
                t.xyz[i][2] = static_cast<signed char>(L - x - y);
                ++i;
            }
}

template <class T>
T* upload(const std::vector<T>& v) {
    T* p = nullptr;
    TLNO_CUDA(cudaMalloc(&p, v.size() * sizeof(T)));
    TLNO_CUDA(cudaMemcpy(p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice));
    return p;
}

// ---- utility kernels ----
__global__ void symmetrize_kernel(double* X, int M) {
    const long long n = (long long)M * M;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
        const int i = static_cast<int>(e / M), j = static_cast<int>(e % M);
        if (j <= i) continue;
        const double v = 0.5 * (X[(long long)i * M + j] + X[(long long)j * M + i]);
        X[(long long)i * M + j] = v;
        X[(long long)j * M + i] = v;
    }
}

__global__ void symmetrize_batch_kernel(double* X, const long long* offs, const int* dims, int count) {
    for (int b = blockIdx.y; b < count; b += gridDim.y) {
        const int M = dims[b];
        double* Y = X + offs[b];
        const long long n = (long long)M * M;
        for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
            const int i = static_cast<int>(e / M), j = static_cast<int>(e % M);
            if (j <= i) continue;
            const double v = 0.5 * (Y[(long long)i * M + j] + Y[(long long)j * M + i]);
            Y[(long long)i * M + j] = v;
            Y[(long long)j * M + i] = v;
        }
    }
}

__global__ void boys_test_kernel(const double* x, int n, int maxn, double* out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double F[40];
    boys_fn(maxn, x[i], F);
    for (int k = 0; k <= maxn; ++k) out[(long long)i * (maxn + 1) + k] = F[k];
}

template <typename R>
__global__ void rys_test_kernel(const double* T, int n, int nroots, double* roots, double* weights) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    for (int r = 0; r < nroots; ++r) {
        R rt, wt;
        rys_root<R>(nroots, R(T[i]), r, rt, wt);
        roots[(long long)i * nroots + r] = double(rt);
        weights[(long long)i * nroots + r] = double(wt);
    }
}

// Test hook of the FP32 shared-memory root path (mode 2), reading the
// interval polynomials from global memory.
template <int N>
__global__ void rys_interval_test_kernel(const double* T, int n, int mode, double* roots, double* weights) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || mode != 2) return;
    float r[N], w[N];
    rys_roots_smem32<N>(float(T[i]), c_tabs.rys32[N], r, w);
    for (int k = 0; k < N; ++k) {
        roots[(long long)i * N + k] = r[k];
        weights[(long long)i * N + k] = w[k];
    }
}

__global__ void absmax_kernel(const double* x, long long n, double* out) {
    __shared__ double red[32];
    double m = 0.0;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x)
        m = fmax(m, fabs(x[e]));
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
    __syncthreads();
    if (threadIdx.x < 32) {
        m = (threadIdx.x < (blockDim.x >> 5)) ? red[threadIdx.x] : 0.0;
        for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
        // non-negative doubles order like their bit patterns
        if (threadIdx.x == 0)
            atomicMax(reinterpret_cast<unsigned long long*>(out), static_cast<unsigned long long>(__double_as_longlong(m)));
    }
}

// max|x| as above, and x rounded to FP32 (the density copy the FP32
// kernels of a mixed build gather from) in the same pass.
__global__ void absmax_f32_kernel(const double* x, long long n, double* out, float* x32) {
    __shared__ double red[32];
    double m = 0.0;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
        const double v = x[e];
        x32[e] = static_cast<float>(v);
        m = fmax(m, fabs(v));
    }
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
    __syncthreads();
    if (threadIdx.x < 32) {
        m = (threadIdx.x < (blockDim.x >> 5)) ? red[threadIdx.x] : 0.0;
        for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
        if (threadIdx.x == 0)
            atomicMax(reinterpret_cast<unsigned long long*>(out), static_cast<unsigned long long>(__double_as_longlong(m)));
    }
}

__global__ void validate_density_kernel(const double* D, int M, unsigned int* status) {
    const long long n = (long long)M * M;
    unsigned int bits = 0;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
        const int i = static_cast<int>(e / M), j = static_cast<int>(e % M);
        const double v = D[e];
        const unsigned long long b = __double_as_longlong(v);
        if ((b & 0x7ff0000000000000ull) == 0x7ff0000000000000ull) { bits |= 1u; continue; }
        if (j <= i) continue;
        const double w = D[(long long)j * M + i];
        const double sc = fmax(1.0, fmax(fabs(v), fabs(w)));
        if (fabs(v - w) > 128.0 * 2.220446049250313e-16 * sc) bits |= 2u;
    }
    if (bits) atomicOr(status, bits);
}

// Density tables of the CVHF screen, per molecule (blockIdx.y): the ns x ns
// table of max |D| over each shell block and its transpose (the symmetric
// maximum the reference keeps per group pair, direct_build.ipp:122-205) and
// rho_max[mol] = max |D| (the largest block maximum).
__global__ void density_blocks_kernel(const double* D, const long long* mat_off, const int* mol_M, int M1,
                                      const int* shell_sph, const int* shell_L, const int* mol_shell_off,
                                      const int* mol_ns, int ns1, const long long* blk_off, double* blk,
                                      double* rho_max) {
    __shared__ double red[32];
    const int mol = blockIdx.y;
    const int M = mol_M ? mol_M[mol] : M1;
    const int ns = mol_ns ? mol_ns[mol] : ns1;
    const int so = mol_shell_off ? mol_shell_off[mol] : 0;
    const double* Dm = D + (mat_off ? mat_off[mol] : 0);
    double* out = blk + (blk_off ? blk_off[mol] : 0);
    const long long n = (long long)ns * ns;
    double m = 0.0;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
        const int i = static_cast<int>(e / ns), j = static_cast<int>(e % ns);
        const int r0 = shell_sph[so + i], c0 = shell_sph[so + j];
        const int nr = 2 * shell_L[so + i] + 1, nc = 2 * shell_L[so + j] + 1;
        double v = 0.0;
        for (int r = 0; r < nr; ++r)
            for (int c = 0; c < nc; ++c) {
                v = fmax(v, fabs(Dm[(long long)(r0 + r) * M + c0 + c]));
                v = fmax(v, fabs(Dm[(long long)(c0 + c) * M + r0 + r]));
            }
        out[e] = v;
        m = fmax(m, v);
    }
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
    __syncthreads();
    if (threadIdx.x < 32) {
        m = (threadIdx.x < (blockDim.x >> 5)) ? red[threadIdx.x] : 0.0;
        for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
        if (threadIdx.x == 0)
            atomicMax(reinterpret_cast<unsigned long long*>(rho_max + mol),
                      static_cast<unsigned long long>(__double_as_longlong(m)));
    }
}

// Incremental-state density step: delta = Dn - Dp (Dp null: first density,
// delta unused), status bit 1 = Dn non-finite, bit 2 = delta non-finite,
// bit 4 = some delta element nonzero; *dmax = max |delta| (max |Dn| without
// Dp), zeroed by the launcher.
__global__ void density_delta_kernel(const double* Dn, const double* Dp, double* delta, long long n,
                                     unsigned int* status, double* dmax) {
    __shared__ double red[32];
    unsigned int bits = 0;
    double m = 0.0;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
        const double v = Dn[e];
        if ((__double_as_longlong(v) & 0x7ff0000000000000ll) == 0x7ff0000000000000ll) {
            bits |= 1u;
            continue;
        }
        double d = v;
        if (Dp) {
            d = v - Dp[e];
            delta[e] = d;
            if ((__double_as_longlong(d) & 0x7ff0000000000000ll) == 0x7ff0000000000000ll) {
                bits |= 2u;
                continue;
            }
            if (d != 0.0) bits |= 4u;
        }
        m = fmax(m, fabs(d));
    }
    if (bits) atomicOr(status, bits);
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
    __syncthreads();
    if (threadIdx.x < 32) {
        m = (threadIdx.x < (blockDim.x >> 5)) ? red[threadIdx.x] : 0.0;
        for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
        if (threadIdx.x == 0)
            atomicMax(reinterpret_cast<unsigned long long*>(dmax), static_cast<unsigned long long>(__double_as_longlong(m)));
    }
}

// out = Gp + dG (Gp null: out = dG); status bit 1 = dG non-finite, bit 2 =
// out non-finite.
__global__ void g_accumulate_kernel(const double* Gp, const double* dG, double* out, long long n, unsigned int* status) {
    unsigned int bits = 0;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
        const double d = dG[e];
        if ((__double_as_longlong(d) & 0x7ff0000000000000ll) == 0x7ff0000000000000ll) {
            bits |= 1u;
            continue;
        }
        const double v = Gp ? Gp[e] + d : d;
        if ((__double_as_longlong(v) & 0x7ff0000000000000ll) == 0x7ff0000000000000ll) bits |= 2u;
        out[e] = v;
    }
    if (bits) atomicOr(status, bits);
}

__global__ void combine_g_kernel(const double* J, const double* K, double* G, long long n) {
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x)
        G[e] = J[e] - 0.5 * K[e];
}

template <typename R>
__global__ void fma_peak_kernel(R* out, int iters, R seed) {
    // 8 independent dependent chains per thread keep the FMA pipes busy.
    R a0 = seed + threadIdx.x, a1 = a0 + R(1), a2 = a0 + R(2), a3 = a0 + R(3);
    R a4 = a0 + R(4), a5 = a0 + R(5), a6 = a0 + R(6), a7 = a0 + R(7);
    const R m = R(0.999999), c = R(1e-7);
    for (int i = 0; i < iters; ++i) {
        a0 = fma(a0, m, c); a1 = fma(a1, m, c); a2 = fma(a2, m, c); a3 = fma(a3, m, c);
        a4 = fma(a4, m, c); a5 = fma(a5, m, c); a6 = fma(a6, m, c); a7 = fma(a7, m, c);
    }
    const R s = a0 + a1 + a2 + a3 + a4 + a5 + a6 + a7;
    if (s == R(-12345)) out[0] = s;  // keeps the chains live
}

// Power-form records of the 5-point Newton-forward interpolant on rows
// k..k+4 of the Rys table: with forward differences d1 = D f0,
// d2 = D^2 f0 / 2, d3 = D^3 f0 / 6, d4 = D^4 f0 / 24,
//   p(t) = f0 + d1 t + d2 t(t-1) + d3 t(t-1)(t-2) + d4 t(t-1)(t-2)(t-3)
//        = c0 + c1 t + c2 t^2 + c3 t^3 + c4 t^4,
//   c1 = d1 - d2 + 2 d3 - 6 d4, c2 = d2 - 3 d3 + 11 d4, c3 = d3 - 6 d4, c4 = d4.
// Record k: [(k * 5 + j) * 2N + i], i < N roots, N <= i < 2N weights.
std::vector<double> rys_power_records(const HostTables& h, int n) {
    const int rows = h.rys_rows[n];
    const int nk = rows - 4;
    std::vector<double> out(static_cast<std::size_t>(nk) * 10 * n, 0.0);
    for (int k = 0; k < nk; ++k) {
        for (int i = 0; i < 2 * n; ++i) {
            const std::vector<double>& src = i < n ? h.rys_roots[n] : h.rys_weights[n];
            const int col = i < n ? i : i - n;
            long double f[5];
            for (int r = 0; r < 5; ++r) f[r] = src[static_cast<std::size_t>(k + r) * n + col];
            const long double d1 = f[1] - f[0];
            const long double d2 = (f[2] - 2 * f[1] + f[0]) / 2;
            const long double d3 = (f[3] - 3 * f[2] + 3 * f[1] - f[0]) / 6;
            const long double d4 = (f[4] - 4 * f[3] + 6 * f[2] - 4 * f[1] + f[0]) / 24;
            const long double c[5] = {f[0], d1 - d2 + 2 * d3 - 6 * d4, d2 - 3 * d3 + 11 * d4, d3 - 6 * d4, d4};
            for (int j = 0; j < 5; ++j) out[(static_cast<std::size_t>(k) * 5 + j) * 2 * n + i] = static_cast<double>(c[j]);
        }
    }
    return out;
}

int sm_count() {
    static int n = 0;
    if (n == 0) {
        int dev = 0;
        TLNO_CUDA(cudaGetDevice(&dev));
        TLNO_CUDA(cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev));
    }
    return n;
}

}  // namespace

void ensure_device_tables() {
    static std::mutex mtx;
    static std::set<int> done;
    int devid = 0;
    TLNO_CUDA(cudaGetDevice(&devid));
    std::lock_guard<std::mutex> lock(mtx);
    if (done.count(devid)) return;
    const HostTables& h = host_tables();
    DevTables t{};
    t.boys = upload(h.boys);
    for (int n = 1; n <= kMaxRoots; ++n) {
        const std::vector<double> rec = rys_power_records(h, n);
        t.rys_h[n] = upload(rec);
        t.rys_h32[n] = upload(std::vector<float>(rec.begin(), rec.end()));
        t.tmax[n] = h.rys_tmax[n];
        for (int i = 0; i < n; ++i) {
            t.h2[n][i] = h.herm_root2[n][i];
            t.hw[n][i] = h.herm_weight[n][i];
        }
    }
    for (int n = 1; n <= kRys32MaxN; ++n) {
        t.rys32[n] = upload(rys32_table(n));
        t.rys32_nint[n] = rys32_intervals(n);
    }


    CartTable ct{};
    build_cart(ct);
    C2STable c2s{};
    build_c2s(c2s);
    upload_constant_tables(t, ct, c2s);
    TLNO_CUDA(cudaGetLastError());
#define TLNO_FAST_UPLOAD(id, a, b, c, d) fast_upload_##id(t, ct, c2s);
    TLNO_FAST_CLASSES(TLNO_FAST_UPLOAD)
#undef TLNO_FAST_UPLOAD
    TLNO_CUDA(cudaGetLastError());
    // The generic kernel may need more than 48 KB of dynamic shared memory.
    const int maxsm = 227 * 1024;
    TLNO_CUDA(cudaFuncSetAttribute(eri_generic_list_kernel<double, kStore>, cudaFuncAttributeMaxDynamicSharedMemorySize, maxsm));
    TLNO_CUDA(cudaFuncSetAttribute(eri_generic_list_kernel<double, kSchwarz>, cudaFuncAttributeMaxDynamicSharedMemorySize, maxsm));
    TLNO_CUDA(cudaFuncSetAttribute(eri_generic_jk_kernel<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, maxsm));
    TLNO_CUDA(cudaFuncSetAttribute(eri_generic_jk_kernel<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, maxsm));
    // (the block-per-quartet kernel also holds a little static shared memory)
    TLNO_CUDA(cudaFuncSetAttribute(eri_generic_cta_jk_kernel<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, maxsm - 1024));
    TLNO_CUDA(cudaFuncSetAttribute(eri_generic_cta_jk_kernel<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, maxsm - 1024));
    done.insert(devid);
}

int generic_warp_bytes(int la, int lb, int lc, int ld) {
    GenericLayout lay;
    lay.init(la, lb, lc, ld);
    return lay.words * 8;
}

static int generic_warps_for(int bytes) {
    int w = (100 * 1024) / bytes;
    if (w > 8) w = 8;
    if (w < 1) w = 1;
    return w;
}

void launch_eri_store(const PlanView& pv, const ClassLaunch& cl, cudaStream_t s) {
    if (cl.n_quartets == 0) return;
    const int bytes = generic_warp_bytes(cl.la, cl.lb, cl.lc, cl.ld);
    const int warps = generic_warps_for(bytes);
    const int grid = std::min((cl.n_quartets + warps - 1) / warps, sm_count() * 8);
    eri_generic_list_kernel<double, kStore><<<grid, 32 * warps, bytes * warps, s>>>(pv, cl);
    TLNO_CUDA(cudaGetLastError());
}

void launch_eri_schwarz(const PlanView& pv, const ClassLaunch& cl, cudaStream_t s) {
    if (cl.n_quartets == 0) return;
    const int bytes = generic_warp_bytes(cl.la, cl.lb, cl.lc, cl.ld);
    const int warps = generic_warps_for(bytes);
    const int grid = std::min((cl.n_quartets + warps - 1) / warps, sm_count() * 8);
    eri_generic_list_kernel<double, kSchwarz><<<grid, 32 * warps, bytes * warps, s>>>(pv, cl);
    TLNO_CUDA(cudaGetLastError());
}

void launch_pair_projectors(const int* pair_A, const int* pair_B, const double* shell_xyz, const int* shell_L,
                            const long long* off, int n_pairs, double* out, cudaStream_t s) {
    if (n_pairs == 0) return;
    const int warps = 8;
    const int grid = std::min((n_pairs + warps - 1) / warps, sm_count() * 16);
    pair_projector_kernel<<<grid, 32 * warps, 0, s>>>(pair_A, pair_B, shell_xyz, shell_L, off, n_pairs, out);
    TLNO_CUDA(cudaGetLastError());
}

// CTA shape of the generic J/K kernel for a class: threads per block and item
// slots per batch, and the dynamic shared memory it needs.
static void generic_cta_shape(int la, int lb, int lc, int ld, int& threads, int& nb_items, int& bytes) {
    GenericCtaLayout lay;
    lay.init(la, lb, lc, ld, 1);
    threads = lay.nas * lay.ncs > 2048 ? 256 : 128;
    nb_items = 64;
    for (;;) {
        lay.init(la, lb, lc, ld, nb_items);
        if (lay.words * 8 <= 100 * 1024 || nb_items <= 16) break;
        nb_items /= 2;
    }
    bytes = lay.words * 8;
}

void launch_eri_jk_generic(const PlanView& pv, const ClassLaunch& cl, bool fp32, int warps, int grid,
                           cudaStream_t s) {
    if (cl.tile_end <= cl.tile_begin) return;
    if (pv.proj && warps <= 0) {
        // one quartet per block at a time, projectors from the plan
        int threads = 0, nb_items = 0, bytes = 0;
        generic_cta_shape(cl.la, cl.lb, cl.lc, cl.ld, threads, nb_items, bytes);
        int per_sm = 0;
        if (fp32) {
            TLNO_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, eri_generic_cta_jk_kernel<float>, threads, bytes));
        } else {
            TLNO_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, eri_generic_cta_jk_kernel<double>, threads, bytes));
        }
        const int ntiles = cl.tile_end - cl.tile_begin;
        const int g = std::max(1, std::min(ntiles, sm_count() * std::max(per_sm, 1)));
        if (fp32)
            eri_generic_cta_jk_kernel<float><<<g, threads, bytes, s>>>(pv, cl, nb_items);
        else
            eri_generic_cta_jk_kernel<double><<<g, threads, bytes, s>>>(pv, cl, nb_items);
        TLNO_CUDA(cudaGetLastError());
        return;
    }
    const int bytes = generic_warp_bytes(cl.la, cl.lb, cl.lc, cl.ld);
    if (warps <= 0) warps = generic_warps_for(bytes);
    while (warps > 1 && bytes * warps > 200 * 1024) --warps;
    const int ntiles = cl.tile_end - cl.tile_begin;
    if (grid <= 0) grid = sm_count() * 4;
    grid = std::min(grid, ntiles);
    if (fp32)
        eri_generic_jk_kernel<float><<<grid, 32 * warps, bytes * warps, s>>>(pv, cl);
    else
        eri_generic_jk_kernel<double><<<grid, 32 * warps, bytes * warps, s>>>(pv, cl);
    TLNO_CUDA(cudaGetLastError());
}

bool has_fast_kernel(int la, int lb, int lc, int ld) { return fast_class_index(la, lb, lc, ld) >= 0; }

int fast_kernel_bras(int la, int lb, int lc, int ld) {
    switch (fast_class_index(la, lb, lc, ld)) {
#define TLNO_FAST_BRAS(id, a, b, c, d) \
    case id: return fast_bras_##id();
        TLNO_FAST_CLASSES(TLNO_FAST_BRAS)
#undef TLNO_FAST_BRAS
        default: return 1;
    }
}

bool launch_eri_jk_fast(const PlanView& pv, const ClassLaunch& cl, bool fp32, int grid, cudaStream_t s) {
    const int idx = fast_class_index(cl.la, cl.lb, cl.lc, cl.ld);
    if (idx < 0) return false;
    if (cl.tile_end <= cl.tile_begin) return true;
    const int ntiles = cl.tile_end - cl.tile_begin;
    // One resident wave of persistent CTAs (a second partial wave would
    // leave most SMs idle while it runs).
    static int resident[TLNO_FAST_COUNT][2] = {};
    int& nb = resident[idx][fp32 ? 1 : 0];
    if (nb == 0) {
        switch (idx) {
#define TLNO_FAST_OCC(id, a, b, c, d) \
    case id: nb = fast_blocks_per_sm_##id(fp32); break;
            TLNO_FAST_CLASSES(TLNO_FAST_OCC)
#undef TLNO_FAST_OCC
            default: nb = 1;
        }
    }
    const int wave = sm_count() * nb;
    grid = (grid <= 0) ? wave : std::min(grid, wave);
    grid = std::min(grid, ntiles);
    switch (idx) {
#define TLNO_FAST_CASE(id, a, b, c, d) \
    case id: fast_launch_##id(fp32, pv, cl, grid, s); break;
        TLNO_FAST_CLASSES(TLNO_FAST_CASE)
#undef TLNO_FAST_CASE
        default: return false;
    }
    TLNO_CUDA(cudaGetLastError());
    return true;
}

void launch_onee(const OneeLaunch& L, cudaStream_t s) {
    if (L.n_pairs == 0) return;
    const int warps = 4;
    const int smem = warps * kOneeWarpWords * static_cast<int>(sizeof(double));
    TLNO_CUDA(cudaFuncSetAttribute(onee_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    const int grid = std::min((L.n_pairs + warps - 1) / warps, sm_count() * 16);
    onee_kernel<<<grid, 32 * warps, smem, s>>>(L);
    TLNO_CUDA(cudaGetLastError());
}

void launch_symmetrize(double* X, const long long* offsets, const int* dims, int count, int max_m,
                       cudaStream_t s) {
    if (count == 0) return;
    dim3 grid(std::min(1024, (max_m * max_m + 255) / 256), std::min(count, 65535));
    symmetrize_batch_kernel<<<grid, 256, 0, s>>>(X, offsets, dims, count);
    TLNO_CUDA(cudaGetLastError());
}

void launch_symmetrize_single(double* X, int M, cudaStream_t s) {
    const long long n = (long long)M * M;
    const int grid = static_cast<int>(std::min<long long>((n + 255) / 256, sm_count() * 32));
    symmetrize_kernel<<<grid, 256, 0, s>>>(X, M);
    TLNO_CUDA(cudaGetLastError());
}

void launch_absmax(const double* x, long long n, double* out, cudaStream_t s) {
    TLNO_CUDA(cudaMemsetAsync(out, 0, sizeof(double), s));
    const int grid = static_cast<int>(std::max<long long>(1, std::min<long long>((n + 1023) / 1024, sm_count() * 4)));
    absmax_kernel<<<grid, 1024, 0, s>>>(x, n, out);
    TLNO_CUDA(cudaGetLastError());
}

void launch_absmax_f32(const double* x, long long n, double* out, float* x32, cudaStream_t s) {
    TLNO_CUDA(cudaMemsetAsync(out, 0, sizeof(double), s));
    const int grid = static_cast<int>(std::max<long long>(1, std::min<long long>((n + 1023) / 1024, sm_count() * 4)));
    absmax_f32_kernel<<<grid, 1024, 0, s>>>(x, n, out, x32);
    TLNO_CUDA(cudaGetLastError());
}

void launch_validate_density(const double* D, int M, unsigned int* status, cudaStream_t s) {
    const long long n = (long long)M * M;
    const int grid = static_cast<int>(std::min<long long>((n + 255) / 256, sm_count() * 16));
    validate_density_kernel<<<std::max(grid, 1), 256, 0, s>>>(D, M, status);
    TLNO_CUDA(cudaGetLastError());
}

void launch_density_blocks(const double* D, const long long* mat_off, const int* mol_M, int M1, const int* shell_sph,
                           const int* shell_L, const int* mol_shell_off, const int* mol_ns, int ns1, int n_mol,
                           long long max_entries, const long long* blk_off, double* blk, double* rho_max,
                           cudaStream_t s) {
    if (n_mol <= 0) return;
    TLNO_CUDA(cudaMemsetAsync(rho_max, 0, sizeof(double) * n_mol, s));
    const int gx = static_cast<int>(std::max<long long>(1, std::min<long long>((max_entries + 255) / 256,
                                                                                sm_count() * 8)));
    dim3 grid(gx, n_mol);
    density_blocks_kernel<<<grid, 256, 0, s>>>(D, mat_off, mol_M, M1, shell_sph, shell_L, mol_shell_off, mol_ns, ns1,
                                               blk_off, blk, rho_max);
    TLNO_CUDA(cudaGetLastError());
}

void launch_density_delta(const double* Dn, const double* Dp, double* delta, long long n, unsigned int* status,
                          double* dmax, cudaStream_t s) {
    TLNO_CUDA(cudaMemsetAsync(status, 0, sizeof(unsigned int), s));
    TLNO_CUDA(cudaMemsetAsync(dmax, 0, sizeof(double), s));
    const int grid = static_cast<int>(std::max<long long>(1, std::min<long long>((n + 255) / 256, sm_count() * 8)));
    density_delta_kernel<<<grid, 256, 0, s>>>(Dn, Dp, delta, n, status, dmax);
    TLNO_CUDA(cudaGetLastError());
}

void launch_g_accumulate(const double* Gp, const double* dG, double* out, long long n, unsigned int* status,
                         cudaStream_t s) {
    TLNO_CUDA(cudaMemsetAsync(status, 0, sizeof(unsigned int), s));
    const int grid = static_cast<int>(std::max<long long>(1, std::min<long long>((n + 255) / 256, sm_count() * 8)));
    g_accumulate_kernel<<<grid, 256, 0, s>>>(Gp, dG, out, n, status);
    TLNO_CUDA(cudaGetLastError());
}

void launch_combine_g(const double* J, const double* K, double* G, long long n, cudaStream_t s) {
    const int grid = static_cast<int>(std::min<long long>((n + 255) / 256, sm_count() * 16));
    combine_g_kernel<<<std::max(grid, 1), 256, 0, s>>>(J, K, G, n);
    TLNO_CUDA(cudaGetLastError());
}

double measure_fma_peak(bool fp32) {
    DeviceBuffer out;
    out.alloc(64);
    const int threads = 256, blocks = sm_count() * 8, iters = 1 << 14;
    cudaEvent_t e0, e1;
    TLNO_CUDA(cudaEventCreate(&e0));
    TLNO_CUDA(cudaEventCreate(&e1));
    double best = 0.0;
    for (int rep = 0; rep < 4; ++rep) {
        TLNO_CUDA(cudaEventRecord(e0));
        if (fp32) fma_peak_kernel<float><<<blocks, threads>>>(out.as<float>(), iters, 1.0f);
        else fma_peak_kernel<double><<<blocks, threads>>>(out.as<double>(), iters, 1.0);
        TLNO_CUDA(cudaEventRecord(e1));
        TLNO_CUDA(cudaEventSynchronize(e1));
        float ms = 0.f;
        TLNO_CUDA(cudaEventElapsedTime(&ms, e0, e1));
        const double flops = 2.0 * 8.0 * double(iters) * threads * blocks;
        if (rep > 0) best = std::max(best, flops / (ms * 1e-3) / 1e12);
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return best;
}

void launch_boys_test(const double* x, int n, int maxn, double* out, cudaStream_t s) {
    boys_test_kernel<<<(n + 127) / 128, 128, 0, s>>>(x, n, maxn, out);
    TLNO_CUDA(cudaGetLastError());
}

void launch_rys_test(const double* t, int n, int nroots, int fp32, double* roots, double* weights,
                     cudaStream_t s) {
    if (fp32 >= 2) {
        const int g = (n + 127) / 128;
        switch (nroots) {
            case 1: rys_interval_test_kernel<1><<<g, 128, 0, s>>>(t, n, fp32, roots, weights); break;
            case 2: rys_interval_test_kernel<2><<<g, 128, 0, s>>>(t, n, fp32, roots, weights); break;
            case 3: rys_interval_test_kernel<3><<<g, 128, 0, s>>>(t, n, fp32, roots, weights); break;
            default: break;
        }
        TLNO_CUDA(cudaGetLastError());
        return;
    }
    if (fp32)
        rys_test_kernel<float><<<(n + 127) / 128, 128, 0, s>>>(t, n, nroots, roots, weights);
    else
        rys_test_kernel<double><<<(n + 127) / 128, 128, 0, s>>>(t, n, nroots, roots, weights);
    TLNO_CUDA(cudaGetLastError());
}

}  // namespace tlno_gpu
