// Host generation of the Boys and Rys interpolation tables.
//
// Boys: F_n(x) = int_0^1 t^{2n} exp(-x t^2) dt sampled at x = k * 0.01 with a
// 96-point Gauss-Legendre rule on [0, 1] -- the same grid, order range and
// quadrature the reference tabulates (core/math/general_math.cpp:12-87), here
// stored grid-major and extended to order 39 so that a 6-term Taylor
// expansion around the nearest node (general_math.cpp:225-294, with
// d^k F_n/dx^k = (-1)^k F_{n+k}) serves every order up to 33.
//
// Rys: for N roots, the quadrature int_0^1 f(t^2) e^{-T t^2} dt =
// sum_i w_i f(r_i) is built from the three-term recurrence of the measure
// e^{-T x} dx / (2 sqrt x) on [0, 1] by the discretised Stieltjes procedure on
// the positive half of a Fejer grid, followed by the Golub-Welsch eigen-solve of
// the Jacobi matrix (Gautschi's method; the reference seeds its table the
// same way, rys_engine.ipp:3537-3739).  Samples are taken at T = k * 0.01 up
// to the per-N asymptotic switch tmax(N) = {29,37,43,49,55,60,65,71,76}
// (rys_engine.ipp:3543-3547) with six guard rows for the 5-point Newton
// stencil; beyond tmax the Hermite asymptotic r_i = h_i^2 / T,
// w_i = g_i / sqrt(T) applies (rys_engine.ipp:3479-3532), where (h_i, g_i) are
// the positive nodes and weights of the 2N-point Gauss-Hermite rule.
#include "tables.hpp"

#include <algorithm>
#include <cmath>
#include <mutex>
#include <stdexcept>
#include <string>
#include <thread>

namespace tlno_gpu {
namespace {

constexpr double kPi = 3.141592653589793238462643383279502884;

// Gauss-Legendre nodes/weights mapped to [0, 1] (Newton on P_n).
void gauss_legendre_unit(int n, std::vector<double>& x, std::vector<double>& w) {
    x.assign(n, 0.0);
    w.assign(n, 0.0);
    for (int i = 0; i < (n + 1) / 2; ++i) {
        double z = std::cos(kPi * (i + 0.75) / (n + 0.5));
        double dp = 1.0;
        for (int it = 0; it < 100; ++it) {
            double p0 = 1.0, p1 = z;
            for (int k = 2; k <= n; ++k) {
                const double pk = ((2.0 * k - 1.0) * z * p1 - (k - 1.0) * p0) / k;
                p0 = p1;
                p1 = pk;
            }
            // P_n = p1, P_{n-1} = p0
            dp = n * (z * p1 - p0) / (z * z - 1.0);
            const double dz = p1 / dp;
            z -= dz;
            if (std::fabs(dz) < 1e-16) break;
        }
        // Recompute the derivative at the converged node.
        double p0 = 1.0, p1 = z;
        for (int k = 2; k <= n; ++k) {
            const double pk = ((2.0 * k - 1.0) * z * p1 - (k - 1.0) * p0) / k;
            p0 = p1;
            p1 = pk;
        }
        dp = n * (z * p1 - p0) / (z * z - 1.0);
        const double wt = 1.0 / ((1.0 - z * z) * dp * dp);  // half of the [-1,1] weight
        x[i] = 0.5 * (1.0 - z);
        x[n - 1 - i] = 0.5 * (1.0 + z);
        w[i] = wt;
        w[n - 1 - i] = wt;
    }
}

struct GL96 {
    std::vector<double> x, w;
    GL96() { gauss_legendre_unit(96, x, w); }
};

const GL96& gl96() {
    static const GL96 g;
    return g;
}

// Symmetric tridiagonal eigen-solve by cyclic Jacobi rotations.  Returns the
// eigenvalues ascending and the squared first components of the normalised
// eigenvectors (the Golub-Welsch weights divided by beta0).
void jacobi_tridiagonal(int n, const double* diag, const double* offd_sq,
                        double* eval, double* v0sq) {
    std::vector<double> a(n * n, 0.0), v(n * n, 0.0);
    for (int i = 0; i < n; ++i) {
        a[i * n + i] = diag[i];
        v[i * n + i] = 1.0;
    }
    for (int i = 1; i < n; ++i) {
        const double e = std::sqrt(std::max(offd_sq[i], 0.0));
        a[(i - 1) * n + i] = e;
        a[i * n + (i - 1)] = e;
    }
    for (int sweep = 0; sweep < 100; ++sweep) {
        double off = 0.0;
        for (int p = 0; p < n; ++p)
            for (int q = p + 1; q < n; ++q) off += a[p * n + q] * a[p * n + q];
        if (off < 1e-34) break;
        for (int p = 0; p < n; ++p) {
            for (int q = p + 1; q < n; ++q) {
                const double apq = a[p * n + q];
                if (std::fabs(apq) < 1e-300) continue;
                const double app = a[p * n + p], aqq = a[q * n + q];
                const double theta = (aqq - app) / (2.0 * apq);
                const double t = (theta >= 0 ? 1.0 : -1.0) /
                                 (std::fabs(theta) + std::sqrt(theta * theta + 1.0));
                const double c = 1.0 / std::sqrt(t * t + 1.0), s = t * c;
                for (int k = 0; k < n; ++k) {
                    const double akp = a[k * n + p], akq = a[k * n + q];
                    a[k * n + p] = c * akp - s * akq;
                    a[k * n + q] = s * akp + c * akq;
                }
                for (int k = 0; k < n; ++k) {
                    const double apk = a[p * n + k], aqk = a[q * n + k];
                    a[p * n + k] = c * apk - s * aqk;
                    a[q * n + k] = s * apk + c * aqk;
                }
                for (int k = 0; k < n; ++k) {
                    const double vkp = v[k * n + p], vkq = v[k * n + q];
                    v[k * n + p] = c * vkp - s * vkq;
                    v[k * n + q] = s * vkp + c * vkq;
                }
            }
        }
    }
    std::vector<int> order(n);
    for (int i = 0; i < n; ++i) order[i] = i;
    std::sort(order.begin(), order.end(),
              [&](int l, int r) { return a[l * n + l] < a[r * n + r]; });
    for (int i = 0; i < n; ++i) {
        eval[i] = a[order[i] * n + order[i]];
        v0sq[i] = v[0 * n + order[i]] * v[0 * n + order[i]];
    }
}

// Positive half of Fejer's first rule on [-1, 1] with 2*nh nodes; for an even
// integrand these give int_0^1 directly.
void fejer_half(int nh, std::vector<double>& x, std::vector<double>& w) {
    const int n = 2 * nh;
    x.assign(nh, 0.0);
    w.assign(nh, 0.0);
    for (int k = 0; k < nh; ++k) {
        const double theta = (2.0 * k + 1.0) * kPi / (2.0 * n);
        x[k] = std::cos(theta);
        double s = 0.0;
        for (int m = 1; m <= n / 2; ++m) s += std::cos(2.0 * m * theta) / (4.0 * m * m - 1.0);
        w[k] = (2.0 / n) * (1.0 - 2.0 * s);
    }
}

struct FejerCache {
    std::vector<double> x[kRysMaxN + 1], w[kRysMaxN + 1];
    FejerCache() {
        for (int n = 1; n <= kRysMaxN; ++n) fejer_half(200 + 24 * n, x[n], w[n]);
    }
};

const FejerCache& fejer_cache() {
    static const FejerCache c;
    return c;
}

void hermite_half_rule(int n, double* root2, double* weight) {
    const int m = 2 * n;
    std::vector<double> diag(m, 0.0), offsq(m, 0.0), ev(m), v0(m);
    for (int k = 1; k < m; ++k) offsq[k] = 0.5 * k;
    jacobi_tridiagonal(m, diag.data(), offsq.data(), ev.data(), v0.data());
    const double beta0 = std::sqrt(kPi);
    int out = 0;
    for (int i = 0; i < m && out < n; ++i) {
        if (ev[i] <= 0.0) continue;
        root2[out] = ev[i] * ev[i];
        weight[out] = beta0 * v0[i];
        ++out;
    }
    if (out != n) throw std::runtime_error("tlno_gpu: Gauss-Hermite rule construction failed");
}

}  // namespace

double rys_tmax(int n) {
    static const double t[kRysMaxN + 1] = {0, 29, 37, 43, 49, 55, 60, 65, 71, 76};
    return (n >= 1 && n <= kRysMaxN) ? t[n] : 0.0;
}

void boys_quadrature(int max_n, double x, double* out) {
    const GL96& g = gl96();
    for (int n = 0; n <= max_n; ++n) out[n] = 0.0;
    for (int i = 0; i < 96; ++i) {
        const double t2 = g.x[i] * g.x[i];
        double term = g.w[i] * std::exp(-x * t2);
        for (int n = 0; n <= max_n; ++n) {
            out[n] += term;
            term *= t2;
        }
    }
}

bool rys_rule_accurate(int n, double t, double* roots, double* weights) {
    const FejerCache& fc = fejer_cache();
    const std::vector<double>& fx = fc.x[n];
    const std::vector<double>& fw = fc.w[n];
    const int m = static_cast<int>(fx.size());
    std::vector<double> X(m), W(m), p_prev(m, 0.0), p_cur(m, 1.0), p_next(m);
    for (int i = 0; i < m; ++i) {
        X[i] = fx[i] * fx[i];
        W[i] = fw[i] * std::exp(-t * X[i]);
    }
    double alpha[kRysMaxN], beta[kRysMaxN];
    double norm_prev = 0.0;
    for (int k = 0; k < n; ++k) {
        double s0 = 0.0, s1 = 0.0;
        for (int i = 0; i < m; ++i) {
            const double q = W[i] * p_cur[i] * p_cur[i];
            s0 += q;
            s1 += q * X[i];
        }
        if (!(s0 > 0.0) || !std::isfinite(s0)) return false;
        alpha[k] = s1 / s0;
        beta[k] = (k == 0) ? s0 : s0 / norm_prev;
        norm_prev = s0;
        if (k + 1 < n) {
            for (int i = 0; i < m; ++i) {
                p_next[i] = (X[i] - alpha[k]) * p_cur[i] - (k > 0 ? beta[k] * p_prev[i] : 0.0);
            }
            p_prev.swap(p_cur);
            p_cur.swap(p_next);
        }
    }
    double ev[kRysMaxN], v0[kRysMaxN];
    jacobi_tridiagonal(n, alpha, beta, ev, v0);
    for (int i = 0; i < n; ++i) {
        roots[i] = ev[i];
        weights[i] = beta[0] * v0[i];
    }
    // Moment check: sum_i w_i r_i^k must reproduce F_k(T) for k < 2N.
    double mu[2 * kRysMaxN];
    boys_quadrature(2 * n - 1, t, mu);
    for (int k = 0; k < 2 * n; ++k) {
        double q = 0.0;
        for (int i = 0; i < n; ++i) q += weights[i] * std::pow(roots[i], k);
        if (std::fabs(q - mu[k]) > std::max(1e-13, 1e-10 * std::fabs(mu[k]))) return false;
    }
    return true;
}

int rys_rows(int n) { return static_cast<int>(rys_tmax(n) * 100.0) + 7; }

int rys32_intervals(int n) { return static_cast<int>(std::ceil(rys_tmax(n) * kRys32PerUnit)); }

std::vector<float> rys32_table(int n) {
    constexpr int nc = kRys32Deg + 1;
    const int nint = rys32_intervals(n);
    std::vector<float> out(static_cast<std::size_t>(nint) * nc * 2 * n, 0.0f);
    // Chebyshev nodes of [-1/2, 1/2] and the inverse of their Vandermonde
    // matrix (monomials in u, lowest power first), in long double.
    long double un[nc];
    for (int j = 0; j < nc; ++j) un[j] = 0.5L * std::cos((2.0L * j + 1.0L) * 3.14159265358979323846264338327950288L / (2.0L * nc));
    long double A[nc][2 * nc];
    for (int r = 0; r < nc; ++r) {
        long double pw = 1.0L;
        for (int c = 0; c < nc; ++c) { A[r][c] = pw; pw *= un[r]; }
        for (int c = 0; c < nc; ++c) A[r][nc + c] = (r == c) ? 1.0L : 0.0L;
    }
    for (int c = 0; c < nc; ++c) {  // Gauss-Jordan with partial pivoting
        int piv = c;
        for (int r = c + 1; r < nc; ++r)
            if (std::fabs(A[r][c]) > std::fabs(A[piv][c])) piv = r;
        for (int k = 0; k < 2 * nc; ++k) std::swap(A[c][k], A[piv][k]);
        const long double d = A[c][c];
        for (int k = 0; k < 2 * nc; ++k) A[c][k] /= d;
        for (int r = 0; r < nc; ++r) {
            if (r == c) continue;
            const long double f = A[r][c];
            for (int k = 0; k < 2 * nc; ++k) A[r][k] -= f * A[c][k];
        }
    }
    const double h = 1.0 / kRys32PerUnit;
    for (int k = 0; k < nint; ++k) {
        double vals[nc][2 * kRysMaxN];
        for (int j = 0; j < nc; ++j) {
            const double T = (k + 0.5 + static_cast<double>(un[j])) * h;
            double r[kRysMaxN], w[kRysMaxN];
            if (!rys_rule_accurate(n, T, r, w))
                throw std::runtime_error("tlno_gpu: Rys rule failed its moment check at N=" + std::to_string(n) +
                                         " T=" + std::to_string(T));
            for (int i = 0; i < n; ++i) {
                vals[j][i] = r[i];
                vals[j][n + i] = w[i];
            }
        }
        for (int i = 0; i < 2 * n; ++i)
            for (int c = 0; c < nc; ++c) {  // coefficient c = sum_j inv(V)[c][j] f(u_j)
                long double acc = 0.0L;
                for (int j = 0; j < nc; ++j) acc += A[c][nc + j] * vals[j][i];
                out[(static_cast<std::size_t>(k) * nc + c) * 2 * n + i] = static_cast<float>(acc);
            }
    }
    return out;
}

const HostTables& host_tables() {
    static std::once_flag once;
    static HostTables tabs;
    std::call_once(once, [] {
        // Boys table (grid-major).
        tabs.boys.assign(static_cast<std::size_t>(kBoysRows) * kBoysOrders, 0.0);
        for (int k = 0; k < kBoysRows; ++k)
            boys_quadrature(kBoysOrders - 1, k * kBoysDx,
                            tabs.boys.data() + static_cast<std::size_t>(k) * kBoysOrders);
        // Hermite asymptotic constants.
        for (int n = 1; n <= kRysMaxN; ++n) hermite_half_rule(n, tabs.herm_root2[n], tabs.herm_weight[n]);
        // Rys tables, rows filled in parallel per root count.
        std::vector<std::thread> workers;
        std::vector<std::string> errors(kRysMaxN + 1);
        for (int n = 1; n <= kRysMaxN; ++n) {
            tabs.rys_tmax[n] = rys_tmax(n);
            tabs.rys_rows[n] = rys_rows(n);
            tabs.rys_roots[n].assign(static_cast<std::size_t>(tabs.rys_rows[n]) * n, 0.0);
            tabs.rys_weights[n].assign(static_cast<std::size_t>(tabs.rys_rows[n]) * n, 0.0);
        }
        const unsigned nthreads = std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
        for (unsigned tid = 0; tid < nthreads; ++tid) {
            workers.emplace_back([tid, nthreads, &errors] {
                for (int n = 1; n <= kRysMaxN; ++n) {
                    for (int k = static_cast<int>(tid); k < tabs.rys_rows[n];
                         k += static_cast<int>(nthreads)) {
                        double r[kRysMaxN], w[kRysMaxN];
                        if (!rys_rule_accurate(n, k * kRysDx, r, w)) {
                            errors[n] = "Rys rule failed its moment check at N=" +
                                        std::to_string(n) + " T=" + std::to_string(k * kRysDx);
                            continue;
                        }
                        for (int i = 0; i < n; ++i) {
                            tabs.rys_roots[n][static_cast<std::size_t>(k) * n + i] = r[i];
                            tabs.rys_weights[n][static_cast<std::size_t>(k) * n + i] = w[i];
                        }
                    }
                }
            });
        }
        for (auto& t : workers) t.join();
        for (const auto& e : errors)
            if (!e.empty()) throw std::runtime_error("tlno_gpu: " + e);
    });
    return tabs;
}

}  // namespace tlno_gpu
