// TEST INFRASTRUCTURE ONLY -- the CPU restatement oracle.  Never linked into
// the shipped library; only tests/, __graft_entry__.smoke() and bench.py's
// cpu_baseline leg may load it, as the checker.
//
// A plain, deliberately unoptimised C++ restatement of the reference
// algorithm for the integral hot path, each part citing the reference file
// it follows (paths relative to the reference repository):
//   * shell normalisation ............ core/shell/shell_contract.cpp:9-48,
//                                      core/shell/shell_math.cpp:50-77
//   * Boys F_n(x) .................... core/math/general_math.cpp:12-164
//                                      (96-point Gauss-Legendre table on a 0.01
//                                      grid, 5-point Newton interpolation,
//                                      upward recursion / quadrature >= 12)
//   * Rys roots and weights .......... integrals/two_electron/rys/
//                                      rys_engine.ipp:3365-3838 (moments for
//                                      N <= 2, discretised Stieltjes on a Fejer
//                                      grid + Jacobi eigen-solve, Hermite
//                                      asymptotic beyond tmax(N)); evaluated
//                                      directly per argument, no table
//   * 2-D Rys VRR, contracted radial
//     accumulation, HRR ket/bra ...... rys_engine.ipp:13630-13842, 3141-3362
//   * final spherical projection ..... rys_engine.ipp:1801-1860 (real solid
//                                      harmonics, PySCF order, unit-diagonal
//                                      Cartesian normalisation)
//   * Schwarz bound / gate ........... rys_engine.ipp:16165-16258,
//                                      native_quartets.ipp:556-574
//   * J/K digestion (full 8-fold sum)  fock/detail/consumer_policies.ipp:87-221
//   * one-electron S, T, V ........... integrals/one_electron/
//                                      onee_integrals.cpp:32-157, 284-887
// Parity is pinned by tests/test_cpu.py against the compiled reference
// (oracle/_ref) and the golden fixtures in tests/golden/.
#include <algorithm>
#include <array>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

namespace {

constexpr double kPi = 3.141592653589793238462643383279502884;

double dfact(int n) {
    double r = 1.0;
    for (int k = n; k > 1; k -= 2) r *= k;
    return r;
}
double binom(int n, int k) {
    if (k < 0 || k > n) return 0.0;
    double r = 1.0;
    for (int i = 1; i <= k; ++i) r = r * (n - k + i) / i;
    return r;
}
int ncart(int L) { return (L + 1) * (L + 2) / 2; }
int nsph(int L) { return 2 * L + 1; }
int coff(int L) { return L * (L + 1) * (L + 2) / 6; }
int ccum(int L) { return (L + 1) * (L + 2) * (L + 3) / 6; }

struct Trip { int x, y, z; };
std::vector<Trip> cart_list() {  // |a| = 0..8, reference order
    std::vector<Trip> t;
    for (int L = 0; L <= 8; ++L)
        for (int x = L; x >= 0; --x)
            for (int y = L - x; y >= 0; --y) t.push_back({x, y, L - x - y});
    return t;
}
const std::vector<Trip>& CT() {
    static const std::vector<Trip> t = cart_list();
    return t;
}
int cflat(int x, int y, int z) {
    const int L = x + y + z, dx = L - x;
    return coff(L) + dx * (dx + 1) / 2 + (dx - y);
}
double angn(int x, int y, int z) { return 1.0 / std::sqrt(dfact(2 * x - 1) * dfact(2 * y - 1) * dfact(2 * z - 1)); }

// ---------------- Boys (general_math.cpp) ----------------
struct GL {
    double x[96], w[96];
    GL() {
        const int n = 96;
        for (int i = 0; i < n / 2; ++i) {
            double z = std::cos(kPi * (i + 0.75) / (n + 0.5)), dp = 0;
            for (int it = 0; it < 64; ++it) {
                double p0 = 1, p1 = z;
                for (int k = 2; k <= n; ++k) { const double pk = ((2.0 * k - 1) * z * p1 - (k - 1.0) * p0) / k; p0 = p1; p1 = pk; }
                dp = n * (z * p1 - p0) / (z * z - 1);
                const double dz = p1 / dp;
                z -= dz;
                if (std::fabs(dz) < 1e-16) break;
            }
            double p0 = 1, p1 = z;
            for (int k = 2; k <= n; ++k) { const double pk = ((2.0 * k - 1) * z * p1 - (k - 1.0) * p0) / k; p0 = p1; p1 = pk; }
            dp = n * (z * p1 - p0) / (z * z - 1);
            const double wt = 1.0 / ((1 - z * z) * dp * dp);
            x[i] = 0.5 * (1 - z); x[n - 1 - i] = 0.5 * (1 + z);
            w[i] = wt; w[n - 1 - i] = wt;
        }
    }
};
const GL& gl() { static const GL g; return g; }

double boys_quad(int n, double x) {
    double v = 0;
    for (int i = 0; i < 96; ++i) { const double t2 = gl().x[i] * gl().x[i]; v += gl().w[i] * std::pow(t2, n) * std::exp(-x * t2); }
    return v;
}
struct BoysTab {
    std::vector<double> v;  // [order][4001]
    BoysTab() : v(33 * 4001, 0.0) {
        for (int k = 0; k <= 4000; ++k) {
            const double x = k * 0.01;
            for (int i = 0; i < 96; ++i) {
                const double t2 = gl().x[i] * gl().x[i];
                double term = gl().w[i] * std::exp(-x * t2);
                for (int n = 0; n <= 32; ++n) { v[n * 4001 + k] += term; term *= t2; }
            }
        }
    }
};
const BoysTab& btab() { static const BoysTab b; return b; }

double boys(int n, double x) {
    if (n > 32) return boys_quad(n, x);
    if (x >= 12.0) {
        if (x < n + 0.5) return boys_quad(n, x);
        const double ex = std::exp(-x);
        double v = 0.5 * std::sqrt(kPi / x) * std::erf(std::sqrt(x));
        for (int m = 0; m < n; ++m) v = ((2.0 * m + 1.0) * v - ex) / (2.0 * x);
        return v;
    }
    const double g = x / 0.01;
    const int k = static_cast<int>(g);
    const double t = g - k;
    const double* f = btab().v.data() + n * 4001 + k;
    const double d1 = f[1] - f[0], d2 = (f[2] - 2 * f[1] + f[0]) / 2, d3 = (f[3] - 3 * f[2] + 3 * f[1] - f[0]) / 6;
    const double d4 = (f[4] - 4 * f[3] + 6 * f[2] - 4 * f[1] + f[0]) / 24;
    const double d5 = (f[5] - 5 * f[4] + 10 * f[3] - 10 * f[2] + 5 * f[1] - f[0]) / 120;
    return f[0] + t * (d1 + (t - 1) * (d2 + (t - 2) * (d3 + (t - 3) * (d4 + (t - 4) * d5))));
}

// ---------------- Rys roots (rys_engine.ipp:3365-3838) ----------------
void jacobi_eig(int n, std::vector<double> a, double* ev, double* v0sq) {
    std::vector<double> v(n * n, 0.0);
    for (int i = 0; i < n; ++i) v[i * n + i] = 1;
    for (int sweep = 0; sweep < 100; ++sweep) {
        double off = 0;
        for (int p = 0; p < n; ++p) for (int q = p + 1; q < n; ++q) off += a[p * n + q] * a[p * n + q];
        if (off < 1e-34) break;
        for (int p = 0; p < n; ++p)
            for (int q = p + 1; q < n; ++q) {
                const double apq = a[p * n + q];
                if (std::fabs(apq) < 1e-300) continue;
                const double th = (a[q * n + q] - a[p * n + p]) / (2 * apq);
                const double t = (th >= 0 ? 1 : -1) / (std::fabs(th) + std::sqrt(th * th + 1));
                const double c = 1 / std::sqrt(t * t + 1), s = t * c;
                for (int k = 0; k < n; ++k) { const double x = a[k * n + p], y = a[k * n + q]; a[k * n + p] = c * x - s * y; a[k * n + q] = s * x + c * y; }
                for (int k = 0; k < n; ++k) { const double x = a[p * n + k], y = a[q * n + k]; a[p * n + k] = c * x - s * y; a[q * n + k] = s * x + c * y; }
                for (int k = 0; k < n; ++k) { const double x = v[k * n + p], y = v[k * n + q]; v[k * n + p] = c * x - s * y; v[k * n + q] = s * x + c * y; }
            }
    }
    std::vector<int> o(n);
    for (int i = 0; i < n; ++i) o[i] = i;
    std::sort(o.begin(), o.end(), [&](int l, int r) { return a[l * n + l] < a[r * n + r]; });
    for (int i = 0; i < n; ++i) { ev[i] = a[o[i] * n + o[i]]; v0sq[i] = v[o[i]] * v[o[i]]; }
}

double rys_tmax(int n) {
    static const double t[10] = {0, 29, 37, 43, 49, 55, 60, 65, 71, 76};
    return n <= 9 ? t[n] : 35.0 + 5.0 * n;
}

void rys(int N, double T, double* r, double* w) {
    if (T >= rys_tmax(N)) {  // Hermite asymptotic: 2N-point Gauss-Hermite, positive half
        const int m = 2 * N;
        std::vector<double> a(m * m, 0.0);
        for (int k = 1; k < m; ++k) a[(k - 1) * m + k] = a[k * m + k - 1] = std::sqrt(0.5 * k);
        std::vector<double> ev(m), v0(m);
        jacobi_eig(m, a, ev.data(), v0.data());
        int out = 0;
        for (int i = 0; i < m && out < N; ++i) {
            if (ev[i] <= 0) continue;
            r[out] = ev[i] * ev[i] / T;
            w[out] = std::sqrt(kPi) * v0[i] / std::sqrt(T);
            ++out;
        }
        return;
    }
    if (N <= 2) {  // moments
        double mu[4];
        for (int k = 0; k < 2 * N; ++k) mu[k] = boys(k, T);
        if (N == 1) { r[0] = mu[1] / mu[0]; w[0] = mu[0]; return; }
        const double a0 = mu[1] / mu[0];
        const double s1 = mu[2] - a0 * mu[1], s2 = mu[3] - a0 * mu[2];
        const double a1 = s2 / s1 - mu[1] / mu[0], b1 = s1 / mu[0];
        const double h = 0.5 * (a0 + a1), dd = 0.5 * (a0 - a1), disc = std::sqrt(dd * dd + b1);
        r[0] = h - disc; r[1] = h + disc;
        const double e0 = r[0] - a0, e1 = r[1] - a0;
        w[0] = mu[0] * b1 / (b1 + e0 * e0); w[1] = mu[0] * b1 / (b1 + e1 * e1);
        return;
    }
    // discretised Stieltjes on the positive half of a Fejer grid
    const int nh = std::min(24 * N + 40, 400), nn = 2 * nh;
    std::vector<double> X(nh), W(nh);
    for (int k = 0; k < nh; ++k) {
        const double th = (2.0 * k + 1) * kPi / (2.0 * nn);
        const double x = std::cos(th);
        double s = 0;
        for (int m = 1; m <= nn / 2; ++m) s += std::cos(2.0 * m * th) / (4.0 * m * m - 1);
        X[k] = x * x;
        W[k] = (2.0 / nn) * (1 - 2 * s) * std::exp(-T * x * x);
    }
    std::vector<double> al(N), be(N), pm(nh, 0.0), pc(nh, 1.0), pn(nh);
    double nprev = 0;
    for (int k = 0; k < N; ++k) {
        double s0 = 0, s1 = 0;
        for (int i = 0; i < nh; ++i) { const double q = W[i] * pc[i] * pc[i]; s0 += q; s1 += q * X[i]; }
        al[k] = s1 / s0;
        be[k] = k == 0 ? s0 : s0 / nprev;
        nprev = s0;
        for (int i = 0; i < nh; ++i) pn[i] = (X[i] - al[k]) * pc[i] - (k ? be[k] * pm[i] : 0.0);
        pm.swap(pc);
        pc.swap(pn);
    }
    std::vector<double> a(N * N, 0.0);
    for (int i = 0; i < N; ++i) a[i * N + i] = al[i];
    for (int i = 1; i < N; ++i) a[(i - 1) * N + i] = a[i * N + i - 1] = std::sqrt(std::max(be[i], 0.0));
    std::vector<double> v0(N);
    jacobi_eig(N, a, r, v0.data());
    for (int i = 0; i < N; ++i) w[i] = be[0] * v0[i];
}

// ---------------- real solid harmonics (PySCF order) ----------------
struct C2S { std::vector<std::array<double, 15>> rows[5]; };  // [L][sph][cart] on unit-normalised Cartesians
const C2S& c2s() {
    static const C2S t = [] {
        C2S t;
        for (int l = 0; l <= 4; ++l) {
            const int nc = ncart(l);
            std::vector<Trip> cs(CT().begin() + coff(l), CT().begin() + coff(l) + nc);
            auto gram = [&](int i, int j) {
                const int sx = cs[i].x + cs[j].x, sy = cs[i].y + cs[j].y, sz = cs[i].z + cs[j].z;
                if ((sx | sy | sz) & 1) return 0.0;
                return dfact(sx - 1) * dfact(sy - 1) * dfact(sz - 1);
            };
            for (int s = 0; s < nsph(l); ++s) {
                std::vector<double> a(nc, 0.0);
                if (l <= 1) a[l == 0 ? 0 : s] = 1;
                else {
                    const int m = s - l, am = std::abs(m);
                    const double vm = m < 0 ? 0.5 : 0.0;
                    for (int tt = 0; tt <= (l - am) / 2; ++tt)
                        for (int u = 0; u <= tt; ++u)
                            for (int vi = 0; vi <= static_cast<int>(std::floor(am / 2.0 - vm)); ++vi) {
                                const int twov = static_cast<int>(std::lround(2 * (vi + vm)));
                                const double c = ((tt + vi) % 2 ? -1.0 : 1.0) * std::pow(0.25, tt) * binom(l, tt) *
                                                 binom(l - tt, am + tt) * binom(tt, u) * binom(am, twov);
                                const int px = 2 * tt + am - 2 * u - twov, py = 2 * u + twov, pz = l - 2 * tt - am;
                                a[cflat(px, py, pz) - coff(l)] += c;
                            }
                }
                double n2 = 0;
                for (int i = 0; i < nc; ++i) for (int j = 0; j < nc; ++j) n2 += a[i] * a[j] * gram(i, j);
                std::array<double, 15> row{};
                for (int i = 0; i < nc; ++i) row[i] = a[i] * std::sqrt(gram(i, i)) / std::sqrt(n2);
                t.rows[l].push_back(row);
            }
        }
        return t;
    }();
    return t;
}

// ---------------- basis ----------------
struct OShell { double c[3]; int L, np; std::vector<double> e, cr; int sph; };
struct OBasis { std::vector<OShell> sh; int M = 0; std::vector<int> Z; std::vector<double> xyz; };

OBasis make_basis(int ns, const double* centers, const int* L, const int* np, const double* ex, const double* co,
                  int na, const int* Z, const double* xyz) {
    OBasis b;
    int off = 0;
    for (int s = 0; s < ns; ++s) {
        OShell sh;
        for (int k = 0; k < 3; ++k) sh.c[k] = centers[3 * s + k];
        sh.L = L[s];
        sh.np = np[s];
        sh.e.assign(ex + off, ex + off + np[s]);
        // make_shell for the (L,0,0) component, then divide by its N_ang
        std::vector<double> c(np[s]);
        const double df = dfact(2 * L[s] - 1);
        for (int i = 0; i < np[s]; ++i)
            c[i] = co[off + i] * std::sqrt(std::pow(2.0, 2.0 * L[s] + 1.5) * std::pow(ex[off + i], L[s] + 1.5) /
                                           (std::pow(kPi, 1.5) * df));
        double n2 = 0;
        for (int i = 0; i < np[s]; ++i)
            for (int j = 0; j < np[s]; ++j) {
                const double p = ex[off + i] + ex[off + j];
                n2 += c[i] * c[j] * std::pow(kPi / p, 1.5) * df / std::pow(2 * p, L[s]);
            }
        for (int i = 0; i < np[s]; ++i) sh.cr.push_back(c[i] / std::sqrt(n2) / angn(L[s], 0, 0));
        sh.sph = b.M;
        b.M += nsph(L[s]);
        b.sh.push_back(sh);
        off += np[s];
    }
    b.Z.assign(Z, Z + na);
    b.xyz.assign(xyz, xyz + 3 * na);
    return b;
}

// ---------------- ERI block (rys_engine.ipp:13630-13842) ----------------
// raw Cartesian block [ncart(a) ncart(b)] x [ncart(c) ncart(d)] with radial coefficients
std::vector<double> eri_cart(const OBasis& B, int ia, int ib, int ic, int id) {
    const OShell &A = B.sh[ia], &Bs = B.sh[ib], &C = B.sh[ic], &D = B.sh[id];
    const int la = A.L, lb = Bs.L, lc = C.L, ld = D.L, LAB = la + lb, LCD = lc + ld, N = (LAB + LCD) / 2 + 1;
    const int nas = ccum(LAB) - coff(la), ncf = ccum(LCD);
    std::vector<double> Tr(nas * ncf, 0.0);
    const int KS = LCD + 1;
    std::vector<double> G[3];
    for (auto& g : G) g.assign((LAB + 1) * KS, 0.0);
    auto pairs = [&](const OShell& X, const OShell& Y, std::vector<std::array<double, 6>>& out) {
        const double r2 = (X.c[0] - Y.c[0]) * (X.c[0] - Y.c[0]) + (X.c[1] - Y.c[1]) * (X.c[1] - Y.c[1]) +
                          (X.c[2] - Y.c[2]) * (X.c[2] - Y.c[2]);
        for (int i = 0; i < X.np; ++i)
            for (int j = 0; j < Y.np; ++j) {
                const double c = X.cr[i] * Y.cr[j];
                if (c == 0) continue;
                const double p = X.e[i] + Y.e[j];
                out.push_back({p, (X.e[i] * X.c[0] + Y.e[j] * Y.c[0]) / p, (X.e[i] * X.c[1] + Y.e[j] * Y.c[1]) / p,
                               (X.e[i] * X.c[2] + Y.e[j] * Y.c[2]) / p,
                               std::exp(-X.e[i] * Y.e[j] / p * r2) * c / p, 1.0 / p});
            }
    };
    std::vector<std::array<double, 6>> bra, ket;
    pairs(A, Bs, bra);
    pairs(C, D, ket);
    double rt[16], wt[16];
    for (const auto& bp : bra)
        for (const auto& kp : ket) {
            const double p = bp[0], q = kp[0], pq = p + q;
            const double PQ[3] = {bp[1] - kp[1], bp[2] - kp[2], bp[3] - kp[3]};
            const double T = p * q / pq * (PQ[0] * PQ[0] + PQ[1] * PQ[1] + PQ[2] * PQ[2]);
            rys(N, T, rt, wt);
            const double pref = 2.0 * std::pow(kPi, 2.5) * bp[4] * kp[4] / std::sqrt(pq);
            for (int r = 0; r < N; ++r) {
                const double t2 = rt[r];
                const double B00 = t2 / (2 * pq), B10 = (1 - q / pq * t2) / (2 * p), B01 = (1 - p / pq * t2) / (2 * q);
                const double P[3] = {bp[1], bp[2], bp[3]}, Q[3] = {kp[1], kp[2], kp[3]};
                for (int ax = 0; ax < 3; ++ax) {
                    auto& g = G[ax];
                    const double c00 = (P[ax] - A.c[ax]) - q / pq * PQ[ax] * t2;
                    const double d00 = (Q[ax] - C.c[ax]) + p / pq * PQ[ax] * t2;
                    g[0] = ax == 2 ? pref * wt[r] : 1.0;
                    if (LAB > 0) g[KS] = c00 * g[0];
                    for (int i = 1; i < LAB; ++i) g[(i + 1) * KS] = c00 * g[i * KS] + i * B10 * g[(i - 1) * KS];
                    for (int k = 0; k < LCD; ++k)
                        for (int i = 0; i <= LAB; ++i) {
                            double v = d00 * g[i * KS + k];
                            if (i) v += i * B00 * g[(i - 1) * KS + k];
                            if (k) v += k * B01 * g[i * KS + k - 1];
                            g[i * KS + k + 1] = v;
                        }
                }
                for (int a = 0; a < nas; ++a) {
                    const Trip ta = CT()[coff(la) + a];
                    for (int c = 0; c < ncf; ++c) {
                        const Trip tc = CT()[c];
                        Tr[a * ncf + c] += G[0][ta.x * KS + tc.x] * G[1][ta.y * KS + tc.y] * G[2][ta.z * KS + tc.z];
                    }
                }
            }
        }
    // HRR ket: (a|c,d) = sum_u C(d,u) CD^(d-u) (a|c+u)   (rys_engine.ipp:3141-3257)
    const int nca = ncart(la), ncb = ncart(lb), ncc = ncart(lc), ncd = ncart(ld);
    const double CD[3] = {C.c[0] - D.c[0], C.c[1] - D.c[1], C.c[2] - D.c[2]};
    const double AB[3] = {A.c[0] - Bs.c[0], A.c[1] - Bs.c[1], A.c[2] - Bs.c[2]};
    std::vector<double> K(nas * ncc * ncd, 0.0);
    for (int a = 0; a < nas; ++a)
        for (int c = 0; c < ncc; ++c)
            for (int d = 0; d < ncd; ++d) {
                const Trip tc = CT()[coff(lc) + c], td = CT()[coff(ld) + d];
                double s = 0;
                for (int ux = 0; ux <= td.x; ++ux)
                    for (int uy = 0; uy <= td.y; ++uy)
                        for (int uz = 0; uz <= td.z; ++uz)
                            s += binom(td.x, ux) * std::pow(CD[0], td.x - ux) * binom(td.y, uy) * std::pow(CD[1], td.y - uy) *
                                 binom(td.z, uz) * std::pow(CD[2], td.z - uz) * Tr[a * ncf + cflat(tc.x + ux, tc.y + uy, tc.z + uz)];
                K[(a * ncc + c) * ncd + d] = s;
            }
    std::vector<double> out(nca * ncb * ncc * ncd, 0.0);
    for (int a = 0; a < nca; ++a)
        for (int b = 0; b < ncb; ++b) {
            const Trip ta = CT()[coff(la) + a], tb = CT()[coff(lb) + b];
            for (int cd = 0; cd < ncc * ncd; ++cd) {
                double s = 0;
                for (int ux = 0; ux <= tb.x; ++ux)
                    for (int uy = 0; uy <= tb.y; ++uy)
                        for (int uz = 0; uz <= tb.z; ++uz)
                            s += binom(tb.x, ux) * std::pow(AB[0], tb.x - ux) * binom(tb.y, uy) * std::pow(AB[1], tb.y - uy) *
                                 binom(tb.z, uz) * std::pow(AB[2], tb.z - uz) *
                                 K[(cflat(ta.x + ux, ta.y + uy, ta.z + uz) - coff(la)) * ncc * ncd + cd];
                out[(a * ncb + b) * ncc * ncd + cd] = s;
            }
        }
    return out;
}

// spherical block [(2la+1)(2lb+1)] x [(2lc+1)(2ld+1)] (projector with N_ang)
std::vector<double> eri_sph(const OBasis& B, int ia, int ib, int ic, int id) {
    const int L[4] = {B.sh[ia].L, B.sh[ib].L, B.sh[ic].L, B.sh[id].L};
    std::vector<double> cur = eri_cart(B, ia, ib, ic, id);
    int dims[4] = {ncart(L[0]), ncart(L[1]), ncart(L[2]), ncart(L[3])};
    for (int idx = 0; idx < 4; ++idx) {  // transform one index at a time
        int nd[4] = {dims[0], dims[1], dims[2], dims[3]};
        nd[idx] = nsph(L[idx]);
        std::vector<double> nxt(static_cast<std::size_t>(nd[0]) * nd[1] * nd[2] * nd[3], 0.0);
        for (int i0 = 0; i0 < dims[0]; ++i0) for (int i1 = 0; i1 < dims[1]; ++i1)
        for (int i2 = 0; i2 < dims[2]; ++i2) for (int i3 = 0; i3 < dims[3]; ++i3) {
            const int ii[4] = {i0, i1, i2, i3};
            const double v = cur[((i0 * dims[1] + i1) * dims[2] + i2) * dims[3] + i3];
            const Trip t = CT()[coff(L[idx]) + ii[idx]];
            for (int s = 0; s < nsph(L[idx]); ++s) {
                const double k = c2s().rows[L[idx]][s][ii[idx]] * angn(t.x, t.y, t.z);
                if (k == 0) continue;
                int jj[4] = {i0, i1, i2, i3};
                jj[idx] = s;
                nxt[((jj[0] * nd[1] + jj[1]) * nd[2] + jj[2]) * nd[3] + jj[3]] += k * v;
            }
        }
        cur.swap(nxt);
        std::copy(nd, nd + 4, dims);
    }
    return cur;
}

double schwarz_pair(const OBasis& B, int i, int j) {
    const auto v = eri_sph(B, i, j, i, j);
    const int n = nsph(B.sh[i].L) * nsph(B.sh[j].L);
    double m = 0;
    for (int s = 0; s < n; ++s) m = std::max(m, v[s * n + s]);
    return std::sqrt(m);
}

// ---------------- one-electron (onee_integrals.cpp) ----------------
void shape(std::vector<double>& S, int la, int lbe, double pa, double ab, double inv2p) {
    const int lt = la + lbe, nc = lbe + 1;
    S.assign((lt + 1) * nc, 0.0);
    S[0] = 1;
    if (lt >= 1) S[nc] = pa;
    for (int n = 1; n < lt; ++n) S[(n + 1) * nc] = pa * S[n * nc] + n * inv2p * S[(n - 1) * nc];
    for (int ib = 0; ib < lbe; ++ib)
        for (int ia = 0; ia <= lt - ib - 1; ++ia) S[ia * nc + ib + 1] = S[(ia + 1) * nc + ib] + ab * S[ia * nc + ib];
}
void hermite(std::vector<double>& E, int la, int lb, double qx, double a, double b) {
    const double p = a + b, PA = -b * qx / p, PB = a * qx / p, i2p = 0.5 / p;
    const int lt = la + lb, nt = lt + 1, col = lb + 1;
    std::vector<double> W((lt + 1) * col * nt, 0.0);
    auto w = [&](int i, int j, int t) -> double& { return W[(i * col + j) * nt + t]; };
    w(0, 0, 0) = std::exp(-a * b / p * qx * qx);
    for (int i = 0; i < lt; ++i)
        for (int t = 0; t <= i + 1; ++t) {
            double v = PA * w(i, 0, t);
            if (t > 0) v += i2p * w(i, 0, t - 1);
            if (t < i) v += (t + 1.0) * w(i, 0, t + 1);
            w(i + 1, 0, t) = v;
        }
    for (int j = 0; j < lb; ++j)
        for (int i = 0; i <= lt; ++i)
            for (int t = 0; t <= std::min(i + j + 1, lt); ++t) {
                double v = PB * w(i, j, t);
                if (t > 0) v += i2p * w(i, j, t - 1);
                if (t < i + j) v += (t + 1.0) * w(i, j, t + 1);
                w(i, j + 1, t) = v;
            }
    E = W;
}

void onee_block(const OBasis& B, int ia, int ib, bool st, bool vv, double nuc_eps, double zsum,
                const std::vector<double>& maxc_a, const std::vector<double>& maxc_b, std::vector<double>& S,
                std::vector<double>& T, std::vector<double>& V) {
    const OShell &A = B.sh[ia], &Bs = B.sh[ib];
    const int la = A.L, lb = Bs.L, nca = ncart(la), ncb = ncart(lb);
    S.assign(nca * ncb, 0.0); T.assign(nca * ncb, 0.0); V.assign(nca * ncb, 0.0);
    const double AB[3] = {A.c[0] - Bs.c[0], A.c[1] - Bs.c[1], A.c[2] - Bs.c[2]};
    const double ab2 = AB[0] * AB[0] + AB[1] * AB[1] + AB[2] * AB[2];
    const double thr = zsum > 0 ? nuc_eps / zsum : 0.0;
    std::vector<double> Sx, Sy, Sz, Ex, Ey, Ez;
    for (int i = 0; i < A.np; ++i)
        for (int j = 0; j < Bs.np; ++j) {
            const double a = A.e[i], b = Bs.e[j], p = a + b, chi = a * b / p, emc = std::exp(-chi * ab2);
            const double P[3] = {(a * A.c[0] + b * Bs.c[0]) / p, (a * A.c[1] + b * Bs.c[1]) / p, (a * A.c[2] + b * Bs.c[2]) / p};
            if (st) {
                const double sss = std::pow(kPi / p, 1.5) * emc;
                shape(Sx, la, lb + 2, P[0] - A.c[0], AB[0], 0.5 / p);
                shape(Sy, la, lb + 2, P[1] - A.c[1], AB[1], 0.5 / p);
                shape(Sz, la, lb + 2, P[2] - A.c[2], AB[2], 0.5 / p);
                const int nc = lb + 3;
                for (int ca = 0; ca < nca; ++ca)
                    for (int cb = 0; cb < ncb; ++cb) {
                        const Trip ta = CT()[coff(la) + ca], tb = CT()[coff(lb) + cb];
                        const double w = A.cr[i] * angn(ta.x, ta.y, ta.z) * Bs.cr[j] * angn(tb.x, tb.y, tb.z) * sss;
                        auto kin = [&](const std::vector<double>& s1, int x, int y) {
                            return b * (2 * y + 1) * s1[x * nc + y] - 2 * b * b * s1[x * nc + y + 2] -
                                   (y >= 2 ? 0.5 * y * (y - 1) * s1[x * nc + y - 2] : 0.0);
                        };
                        const double sx = Sx[ta.x * nc + tb.x], sy = Sy[ta.y * nc + tb.y], sz = Sz[ta.z * nc + tb.z];
                        S[ca * ncb + cb] += w * sx * sy * sz;
                        T[ca * ncb + cb] += w * (kin(Sx, ta.x, tb.x) * sy * sz + sx * kin(Sy, ta.y, tb.y) * sz +
                                                 sx * sy * kin(Sz, ta.z, tb.z));
                    }
            }
            if (vv) {
                if (2 * kPi / p * emc * maxc_a[i] * maxc_b[j] < thr) continue;
                const int lt = la + lb;
                std::vector<double> Rs(ccum(lt), 0.0);
                for (std::size_t K = 0; K < B.Z.size(); ++K) {
                    if (B.Z[K] == 0) continue;
                    const double pc[3] = {P[0] - B.xyz[3 * K], P[1] - B.xyz[3 * K + 1], P[2] - B.xyz[3 * K + 2]};
                    const double x = p * (pc[0] * pc[0] + pc[1] * pc[1] + pc[2] * pc[2]);
                    std::vector<double> nxt(ccum(lt), 0.0), cur(ccum(lt), 0.0);
                    for (int n = lt; n >= 0; --n) {
                        cur.assign(ccum(lt), 0.0);
                        cur[0] = std::pow(-2 * p, n) * boys(n, x);
                        for (int tot = 1; tot <= lt - n; ++tot)
                            for (int t = tot; t >= 0; --t)
                                for (int u = tot - t; u >= 0; --u) {
                                    const int v = tot - t - u;
                                    double val;
                                    if (t) val = pc[0] * nxt[cflat(t - 1, u, v)] + (t > 1 ? (t - 1) * nxt[cflat(t - 2, u, v)] : 0);
                                    else if (u) val = pc[1] * nxt[cflat(t, u - 1, v)] + (u > 1 ? (u - 1) * nxt[cflat(t, u - 2, v)] : 0);
                                    else val = pc[2] * nxt[cflat(t, u, v - 1)] + (v > 1 ? (v - 1) * nxt[cflat(t, u, v - 2)] : 0);
                                    cur[cflat(t, u, v)] = val;
                                }
                        nxt.swap(cur);
                    }
                    for (int r = 0; r < ccum(lt); ++r) Rs[r] += B.Z[K] * nxt[r];
                }
                hermite(Ex, la, lb, AB[0], a, b);
                hermite(Ey, la, lb, AB[1], a, b);
                hermite(Ez, la, lb, AB[2], a, b);
                const int nt = lt + 1, col = lb + 1;
                for (int ca = 0; ca < nca; ++ca)
                    for (int cb = 0; cb < ncb; ++cb) {
                        const Trip ta = CT()[coff(la) + ca], tb = CT()[coff(lb) + cb];
                        double s = 0;
                        for (int t = 0; t <= ta.x + tb.x; ++t)
                            for (int u = 0; u <= ta.y + tb.y; ++u)
                                for (int v = 0; v <= ta.z + tb.z; ++v)
                                    s += Ex[(ta.x * col + tb.x) * nt + t] * Ey[(ta.y * col + tb.y) * nt + u] *
                                         Ez[(ta.z * col + tb.z) * nt + v] * Rs[cflat(t, u, v)];
                        V[ca * ncb + cb] += -2 * kPi / p * A.cr[i] * angn(ta.x, ta.y, ta.z) * Bs.cr[j] * angn(tb.x, tb.y, tb.z) * s;
                    }
            }
        }
}

thread_local std::string g_err;

}  // namespace

extern "C" {

const char* orc_last_error() { return g_err.c_str(); }

double orc_boys(int n, double x) { return boys(n, x); }

void orc_rys(int n, double t, double* r, double* w) { rys(n, t, r, w); }

void* orc_basis_create(int ns, const double* centers, const int* L, const int* np, const double* ex,
                       const double* co, int na, const int* Z, const double* xyz) {
    return new OBasis(make_basis(ns, centers, L, np, ex, co, na, Z, xyz));
}
void orc_basis_destroy(void* h) { delete static_cast<OBasis*>(h); }
int orc_basis_n_sph(void* h) { return static_cast<OBasis*>(h)->M; }

int orc_eri_sph_block(void* h, int a, int b, int c, int d, double* out) {
    const auto v = eri_sph(*static_cast<OBasis*>(h), a, b, c, d);
    std::copy(v.begin(), v.end(), out);
    return 0;
}

int orc_schwarz(void* h, double* out) {
    const OBasis& B = *static_cast<OBasis*>(h);
    const int ns = static_cast<int>(B.sh.size());
    for (int i = 0; i < ns; ++i)
        for (int j = 0; j <= i; ++j) out[i * (i + 1) / 2 + j] = schwarz_pair(B, i, j);
    return 0;
}

// J and K (full 8-fold sum over unique shell quartets with Schwarz gate
// Q_ab Q_cd >= tau); J[a,b] = sum (ab|cd) D[c,d], K[a,c] = sum (ab|cd) D[b,d].
int orc_jk(void* h, const double* D, double tau, double* J, double* K) {
    const OBasis& B = *static_cast<OBasis*>(h);
    const int ns = static_cast<int>(B.sh.size()), M = B.M;
    std::vector<double> Q(ns * (ns + 1) / 2);
    orc_schwarz(h, Q.data());
    std::fill(J, J + M * M, 0.0);
    std::fill(K, K + M * M, 0.0);
    std::vector<std::pair<int, int>> pairs;
    for (int i = 0; i < ns; ++i) for (int j = 0; j <= i; ++j) pairs.push_back({i, j});
    for (std::size_t p = 0; p < pairs.size(); ++p)
        for (std::size_t q = 0; q <= p; ++q) {
            const auto [a, b] = pairs[p];
            const auto [c, d] = pairs[q];
            if (!(Q[p] * Q[q] >= tau)) continue;
            const auto v = eri_sph(B, a, b, c, d);
            const int na = nsph(B.sh[a].L), nb = nsph(B.sh[b].L), nc = nsph(B.sh[c].L), nd = nsph(B.sh[d].L);
            const int a0 = B.sh[a].sph, b0 = B.sh[b].sph, c0 = B.sh[c].sph, d0 = B.sh[d].sph;
            // every distinct permutation of the block contributes once
            const int idx[4] = {a, b, c, d};
            (void)idx;
            for (int ia = 0; ia < na; ++ia) for (int ib = 0; ib < nb; ++ib)
            for (int ic = 0; ic < nc; ++ic) for (int id = 0; id < nd; ++id) {
                const double x = v[((ia * nb + ib) * nc + ic) * nd + id];
                const int A_ = a0 + ia, B_ = b0 + ib, C_ = c0 + ic, D_ = d0 + id;
                // enumerate the 8 index permutations, skipping duplicates at shell level
                const int perm[8][4] = {{A_, B_, C_, D_}, {B_, A_, C_, D_}, {A_, B_, D_, C_}, {B_, A_, D_, C_},
                                        {C_, D_, A_, B_}, {D_, C_, A_, B_}, {C_, D_, B_, A_}, {D_, C_, B_, A_}};
                const bool use[8] = {true, a != b, c != d, a != b && c != d, p != q, p != q && c != d,
                                     p != q && a != b, p != q && a != b && c != d};
                for (int k = 0; k < 8; ++k) {
                    if (!use[k]) continue;
                    const int* P = perm[k];
                    J[P[0] * M + P[1]] += x * D[P[2] * M + P[3]];
                    K[P[0] * M + P[2]] += x * D[P[1] * M + P[3]];
                }
            }
        }
    return 0;
}

// S, T, V spherical with the reference's default screening when screening != 0.
int orc_onee(void* h, int screening, double* S, double* T, double* V) {
    const OBasis& B = *static_cast<OBasis*>(h);
    const int ns = static_cast<int>(B.sh.size()), M = B.M;
    std::fill(S, S + M * M, 0.0);
    std::fill(T, T + M * M, 0.0);
    std::fill(V, V + M * M, 0.0);
    double zsum = 0;
    for (int z : B.Z) zsum += std::fabs(static_cast<double>(z));
    const double eps = screening ? 1e-15 : 0.0;
    auto c0 = [&](const OShell& s, int i) { return s.cr[i] * angn(s.L, 0, 0); };
    std::vector<std::vector<double>> maxc(ns);
    for (int s = 0; s < ns; ++s) {
        double mx = 0;
        for (int x = B.sh[s].L; x >= 0; --x) for (int y = B.sh[s].L - x; y >= 0; --y) mx = std::max(mx, angn(x, y, B.sh[s].L - x - y));
        for (int i = 0; i < B.sh[s].np; ++i) maxc[s].push_back(std::fabs(B.sh[s].cr[i]) * mx);
    }
    std::vector<double> Sc, Tc, Vc;
    for (int i = 0; i < ns; ++i)
        for (int j = 0; j <= i; ++j) {
            int a = i, b = j;
            if (B.sh[b].L > B.sh[a].L) std::swap(a, b);
            const OShell &A = B.sh[a], &Bs = B.sh[b];
            const double r2 = (A.c[0] - Bs.c[0]) * (A.c[0] - Bs.c[0]) + (A.c[1] - Bs.c[1]) * (A.c[1] - Bs.c[1]) +
                              (A.c[2] - Bs.c[2]) * (A.c[2] - Bs.c[2]);
            bool dov = true;
            if (eps > 0) {  // group-pair decay screening (onee_matrices.cpp:96-216)
                double amin_a = 1e300, amin_b = 1e300, Ka = 0, Kb = 0, bound = 0;
                for (int k = 0; k < A.np; ++k) { amin_a = std::min(amin_a, A.e[k]); Ka += std::fabs(c0(A, k)) * std::pow(kPi / A.e[k], 0.75); }
                for (int k = 0; k < Bs.np; ++k) { amin_b = std::min(amin_b, Bs.e[k]); Kb += std::fabs(c0(Bs, k)) * std::pow(kPi / Bs.e[k], 0.75); }
                const double mu = amin_a * amin_b / (amin_a + amin_b);
                if (Ka * Kb * std::exp(-mu * r2) < eps) continue;
                for (int x = 0; x < A.np; ++x)
                    for (int y = 0; y < Bs.np; ++y) {
                        const double p = A.e[x] + Bs.e[y];
                        bound += std::fabs(c0(A, x) * c0(Bs, y)) * std::pow(kPi / p, 1.5) * std::exp(-A.e[x] * Bs.e[y] / p * r2);
                    }
                dov = bound >= eps;
            }
            onee_block(B, a, b, true, dov, eps, zsum, maxc[a], maxc[b], Sc, Tc, Vc);
            const int la = A.L, lb = Bs.L, nca = ncart(la), ncb = ncart(lb);
            for (int sa = 0; sa < nsph(la); ++sa)
                for (int sb = 0; sb < nsph(lb); ++sb) {
                    double vs = 0, vt = 0, vv = 0;
                    for (int ca = 0; ca < nca; ++ca)
                        for (int cb = 0; cb < ncb; ++cb) {
                            const double k = c2s().rows[la][sa][ca] * c2s().rows[lb][sb][cb];
                            vs += k * Sc[ca * ncb + cb];
                            vt += k * Tc[ca * ncb + cb];
                            vv += k * Vc[ca * ncb + cb];
                        }
                    const int r = A.sph + sa, c = Bs.sph + sb;
                    S[r * M + c] = S[c * M + r] = vs;
                    T[r * M + c] = T[c * M + r] = vt;
                    V[r * M + c] = V[c * M + r] = vv;
                }
        }
    return 0;
}

}  // extern "C"
