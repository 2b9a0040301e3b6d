// Host-side generation of the interpolation tables the device kernels read:
// the Boys function F_n(x) on a 0.01 grid and the Rys roots/weights per root
// count on the same grid, plus the large-T Hermite asymptotic constants.
#pragma once

#include <vector>

namespace tlno_gpu {

// Boys table: F_n(k * kBoysDx) for k = 0..kBoysRows-1 and n = 0..kBoysOrders-1,
// stored grid-major (row k holds all orders contiguously) so that one Taylor
// evaluation reads a single contiguous run.
constexpr int kBoysOrders = 40;       // orders 0..39 (Taylor needs n+5)
constexpr int kBoysGrid = 4000;       // x in [0, 40]
constexpr int kBoysRows = kBoysGrid + 8;
constexpr double kBoysDx = 0.01;
constexpr double kBoysXMax = 40.0;

// Rys tables: root counts 1..kRysMaxN, grid T = k * 0.01 for
// k = 0 .. rows(N)-1 with rows(N) = int(tmax(N) * 100) + 7, layout
// [k * N + n] for roots (t^2) and weights separately.
constexpr int kRysMaxN = 9;
constexpr double kRysDx = 0.01;

struct HostTables {
    std::vector<double> boys;                 // kBoysRows * kBoysOrders
    double rys_tmax[kRysMaxN + 1] = {0};
    int rys_rows[kRysMaxN + 1] = {0};
    std::vector<double> rys_roots[kRysMaxN + 1];
    std::vector<double> rys_weights[kRysMaxN + 1];
    // Positive Gauss-Hermite nodes squared and weights for 2N-point rules.
    double herm_root2[kRysMaxN + 1][kRysMaxN] = {{0}};
    double herm_weight[kRysMaxN + 1][kRysMaxN] = {{0}};
};

// FP32 Rys tables of the mixed-precision kernels for root counts
// 1..kRys32MaxN: on each interval [k h, (k+1) h), h = 1 / kRys32PerUnit, of
// [0, tmax(N)) the N roots and N weights are degree-kRys32Deg polynomials in
// u = T / h - k - 1/2 in [-1/2, 1/2), interpolating the accurate rule at the
// Chebyshev nodes of the interval (near-minimax; error below 2e-10 times the
// sixth derivative, far under FP32 rounding).  Record k holds
// (kRys32Deg + 1) coefficient rows of 2N floats (N roots, then N weights),
// lowest power first: [(k * (kRys32Deg + 1) + j) * 2N + i].  Small enough to
// sit in shared memory (N = 3: 24.8 KB).
constexpr int kRys32MaxN = 3;
constexpr int kRys32PerUnit = 4;
constexpr int kRys32Deg = 5;
int rys32_intervals(int n);
std::vector<float> rys32_table(int n);

// Rows of the Rys grid of root count n (tmax(n) / 0.01 + 7 guard rows for
// the 5-point stencil).
int rys_rows(int n);

// Builds (once per process, thread-safe) and returns the tables.
const HostTables& host_tables();

// Accurate (non-tabulated) generators, exposed for self-checks.
void boys_quadrature(int max_n, double x, double* out);
bool rys_rule_accurate(int n, double t, double* roots, double* weights);
double rys_tmax(int n);

}  // namespace tlno_gpu
