// Test program of the C++ shim (tests/shim/tlno_b200_shim.hpp): builds the
// reference's std::vector<Shell> with its own make_shell from a shell file,
// runs the reference's fock::build_coulomb_j / build_exchange_k /
// build_rhf_g and its EriDirectJKIncrementalState, then the same calls
// through the shim on the GPU, and prints the largest differences as one
// JSON line.  Built by oracle/build_ref.sh against the reference headers
// (linking the compiled reference and the engine); run by
// tests/test_gpu_shim.py.
//
// Shell file: n_shells, then per shell "x y z L nprim e_1..e_n c_1..c_n".
#include <omp.h>

#include <cmath>
#include <cstdio>
#include <fstream>
#include <random>
#include <string>
#include <vector>

#include "core/basis/cartesian_shells.hpp"
#include "core/shell/shell_contract.hpp"
#include "tests/shim/tlno_b200_shim.hpp"

namespace {

double maxdiff(const std::vector<double>& a, const std::vector<double>& b) {
    double m = 0.0;
    for (std::size_t i = 0; i < a.size(); ++i) m = std::max(m, std::fabs(a[i] - b[i]));
    return m;
}

}  // namespace

int run(int argc, char** argv);

int main(int argc, char** argv) {
    // the reference's G and K endpoints refuse more than one OpenMP thread
    // (rys_engine.ipp:16853-16857)
    omp_set_num_threads(1);
    try {
        return run(argc, argv);
    } catch (const std::exception& e) {
        std::string msg = e.what();
        for (char& c : msg)
            if (c == '"') c = '\'';
        std::printf("{\"error\": \"%s\"}\n", msg.c_str());
        return 3;
    }
}

int run(int argc, char** argv) {
    if (argc < 2) {
        std::fprintf(stderr, "usage: shim_test SHELL_FILE [schwarz] [density_threshold]\n");
        return 2;
    }
    const double tau = argc > 2 ? std::stod(argv[2]) : 1e-12;
    const double tden = argc > 3 ? std::stod(argv[3]) : 1e-10;
    namespace basis = tlno::core::basis;
    namespace fock = tlno::integrals::twoe::fock;
    namespace twoe = tlno::integrals::twoe;
    std::ifstream in(argv[1]);
    int ns = 0;
    in >> ns;
    std::vector<basis::Shell> shells;
    int M = 0;
    for (int s = 0; s < ns; ++s) {
        double x, y, z;
        int L, np;
        in >> x >> y >> z >> L >> np;
        basis::RawShell raw;
        raw.label = "shell";
        raw.exponents.resize(np);
        raw.coefficients.resize(np);
        for (auto& e : raw.exponents) in >> e;
        for (auto& c : raw.coefficients) in >> c;
        for (const auto& ang : basis::detail::cartesian_tuples_for_total_L(L)) {
            raw.ang = ang;
            shells.push_back(tlno::core::shell::make_shell(raw, {x, y, z}));
        }
        M += 2 * L + 1;
    }
    // D = C C^T, C M x (M / 5) with N(0,1)/sqrt(M) entries (seed 7)
    const int nocc = std::max(1, M / 5);
    std::mt19937_64 rng(7);
    std::normal_distribution<double> nd(0.0, 1.0 / std::sqrt(double(M)));
    std::vector<double> C(static_cast<std::size_t>(M) * nocc), D(static_cast<std::size_t>(M) * M, 0.0);
    for (auto& c : C) c = nd(rng);
    for (int i = 0; i < M; ++i)
        for (int j = 0; j <= i; ++j) {
            double v = 0.0;
            for (int k = 0; k < nocc; ++k) v += C[i * nocc + k] * C[j * nocc + k];
            D[static_cast<std::size_t>(i) * M + j] = D[static_cast<std::size_t>(j) * M + i] = v;
        }
    fock::ScreeningOptions opt;
    opt.integral_threshold = tau;
    fock::ScreeningOptions dopt = opt;
    dopt.density_threshold = tden;

    const auto rplan = fock::build_direct_plan(shells, opt);
    const auto gplan = tlno_b200::build_direct_plan(shells, opt);
    double dj = maxdiff(fock::build_coulomb_j(rplan, D, opt).j, tlno_b200::build_coulomb_j(gplan, D, opt).j);
    double dk = maxdiff(fock::build_exchange_k(rplan, D, opt).k, tlno_b200::build_exchange_k(gplan, D, opt).k);
    double dg = maxdiff(fock::build_rhf_g(rplan, D, opt).g, tlno_b200::build_rhf_g(gplan, D, opt).g);
    double dgs = maxdiff(fock::build_rhf_g(rplan, D, dopt).g, tlno_b200::build_rhf_g(gplan, D, dopt).g);
    // the error texts are the reference's
    std::string err_ref, err_gpu;
    std::vector<double> bad = D;
    bad[1] += 1e-3;
    try { (void)fock::build_coulomb_j(rplan, bad, opt); } catch (const std::exception& e) { err_ref = e.what(); }
    try { (void)tlno_b200::build_coulomb_j(gplan, bad, opt); } catch (const std::exception& e) { err_gpu = e.what(); }
    // incremental state over a short sequence
    twoe::EriDirectJKIncrementalOptions io;
    io.base_options.schwarz_threshold = tau;
    io.exact_rebuild_interval = 3;
    io.delta_density_threshold = 1e-12;
    const auto eplan = twoe::build_eri_packed_plan_for_G_rys(shells, io.base_options);
    twoe::EriDirectJKIncrementalState rs(eplan, io);
    tlno_b200::EriDirectJKIncrementalState gs(gplan, io);
    double dinc = 0.0;
    bool same_status = true;
    std::vector<double> Dk = D;
    for (int step = 0; step < 5; ++step) {
        for (int i = 0; i < M; ++i)
            for (int j = 0; j <= i; ++j) {
                const double v = 1e-3 * std::cos(0.1 * (i + 2 * j + step));
                Dk[static_cast<std::size_t>(i) * M + j] += v;
                if (i != j) Dk[static_cast<std::size_t>(j) * M + i] += v;
            }
        const auto a = rs.update(Dk);
        const auto b = gs.update(Dk);
        same_status = same_status && a == b;
        dinc = std::max(dinc, maxdiff(rs.g(), gs.g()));
    }
    const auto rc = rs.counters(), gc = gs.counters();
    same_status = same_status && rc.updates == gc.updates && rc.exact_rebuilds == gc.exact_rebuilds &&
                  rc.incremental_updates == gc.incremental_updates;
    std::printf("{\"M\": %d, \"J\": %.3e, \"K\": %.3e, \"G\": %.3e, \"G_density_screened\": %.3e, "
                "\"incremental_G\": %.3e, \"incremental_status_match\": %s, \"same_error_text\": %s, "
                "\"error_text\": \"%s\"}\n",
                M, dj, dk, dg, dgs, dinc, same_status ? "true" : "false",
                (err_ref == err_gpu && !err_ref.empty()) ? "true" : "false", err_gpu.c_str());
    const bool ok = dj < 1e-12 && dk < 1e-12 && dg < 1e-12 && dgs < 1e-12 && dinc < 1e-12 && same_status &&
                    err_ref == err_gpu && !err_ref.empty();
    return ok ? 0 : 1;
}
