// C++ shim a maintainer of the reference adds to keep its J/K signatures and
// run them on the B200 engine: the same functions, argument meaning, result
// types and exception texts as integrals/two_electron/fock/jk_direct.hpp:
// 46-96 and fock/eri_direct_jk.hpp:36-135, forwarding to the C ABI of
// include/tlno_gpu.h.  Header-only; compiled against the reference's own
// headers by tests/shim/shim_test.cpp.
#pragma once

#include <cstdint>
#include <memory>
#include <stdexcept>
#include <vector>

#include "include/tlno_gpu.h"
#include "integrals/two_electron/fock/eri_direct_jk.hpp"
#include "integrals/two_electron/fock/jk_direct.hpp"

namespace tlno_b200 {

namespace fock = tlno::integrals::twoe::fock;
namespace twoe = tlno::integrals::twoe;

inline void check(int rc) {
    if (rc < 0) throw std::runtime_error(tlno_gpu_last_error());
}

inline tlno_gpu_screening to_c(const fock::ScreeningOptions& o, double mixed_threshold = 1e-9) {
    return tlno_gpu_screening{o.integral_threshold, o.primitive_fastschwarz_threshold, o.decay_threshold,
                              o.density_threshold, mixed_threshold};
}

// The counterpart of fock::DirectPlan: an immutable shared handle.
struct DirectPlan {
    twoe::EriPackedPlanProfile profile;
    std::shared_ptr<tlno_gpu_context> ctx;
};

// fock::build_direct_plan over the reference's std::vector<Shell> (one record
// per Cartesian component, make_shell-normalised).
inline DirectPlan build_direct_plan(const std::vector<tlno::core::basis::Shell>& basis,
                                    const fock::ScreeningOptions& options = {}, int device = 0) {
    std::vector<double> centers, exps, coefs;
    std::vector<int> ang, nprim;
    for (const auto& s : basis) {
        centers.insert(centers.end(), s.center.begin(), s.center.end());
        ang.insert(ang.end(), s.ang.begin(), s.ang.end());
        nprim.push_back(static_cast<int>(s.primitives.size()));
        for (const auto& p : s.primitives) {
            exps.push_back(p.exponent);
            coefs.push_back(p.coefficient);
        }
    }
    tlno_gpu_context* raw = nullptr;
    check(tlno_gpu_create_from_components(static_cast<int>(basis.size()), centers.data(), ang.data(), nprim.data(),
                                          exps.data(), coefs.data(), 0, nullptr, nullptr, device, &raw));
    DirectPlan plan;
    plan.ctx = std::shared_ptr<tlno_gpu_context>(raw, tlno_gpu_destroy);
    const tlno_gpu_screening s = to_c(options);
    check(tlno_gpu_plan(plan.ctx.get(), &s));
    tlno_gpu_profile p{};
    check(tlno_gpu_plan_profile(plan.ctx.get(), &p));
    plan.profile.M = p.M;
    plan.profile.shell_groups = static_cast<std::uint64_t>(p.n_shells);
    plan.profile.pair_groups = static_cast<std::uint64_t>(p.shell_pairs);
    return plan;
}

inline std::vector<double> run(const DirectPlan& plan, const std::vector<double>& density,
                               const fock::ScreeningOptions& options, int want) {
    const std::size_t m = static_cast<std::size_t>(plan.profile.M);
    if (density.size() != m * m)
        throw std::runtime_error("eri_ao_tensor_hgp: density must be spherical M x M row-major.");
    std::vector<double> out(m * m);
    const tlno_gpu_screening s = to_c(options);
    double* J = want == TLNO_GPU_WANT_J ? out.data() : nullptr;
    double* K = want == TLNO_GPU_WANT_K ? out.data() : nullptr;
    double* G = want == TLNO_GPU_WANT_G ? out.data() : nullptr;
    check(tlno_gpu_jk_with_options(plan.ctx.get(), density.data(), J, K, G, want, &s));
    return out;
}

inline fock::CoulombJResult build_coulomb_j(const DirectPlan& plan, const std::vector<double>& density,
                                            const fock::ScreeningOptions& options) {
    fock::CoulombJResult r;
    r.j = run(plan, density, options, TLNO_GPU_WANT_J);
    r.M = plan.profile.M;
    return r;
}

inline fock::ExchangeKResult build_exchange_k(const DirectPlan& plan, const std::vector<double>& density,
                                              const fock::ScreeningOptions& options) {
    fock::ExchangeKResult r;
    r.k = run(plan, density, options, TLNO_GPU_WANT_K);
    r.M = plan.profile.M;
    return r;
}

inline fock::DirectResult build_rhf_g(const DirectPlan& plan, const std::vector<double>& density,
                                      const fock::ScreeningOptions& options) {
    fock::DirectResult r;
    r.g = run(plan, density, options, TLNO_GPU_WANT_G);
    r.M = plan.profile.M;
    return r;
}

// EriDirectJKIncrementalState with the reference's options and results.
class EriDirectJKIncrementalState {
public:
    EriDirectJKIncrementalState(const DirectPlan& plan, const twoe::EriDirectJKIncrementalOptions& o)
        : plan_(plan) {
        tlno_gpu_incremental_options c{};
        c.base_options = tlno_gpu_screening{o.base_options.schwarz_threshold,
                                            o.base_options.primitive_fastschwarz_threshold,
                                            o.base_options.decay_threshold, o.base_options.density_threshold, 1e-9};
        c.exact_rebuild_interval = o.exact_rebuild_interval;
        c.delta_density_threshold = o.delta_density_threshold;
        c.use_first_delta_density_threshold = o.use_first_delta_density_threshold ? 1 : 0;
        c.first_delta_density_threshold = o.first_delta_density_threshold;
        tlno_gpu_incremental* raw = nullptr;
        check(tlno_gpu_incremental_create(plan_.ctx.get(), &c, &raw));
        st_ = std::shared_ptr<tlno_gpu_incremental>(raw, tlno_gpu_incremental_destroy);
    }
    twoe::EriDirectJKUpdateStatus update(const std::vector<double>& density, bool force_exact_rebuild = false) {
        const std::size_t m = static_cast<std::size_t>(plan_.profile.M);
        if (density.size() != m * m)
            throw std::runtime_error(
                "eri_ao_tensor_hgp: incremental density must be spherical M x M row-major.");
        const int rc = tlno_gpu_incremental_update(st_.get(), density.data(), force_exact_rebuild ? 1 : 0, 0);
        check(rc);
        g_.resize(m * m);
        check(tlno_gpu_incremental_g(st_.get(), g_.data(), 0));
        return static_cast<twoe::EriDirectJKUpdateStatus>(rc);
    }
    const std::vector<double>& g() const noexcept { return g_; }
    twoe::EriDirectJKIncrementalCounters counters() const {
        tlno_gpu_incremental_info i{};
        check(tlno_gpu_incremental_info_get(st_.get(), &i));
        twoe::EriDirectJKIncrementalCounters c;
        c.updates = i.updates;
        c.exact_rebuilds = i.exact_rebuilds;
        c.incremental_updates = i.incremental_updates;
        c.skipped_updates = i.skipped_updates;
        return c;
    }

private:
    DirectPlan plan_;
    std::shared_ptr<tlno_gpu_incremental> st_;
    std::vector<double> g_;
};

}  // namespace tlno_b200
