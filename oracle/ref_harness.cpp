// TEST INFRASTRUCTURE ONLY -- never linked into the shipped library.
//
// C-ABI harness around the UNMODIFIED origo-tlno reference engine, compiled
// from its own sources by oracle/build_ref.sh into oracle/_ref/libtlno_ref.so.
// Only tests/, __graft_entry__.smoke() and bench.py (cpu_baseline leg and the
// `--impl reference` arm) may load it, always as the checker or as the timed
// CPU baseline, never as the product path.
//
// This translation unit includes the reference's Rys engine the same way the
// reference's own experiment hosts do (benchmarks/two_electron_engine/src/
// rys_native_lane_ablation.cpp:8-9): it defines TLNO_BUILD_RYS_AUDIT and
// includes integrals/two_electron/rys/rys_engine.ipp, which makes the
// engine's internal per-quartet producer (compute_quartet_block_rys_impl,
// rys_engine.ipp:13754) and its final spherical projector
// (get_final_sph_pair_projector, rys_engine.ipp:1844) reachable for a
// per-ERI oracle.  For the AVX2 route this macro changes no arithmetic
// (TLNO_NATIVE_LEAN_BASIS_PLAN only applies to the portable route).
//
// Every entry point returns 0 on success and a negative value on failure;
// ref_last_error() returns the exception text of the last failure.

#define TLNO_BUILD_RYS_AUDIT 1
#include "integrals/two_electron/rys/rys_engine.ipp"

#include "core/basis/cartesian_shells.hpp"
#include "core/math/general_math.hpp"
#include "core/shell/shell_contract.hpp"
#include "integrals/one_electron/onee_matrices.hpp"
#include "integrals/two_electron/fock/eri_direct_jk.hpp"
#include "integrals/two_electron/fock/jk_direct.hpp"

#include <chrono>
#include <cstring>
#include <memory>
#include <string>

using namespace tlno::integrals::twoe;

namespace {

namespace basis_ns = tlno::core::basis;

thread_local std::string g_ref_error;

struct RefBasis {
    basis_ns::BasisBuildResult build;  // one Shell per Cartesian component
    std::vector<int> shell_L;          // per contracted shell
    std::vector<int> shell_first_comp; // first Cartesian component index
    int n_sph = 0;
};

template <class F>
int guarded(F&& f) {
    try {
        f();
        return 0;
    } catch (const std::exception& e) {
        g_ref_error = e.what();
    } catch (...) {
        g_ref_error = "unknown exception";
    }
    return -1;
}

// Expands one contracted shell into its Cartesian components in the
// reference's descending-lex order (core/basis/cartesian_shells.hpp:17-28)
// and normalises each with the reference's make_shell
// (core/shell/shell_contract.cpp:41-48).
void add_shell(RefBasis& rb, const double* center, int L, int nprim,
               const double* exps, const double* coefs) {
    const auto tuples = basis_ns::detail::cartesian_tuples_for_total_L(L);
    rb.shell_L.push_back(L);
    rb.shell_first_comp.push_back(static_cast<int>(rb.build.basis.size()));
    for (const auto& ang : tuples) {
        basis_ns::RawShell raw;
        raw.label = "shell";
        raw.ang = ang;
        raw.exponents.assign(exps, exps + nprim);
        raw.coefficients.assign(coefs, coefs + nprim);
        rb.build.basis.push_back(tlno::core::shell::make_shell(
            raw, {center[0], center[1], center[2]}));
    }
    rb.n_sph += 2 * L + 1;
}

const ContractedShellGroupH& group_of(const std::vector<ContractedShellGroupH>& g,
                                      int shell) {
    return g.at(static_cast<std::size_t>(shell));
}

}  // namespace

extern "C" {

const char* ref_last_error() { return g_ref_error.c_str(); }

// Shells in SoA form: centers[3*n], L[n], nprim[n], exponents and raw
// contraction coefficients packed back to back (prim_offset implied by nprim).
// Atoms: natom charges and centres (bohr) for the nuclear attraction.
void* ref_basis_create(int n_shells, const double* centers, const int* L,
                       const int* nprim, const double* exps,
                       const double* coefs, int natom, const int* Z,
                       const double* atom_xyz) {
    RefBasis* out = nullptr;
    const int rc = guarded([&] {
        auto rb = std::make_unique<RefBasis>();
        std::size_t off = 0;
        for (int s = 0; s < n_shells; ++s) {
            add_shell(*rb, centers + 3 * s, L[s], nprim[s], exps + off,
                      coefs + off);
            off += static_cast<std::size_t>(nprim[s]);
        }
        for (int a = 0; a < natom; ++a) {
            rb->build.nuclear_charges.push_back(Z[a]);
            rb->build.nuclear_centers.push_back(
                {atom_xyz[3 * a], atom_xyz[3 * a + 1], atom_xyz[3 * a + 2]});
            rb->build.electron_count += Z[a];
        }
        out = rb.release();
    });
    return rc == 0 ? out : nullptr;
}

void ref_basis_destroy(void* h) { delete static_cast<RefBasis*>(h); }

int ref_basis_n_sph(void* h) { return static_cast<RefBasis*>(h)->n_sph; }

int ref_basis_n_cart(void* h) {
    return static_cast<int>(static_cast<RefBasis*>(h)->build.basis.size());
}

// Normalised per-component coefficients exactly as make_shell stores them:
// out[k] for component k, primitive p at out[k*max_prim + p].
int ref_basis_component_coefs(void* h, int max_prim, double* out) {
    return guarded([&] {
        const auto& b = static_cast<RefBasis*>(h)->build.basis;
        for (std::size_t k = 0; k < b.size(); ++k)
            for (std::size_t p = 0; p < b[k].primitives.size(); ++p)
                out[k * static_cast<std::size_t>(max_prim) + p] =
                    b[k].primitives[p].coefficient;
    });
}

// Spherical S, T, V (M x M row-major) through the reference's public
// build_one_electron_spherical_matrices (onee_matrices.cpp:622-627).
int ref_onee_sph(void* h, int screening, double* S, double* T, double* V) {
    return guarded([&] {
        auto* rb = static_cast<RefBasis*>(h);
        tlno::integrals::onee::set_onee_screening_enabled(screening != 0);
        const auto m =
            tlno::integrals::onee::build_one_electron_spherical_matrices(rb->build);
        tlno::integrals::onee::set_onee_screening_enabled(true);
        const std::size_t n = m.overlap.values.size();
        std::memcpy(S, m.overlap.values.data(), n * sizeof(double));
        std::memcpy(T, m.kinetic.values.data(), n * sizeof(double));
        std::memcpy(V, m.nuclear.values.data(), n * sizeof(double));
    });
}

// Cartesian S, T, V (ncart x ncart) through build_one_electron_matrices.
int ref_onee_cart(void* h, int screening, double* S, double* T, double* V) {
    return guarded([&] {
        auto* rb = static_cast<RefBasis*>(h);
        tlno::integrals::onee::set_onee_screening_enabled(screening != 0);
        const auto m = tlno::integrals::onee::build_one_electron_matrices(rb->build);
        tlno::integrals::onee::set_onee_screening_enabled(true);
        const std::size_t n = m.overlap.values.size();
        std::memcpy(S, m.overlap.values.data(), n * sizeof(double));
        std::memcpy(T, m.kinetic.values.data(), n * sizeof(double));
        std::memcpy(V, m.nuclear.values.data(), n * sizeof(double));
    });
}

// J, K and G = J - K/2 through the public facade (fock/jk_direct.hpp:46-96).
// Any output pointer may be null.  The plan is built outside any timing.
int ref_jk(void* h, const double* density, double schwarz_threshold,
           double density_threshold, double* J, double* K, double* G) {
    return guarded([&] {
        namespace fock = tlno::integrals::twoe::fock;
        auto* rb = static_cast<RefBasis*>(h);
        fock::ScreeningOptions opt;
        opt.integral_threshold = schwarz_threshold;
        opt.density_threshold = density_threshold;
        const fock::DirectPlan plan = fock::build_direct_plan(rb->build.basis, opt);
        const std::size_t m = static_cast<std::size_t>(plan.profile.M);
        std::vector<double> d(density, density + m * m);
        if (J) {
            const auto r = fock::build_coulomb_j(plan, d, opt);
            std::memcpy(J, r.j.data(), m * m * sizeof(double));
        }
        if (K) {
            const auto r = fock::build_exchange_k(plan, d, opt);
            std::memcpy(K, r.k.data(), m * m * sizeof(double));
        }
        if (G) {
            const auto r = fock::build_rhf_g(plan, d, opt);
            std::memcpy(G, r.g.data(), m * m * sizeof(double));
        }
    });
}

// J, K and G with every field of the reference's fock::ScreeningOptions
// (fock/jk_direct.hpp:18-24): the plan is built with the same options and
// each endpoint receives them, as a caller of the public facade does.
int ref_jk_opts(void* h, const double* density, double schwarz_threshold,
                double primitive_fastschwarz_threshold, double decay_threshold,
                double density_threshold, double* J, double* K, double* G) {
    return guarded([&] {
        namespace fock = tlno::integrals::twoe::fock;
        auto* rb = static_cast<RefBasis*>(h);
        fock::ScreeningOptions opt;
        opt.integral_threshold = schwarz_threshold;
        opt.primitive_fastschwarz_threshold = primitive_fastschwarz_threshold;
        opt.decay_threshold = decay_threshold;
        opt.density_threshold = density_threshold;
        const fock::DirectPlan plan = fock::build_direct_plan(rb->build.basis, opt);
        const std::size_t m = static_cast<std::size_t>(plan.profile.M);
        std::vector<double> d(density, density + m * m);
        if (J) {
            const auto r = fock::build_coulomb_j(plan, d, opt);
            std::memcpy(J, r.j.data(), m * m * sizeof(double));
        }
        if (K) {
            const auto r = fock::build_exchange_k(plan, d, opt);
            std::memcpy(K, r.k.data(), m * m * sizeof(double));
        }
        if (G) {
            const auto r = fock::build_rhf_g(plan, d, opt);
            std::memcpy(G, r.g.data(), m * m * sizeof(double));
        }
    });
}

// G = J - K/2 through the compatibility endpoint build_jk_direct_for_G_rys
// (fock/eri_direct_jk.hpp:36-39) on an EriPackedPlan.
int ref_jk_compat(void* h, const double* density, double schwarz_threshold,
                  double density_threshold, double* G) {
    return guarded([&] {
        auto* rb = static_cast<RefBasis*>(h);
        EriPackedBuildOptions opt;
        opt.schwarz_threshold = schwarz_threshold;
        opt.density_threshold = density_threshold;
        const EriPackedPlan plan = build_eri_packed_plan_for_G_rys(rb->build.basis, opt);
        const std::size_t m = static_cast<std::size_t>(plan.profile.M);
        std::vector<double> d(density, density + m * m);
        const auto r = build_jk_direct_for_G_rys(plan, d, opt);
        std::memcpy(G, r.g.data(), m * m * sizeof(double));
    });
}

// ERI checksum stream (build_eri_packed_for_G_rys, twoe_integrals.hpp:117,
// the endpoint benchmarks/two_electron_engine/src/twoe_timing.cpp times):
// the sum of every canonical unique spherical ERI that survives the screen.
// Also returns the plan's profile counters.
int ref_eri_checksum(void* h, double schwarz_threshold, double* checksum,
                     double* seconds) {
    return guarded([&] {
        auto* rb = static_cast<RefBasis*>(h);
        EriPackedBuildOptions opt;
        opt.schwarz_threshold = schwarz_threshold;
        const EriPackedPlan plan = build_eri_packed_plan_for_G_rys(rb->build.basis, opt);
        const auto t0 = std::chrono::steady_clock::now();
        const EriPackedGData r = build_eri_packed_for_G_rys(plan, opt);
        const auto t1 = std::chrono::steady_clock::now();
        if (r.values.size() != 1) throw std::runtime_error("expected one ERI checksum");
        *checksum = r.values.front();
        if (seconds) *seconds = std::chrono::duration<double>(t1 - t0).count();
    });
}

// EriDirectJKIncrementalState (fock/eri_direct_jk.hpp:41-135) over the
// reference's own plan.
struct RefIncremental {
    std::unique_ptr<EriDirectJKIncrementalState> state;
};

void* ref_incremental_create(void* h, double schwarz_threshold,
                             unsigned long long exact_rebuild_interval,
                             double delta_density_threshold,
                             int use_first_delta_density_threshold,
                             double first_delta_density_threshold) {
    RefIncremental* out = nullptr;
    const int rc = guarded([&] {
        auto* rb = static_cast<RefBasis*>(h);
        EriDirectJKIncrementalOptions o;
        o.base_options.schwarz_threshold = schwarz_threshold;
        o.exact_rebuild_interval = exact_rebuild_interval;
        o.delta_density_threshold = delta_density_threshold;
        o.use_first_delta_density_threshold = use_first_delta_density_threshold != 0;
        o.first_delta_density_threshold = first_delta_density_threshold;
        const EriPackedPlan plan =
            build_eri_packed_plan_for_G_rys(rb->build.basis, o.base_options);
        auto st = std::make_unique<RefIncremental>();
        st->state = std::make_unique<EriDirectJKIncrementalState>(plan, o);
        out = st.release();
    });
    return rc == 0 ? out : nullptr;
}

void ref_incremental_destroy(void* s) { delete static_cast<RefIncremental*>(s); }

// One update; writes the cached G (M x M), the status (1 exact rebuild,
// 2 incremental update, 3 skipped unchanged) and the counters
// [updates, exact_rebuilds, incremental_updates, skipped_updates].
int ref_incremental_update(void* s, const double* density, int force, double* G,
                           int* status, unsigned long long* counters,
                           double* last_delta, double* last_threshold) {
    return guarded([&] {
        auto* st = static_cast<RefIncremental*>(s);
        const std::size_t m = static_cast<std::size_t>(st->state->M());
        std::vector<double> d(density, density + m * m);
        const auto r = st->state->update(d, force != 0);
        *status = static_cast<int>(r);
        const auto& g = st->state->g();
        std::memcpy(G, g.data(), m * m * sizeof(double));
        const auto& c = st->state->counters();
        counters[0] = c.updates;
        counters[1] = c.exact_rebuilds;
        counters[2] = c.incremental_updates;
        counters[3] = c.skipped_updates;
        *last_delta = st->state->last_max_abs_density_delta();
        *last_threshold = st->state->last_effective_density_threshold();
    });
}

// The per-Cartesian-component records of the basis exactly as the reference
// holds them (std::vector<Shell>, core/basis/types.hpp:30-35): centre,
// angular triple, primitive count and the make_shell-normalised primitives
// (exponents and coefficients packed back to back).  Call with null arrays to
// get the component and primitive counts.
int ref_basis_components(void* h, int* n_components, int* n_prims, double* centers,
                         int* ang, int* nprim, double* exps, double* coefs) {
    return guarded([&] {
        const auto& b = static_cast<RefBasis*>(h)->build.basis;
        *n_components = static_cast<int>(b.size());
        int np = 0;
        for (const auto& s : b) np += static_cast<int>(s.primitives.size());
        *n_prims = np;
        if (!centers) return;
        int p = 0;
        for (std::size_t k = 0; k < b.size(); ++k) {
            for (int a = 0; a < 3; ++a) {
                centers[3 * k + a] = b[k].center[a];
                ang[3 * k + a] = b[k].ang[a];
            }
            nprim[k] = static_cast<int>(b[k].primitives.size());
            for (const auto& pr : b[k].primitives) {
                exps[p] = pr.exponent;
                coefs[p] = pr.coefficient;
                ++p;
            }
        }
    });
}

// Wall-clock seconds of `reps` J+K builds (build_coulomb_j followed by
// build_exchange_k) on an already built plan; per-rep times in out_times.
int ref_time_jk(void* h, const double* density, double schwarz_threshold,
                int reps, double* out_times) {
    return guarded([&] {
        namespace fock = tlno::integrals::twoe::fock;
        auto* rb = static_cast<RefBasis*>(h);
        fock::ScreeningOptions opt;
        opt.integral_threshold = schwarz_threshold;
        const fock::DirectPlan plan = fock::build_direct_plan(rb->build.basis, opt);
        const std::size_t m = static_cast<std::size_t>(plan.profile.M);
        std::vector<double> d(density, density + m * m);
        for (int r = 0; r < reps; ++r) {
            const auto t0 = std::chrono::steady_clock::now();
            const auto j = fock::build_coulomb_j(plan, d, opt);
            const auto k = fock::build_exchange_k(plan, d, opt);
            const auto t1 = std::chrono::steady_clock::now();
            out_times[r] = std::chrono::duration<double>(t1 - t0).count();
            if (j.j.empty() || k.k.empty()) throw std::runtime_error("empty");
        }
    });
}

// Contracted spherical ERI block of shells (A B | C D), layout
// [(2La+1)(2Lb+1)] x [(2Lc+1)(2Ld+1)] row-major, following the reference's
// own Schwarz-bound code path (rys_engine.ipp:16194-16241): the raw
// Cartesian Rys/HRR block, then the final pair projectors on both sides.
int ref_eri_sph_block(void* h, int sA, int sB, int sC, int sD, double* out) {
    return guarded([&] {
        auto* rb = static_cast<RefBasis*>(h);
        const auto groups = build_groups_h(rb->build.basis);
        const auto& gA = group_of(groups, sA);
        const auto& gB = group_of(groups, sB);
        const auto& gC = group_of(groups, sC);
        const auto& gD = group_of(groups, sD);
        std::vector<double> cart;
        compute_quartet_block_rys_impl(gA, gB, gC, gD, nullptr, nullptr,
                                       nullptr, nullptr, cart);
        const auto& lp = get_final_sph_pair_projector(gA.L, gB.L);
        const auto& rp = get_final_sph_pair_projector(gC.L, gD.L);
        const std::size_t cols = static_cast<std::size_t>(rp.cart_cols);
        for (int i = 0; i < lp.sph_rows; ++i) {
            for (int j = 0; j < rp.sph_rows; ++j) {
                double v = 0.0;
                for (const auto& l : lp.rows[static_cast<std::size_t>(i)])
                    for (const auto& r : rp.rows[static_cast<std::size_t>(j)])
                        v += l.coeff * r.coeff *
                             cart[static_cast<std::size_t>(l.index) * cols +
                                  static_cast<std::size_t>(r.index)];
                out[static_cast<std::size_t>(i) * rp.sph_rows + j] = v;
            }
        }
    });
}

// Schwarz bound per shell pair, as the reference computes it
// (get_rys_spherical_pair_schwarz_bounds, rys_engine.ipp:16165).  Output is
// indexed by the canonical shell-pair index i*(i+1)/2 + j (i >= j).
int ref_schwarz_pair_max(void* h, double* out) {
    return guarded([&] {
        auto* rb = static_cast<RefBasis*>(h);
        const auto bd = get_basis_data_h_shared(rb->build.basis);
        const auto& sb = get_rys_spherical_pair_schwarz_bounds(*bd);
        for (std::size_t pg = 0; pg < bd->pair_groups.size(); ++pg) {
            int a = bd->pair_groups[pg].first;
            int b = bd->pair_groups[pg].second;
            if (a < b) std::swap(a, b);
            out[static_cast<std::size_t>(a) * (a + 1) / 2 + b] =
                sb.pair_group_max[pg];
        }
    });
}

// Boys function copies used by the reference.
double ref_boys_single(int n, double x) {
    return tlno::core::math::boys_single(n, x);
}
void ref_boys_r000_all(int max_n, double x, double p, double* out) {
    tlno::core::math::boys_r000_all(max_n, x, p, out);
}
double ref_boys_hgp(int m, double x) { return boys_eval_hgp(m, x); }

// Rys roots (t^2) and weights: production table path and the accurate
// generator that seeds it.
void ref_rys_roots(int n, double t, double* roots, double* weights) {
    rys_roots_weights(n, t, roots, weights);
}
void ref_rys_roots_accurate(int n, double t, double* roots, double* weights) {
    rys_roots_weights_accurate(n, t, roots, weights);
}

}  // extern "C"
