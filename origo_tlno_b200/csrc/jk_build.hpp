// Internal J/K build machinery shared by the C-ABI translation units
// (capi.cpp, incremental.cpp): option validation, the per-build
// specification and the enqueue of one screened J/K build.
#pragma once

#include <cstdint>
#include <cstring>
#include <functional>
#include <memory>
#include <string>

#include "context.hpp"
#include "plan.hpp"

namespace tlno_gpu {

// Runs f and turns any exception into a status code and the calling
// thread's last-error text.
int run_guarded(const std::function<void()>& f);

void set_device(int device);

inline bool finite_bits(double v) {
    std::uint64_t bits;
    std::memcpy(&bits, &v, sizeof(bits));
    return (bits & 0x7ff0000000000000ull) != 0x7ff0000000000000ull;
}

// Finite, non-negative thresholds (the reference's messages).
void validate_screening(const tlno_gpu_screening& o);
// Option combinations the reference rejects at build time.
void validate_build_combination(const tlno_gpu_screening& o);
// Finite and symmetric within 128 eps (direct_build.ipp:25-96), host buffer.
void validate_density_host(const double* D, int M);

// What one J/K build computes and how it is screened.
struct BuildSpec {
    bool want_j = true, want_k = true, mixed = false;
    double mixed_threshold = 1e-9;
    int den_mode = 0;      // 0 off; 1 J and K predicates apart; 2 fused G predicate
    double den_thr = 0.0;  // density_threshold
    double fs_thr2 = 0.0;  // primitive FASTSCHWARZ threshold squared
};
BuildSpec spec_from(const tlno_gpu_screening& o, bool want_j, bool want_k, bool mixed, bool fused_g);

// Enqueues one J/K build over device buffers on stream s: J, K zeroed, the
// class kernels, the final symmetrisation.  A density-screened build needs
// ensure_density_tables(plan) first.
void enqueue_jk(Plan2e& plan, const Tuning& tune, const BuildSpec& spec, const double* dD, double* dJ,
                double* dK, long long total, int M_single, double* d_dmax, float* dD32, cudaStream_t s,
                StreamFan* fan = nullptr);

// Two-electron plan of a context's basis for the shell-level screen of o.
std::unique_ptr<Plan2e> make_plan(const tlno_gpu_context* ctx, const tlno_gpu_screening& o);

void ensure_work(JkWork& w, long long total);

}  // namespace tlno_gpu
